// k_mom3d.cu - internal-mode (3-D) momentum kernels of INTERNAL_STEP
// (FVCOM_source/internal_step.F:29-1607): ADJUST2D3D, BCOND_GCN(5/8), BOTTOM_ROUGHNESS,
// ADVECTION_EDGE_GCN, BAROPG, VERTVL_EDGE, VISCOF_H, ADV_UV_EDGE_GCN, VDIF_UV,
// BCOND_GCN(3), WREAL.
//
// Thread shapes: column kernels (vertical prefix sums and tridiagonal solves) run one
// thread per cell or node looping over the layers; layer-parallel gathers run on 32 x 8
// blocks (32 consecutive cells/nodes of one layer per warp, 8 layers per block) so a warp
// reads one coalesced 256-byte row of each field and the 2-D mesh metrics it needs are
// shared by the eight warps through L1.
#include "fvg_model.h"

// The FP32 instantiations of the precision form's flux kernels are compiled from this
// same source a second time with -DFVG_F32_TU and multiply-add contraction (build.py),
// into namespace fvg_f32; the FP64 translation unit forwards their launches there.
#ifdef FVG_F32_TU
namespace fvg_f32 {
using namespace fvg;
#else
namespace fvg {
#endif

#define ONE_THIRD (1.0 / 3.0)
constexpr int kMaxKB = 64;
__device__ __constant__ double dAlpha3[5] = {0.0, 0.25, 1.0 / 3.0, 0.5, 1.0};

static inline int nblk(int n, int b) { return (n + b - 1) / b; }


// River clamp / tangential projection (bcond_gcn.F:345-405, 443-499, 552-608).
__device__ inline void bc_solid3(const Dev& P, int i, double& uu, double& vv) {
  int rj = P.cell_bcriv[i];
  if (rj > 0) {
    double ca = P.cos_angleq[rj], sa = P.sin_angleq[rj];
    double untmp = uu * ca + vv * sa;
    double vntmp = -uu * sa + vv * ca;
    untmp = fmax(untmp, 0.0);
    uu = untmp * ca - vntmp * sa;
    vv = untmp * sa + vntmp * ca;
  } else if (!P.gcy) {  // GCY (bcond_gcy.F) keeps the river clamp only
    double sa = P.sin_alpha[i], ca = P.cos_alpha[i];
    double ui = uu * (sa * sa) - vv * sa * ca;
    double vi = -uu * sa * ca + vv * (ca * ca);
    uu = ui;
    vv = vi;
  }
}

// -------------------------------------------------------------------------------------
// ADJUST2D3D(1) (adjust2d3d.F:57-63), BCOND_GCN(5,0) (bcond_gcn.F:537-611),
// BCOND_GCN(8,0) wind (bcond_gcn.F:661-683), BOTTOM_ROUGHNESS cell part (brough.F:76-193).
// One thread per cell column.
// -------------------------------------------------------------------------------------
__global__ void k_cell_pre(const Dev P, int parts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  const int KBM1 = P.KBM1;
  if (parts & CP_ADJUST1) {
    double uac = 0.0, vac = 0.0;
    for (int k = 1; k <= KBM1; ++k) uac = uac + P.u[C3(P, i, k)] * P.dz1[C3(P, i, k)];
    for (int k = 1; k <= KBM1; ++k) vac = vac + P.v[C3(P, i, k)] * P.dz1[C3(P, i, k)];
    double du = 1.0 * (P.ua[i] - uac), dv = 1.0 * (P.va[i] - vac);
    for (int k = 1; k <= KBM1; ++k) {
      P.u[C3(P, i, k)] = P.u[C3(P, i, k)] + du;
      P.v[C3(P, i, k)] = P.v[C3(P, i, k)] + dv;
    }
  }
  if (parts & CP_BC5) {
    int b = P.isbce[i];
    if (b == 3 || b == 1) {
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = C3(P, i, k);
        double uu = P.u[q], vv = P.v[q];
        if (b == 3) {
          if (!P.gcy) { uu = 0.0; vv = 0.0; }
        } else {
          bc_solid3(P, i, uu, vv);
        }
        P.u[q] = uu;
        P.v[q] = vv;
      }
    }
  }
  if ((parts & CP_BCOND8) && P.have_wind) {
    double ramp = ramp_int(P);
    P.wusurf[i] = -P.wsx[i] * ramp * 0.001;
    P.wvsurf[i] = -P.wsy[i] * ramp * 0.001;
  }
  if (parts & CP_BROUGH) {
    const double VK2 = 0.160;
    double zb = P.zz1[C3(P, i, KBM1)] - P.z1[C3(P, i, P.KB)];
    double lg = (P.dt1[i] > 3.0) ? log(zb * P.dt1[i] / P.cc_z0b[i]) : log(zb * 3.0 / P.cc_z0b[i]);
    double cbc = VK2 / (lg * lg);
    if (cbc < P.cbcmin) cbc = P.cbcmin;
    P.cbc[i] = cbc;
    double ub = P.u[C3(P, i, KBM1)], vb = P.v[C3(P, i, KBM1)];
    double btps = cbc * sqrt(ub * ub + vb * vb);
    double wu = -btps * ub, wv = -btps * vb;
    double cff = 0.75 * P.dz1[C3(P, i, KBM1)] * P.d1[i];
    wu = (wu >= 0.0 ? 1.0 : -1.0) * fmin(fabs(wu), fabs(ub * cff / P.dti));
    wv = (wv >= 0.0 ? 1.0 : -1.0) * fmin(fabs(wv), fabs(vb * cff / P.dti));
    P.wubot[i] = wu;
    P.wvbot[i] = wv;
    P.taubm[i] = sqrt(wu * wu + wv * wv);
  }
}

// Least-squares gradient of U,V on layer k (advection_edge_gcn.F:533-536).
template <typename R>
struct G3 {
  R ux, uy, vx, vy;
};
template <typename R>
__device__ inline G3<R> grad3(const Dev& P, int c, const double* U, const double* V) {
  typedef Mesh<R> Mh;
  int k1, k2, k3;
  R A[4], B[4];
  lsq_coef<R>(P, c, k1, k2, k3, A, B);
  const R a1 = A[0], a2 = A[1], a3 = A[2], a4 = A[3], b1 = B[0], b2 = B[1], b3 = B[2], b4 = B[3];
  R u0 = (R)U[c], u1 = (R)U[k1], u2 = (R)U[k2], u3 = (R)U[k3];
  R v0 = (R)V[c], v1 = (R)V[k1], v2 = (R)V[k2], v3 = (R)V[k3];
  if (P.gcy && (k1 == 0 || k2 == 0 || k3 == 0)) {
    double gu, gv;
    if (k1 == 0) { ghost_uv(P, U, V, c, 1, gu, gv); u1 = (R)gu; v1 = (R)gv; }
    if (k2 == 0) { ghost_uv(P, U, V, c, 2, gu, gv); u2 = (R)gu; v2 = (R)gv; }
    if (k3 == 0) { ghost_uv(P, U, V, c, 3, gu, gv); u3 = (R)gu; v3 = (R)gv; }
  }
  G3<R> g;
  g.ux = a1 * u0 + a2 * u1 + a3 * u2 + a4 * u3;
  g.uy = b1 * u0 + b2 * u1 + b3 * u2 + b4 * u3;
  g.vx = a1 * v0 + a2 * v1 + a3 * v2 + a4 * v3;
  g.vy = b1 * v0 + b2 * v1 + b3 * v2 + b4 * v3;
  return g;
}

// Horizontal flux of one edge on one layer (advection_edge_gcn.F:449-603 and
// adv_uv_edge_gcn.F:580-779 share this body), evaluated in R.
template <typename R>
struct EdgeFlux {
  R xadv, yadv, fxx, fyy, viscof;
};

template <typename R>
__device__ inline G3<R> load_g3(const Dev& P, int c, int k) {
  size_t q = C3(P, c, k);
  G3<R> g;
  if constexpr (sizeof(R) == 4) {
    const float4 a = P.f.g34[q];
    g.ux = a.x;
    g.uy = a.y;
    g.vx = a.z;
    g.vy = a.w;
  } else {
    g.ux = P.g3[0][q];
    g.uy = P.g3[1][q];
    g.vx = P.g3[2][q];
    g.vy = P.g3[3][q];
  }
  return g;
}

// Least-squares gradient of U, V of every cell and layer (the COFA1..COFA8 inputs of
// advection_edge_gcn.F:533-548 and adv_uv_edge_gcn.F:704-719), evaluated once per cell.
template <typename R>
__global__ void __launch_bounds__(256) k_grad3(const Dev P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  int kb, ke;
  col_range(P, 1, P.KBM1, kb, ke);
  for (int k = kb; k <= ke; ++k) {
    G3<R> g = grad3<R>(P, i, P.u + C3(P, 0, k), P.v + C3(P, 0, k));
    size_t q = C3(P, i, k);
    if constexpr (sizeof(R) == 4) {
      P.f.g34[q] = make_float4(g.ux, g.uy, g.vx, g.vy);
    } else {
      P.g3[0][q] = g.ux;
      P.g3[1][q] = g.uy;
      P.g3[2][q] = g.vx;
      P.g3[3][q] = g.vy;
    }
  }
}

// Slope limiters UALFA, VALFA of each cell and layer for the limited ADVECTION and ADV_UV
// (advection_edge_gcn.F:118-259, adv_uv_edge_gcn.F:152-330): the cell's three edges with a
// wet side on the layer, from the cell's own gradient and the two cells' U, V.
template <typename R>
__global__ void __launch_bounds__(256) k_alfa3(const Dev P) {
  typedef Mesh<R> Mh;
  const int c = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (c > P.N) return;
  const size_t n1 = P.N + 1;
  int kb, ke;
  col_range(P, 1, P.KBM1, kb, ke);
  for (int k = kb; k <= ke; ++k) {
    const double* U = P.u + C3(P, 0, k);
    const double* V = P.v + C3(P, 0, k);
    const G3<R> g = load_g3<R>(P, c, k);
    R au = (R)1, av = (R)1;
    for (int s = 0; s < 3; ++s) {
      const size_t q = (size_t)s * n1 + c;
      const int ia = P.ce_ia[q], ib = P.ce_ib[q];
      if (!(P.iswetct[ia] * P.iswetc[ia] == 1 || P.iswetct[ib] * P.iswetc[ib] == 1)) continue;
      const bool a_side = (P.ce_code[q] & 1) == 0;
      const R x = a_side ? Mh::s_xoa(P, q) : Mh::s_xob(P, q);
      const R y = a_side ? Mh::s_yoa(P, q) : Mh::s_yob(P, q);
      lim_alfa<R>(fabs((R)U[ia] - (R)U[ib]), g.ux * x + g.uy * y, au);
      lim_alfa<R>(fabs((R)V[ia] - (R)V[ib]), g.vx * x + g.vy * y, av);
    }
    Mh::alfa3(P, 0)[C3(P, c, k)] = au;
    Mh::alfa3(P, 1)[C3(P, c, k)] = av;
  }
}

// q: the edge's slot in the cell slot table (offsets and DLTXC/DLTYC of the edge).
// The cell's own side of its edges on one layer, loaded once for its three edges.
template <typename R>
struct Own3 {
  G3<R> g;
  R u, v, art, cc;
};

// OWN (FP32 form, no limiter): `own` holds the values of the cell on the edge's `side`
// (0: IA, 1: IB), so that only the other cell is gathered.
template <typename R, bool LIM, bool OWN = false>
__device__ inline EdgeFlux<R> edge_flux3(const Dev& P, size_t q, int ia, int ib, int k, R dij, bool exflux_form,
                                         const Own3<R>& own = Own3<R>(), int side = 0) {
  typedef Mesh<R> Mh;
  const R half = (R)0.5, one = (R)1.0;
  const double* U = P.u + C3(P, 0, k);
  const double* V = P.v + C3(P, 0, k);
  const auto G = Mh::s_geo(P, q);  // XOA, YOA, XOB, YOB
  R xija = G.x, yija = G.y;
  R xijb = G.z, yijb = G.w;
  G3<R> ga, gb;
  R uij1, vij1, uij2, vij2;
  R arta, artb, cca, ccb;
  if constexpr (!LIM) {
    if constexpr (OWN) {
      const int o = side == 0 ? ib : ia;
      const G3<R> go = load_g3<R>(P, o, k);
      const R uo = (R)U[o], vo = (R)V[o];
      ga = side == 0 ? own.g : go;
      gb = side == 0 ? go : own.g;
      const R ua = side == 0 ? own.u : uo, va = side == 0 ? own.v : vo;
      const R ub = side == 0 ? uo : own.u, vb = side == 0 ? vo : own.v;
      uij1 = ua + ga.ux * xija + ga.uy * yija;
      vij1 = va + ga.vx * xija + ga.vy * yija;
      uij2 = ub + gb.ux * xijb + gb.uy * yijb;
      vij2 = vb + gb.vx * xijb + gb.vy * yijb;
      const R arto = Mh::art(P, o), cco = Mh::cc_hvc(P, o);
      arta = side == 0 ? own.art : arto;
      artb = side == 0 ? arto : own.art;
      cca = side == 0 ? own.cc : cco;
      ccb = side == 0 ? cco : own.cc;
    } else {
      ga = load_g3<R>(P, ia, k);
      uij1 = (R)U[ia] + ga.ux * xija + ga.uy * yija;
      vij1 = (R)V[ia] + ga.vx * xija + ga.vy * yija;
      gb = load_g3<R>(P, ib, k);
      uij2 = (R)U[ib] + gb.ux * xijb + gb.uy * yijb;
      vij2 = (R)V[ib] + gb.vx * xijb + gb.vy * yijb;
      arta = Mh::art(P, ia);
      artb = Mh::art(P, ib);
      cca = Mh::cc_hvc(P, ia);
      ccb = Mh::cc_hvc(P, ib);
    }
  } else {
    arta = Mh::art(P, ia);
    artb = Mh::art(P, ib);
    cca = Mh::cc_hvc(P, ia);
    ccb = Mh::cc_hvc(P, ib);
    ga = load_g3<R>(P, ia, k);
    gb = load_g3<R>(P, ib, k);
    const size_t qa = C3(P, ia, k), qb = C3(P, ib, k);
    lim_faces<R>(P.limiter, (R)U[ia], (R)U[ib], ga.ux * xija + ga.uy * yija, gb.ux * xijb + gb.uy * yijb,
                 Mh::alfa3(P, 0)[qa], Mh::alfa3(P, 0)[qb], uij1, uij2);
    lim_faces<R>(P.limiter, (R)V[ia], (R)V[ib], ga.vx * xija + ga.vy * yija, gb.vx * xijb + gb.vy * yijb,
                 Mh::alfa3(P, 1)[qa], Mh::alfa3(P, 1)[qb], vij1, vij2);
  }
  R uij = half * (uij1 + uij2);
  R vij = half * (vij1 + vij2);
  R viscof1 = arta * sqrt(ga.ux * ga.ux + ga.vy * ga.vy + half * ((ga.uy + ga.vx) * (ga.uy + ga.vx)));
  R viscof2 = artb * sqrt(gb.ux * gb.ux + gb.vy * gb.vy + half * ((gb.uy + gb.vx) * (gb.uy + gb.vx)));
  R viscof = ((R)P.fact * half * (viscof1 * cca + viscof2 * ccb) + (R)P.fm1 * half * (cca + ccb)) / (R)P.hprnu;
  R txx = (ga.ux + gb.ux) * viscof;
  R tyy = (ga.vy + gb.vy) * viscof;
  R txy = half * (ga.uy + gb.uy + ga.vx + gb.vx) * viscof;
  const auto DD = Mh::s_dd(P, q);
  const R dltxc = DD.x, dltyc = DD.y;
  EdgeFlux<R> f;
  f.fxx = dij * (txx * dltyc - txy * dltxc);
  f.fyy = dij * (txy * dltyc - tyy * dltxc);
  f.viscof = viscof;
  if (exflux_form) {
    // adv_uv_edge_gcn.F:730, 752-753
    R exflux = dij * (-uij * dltyc + vij * dltxc);
    R sg = fsign1(exflux);
    f.xadv = exflux * ((one - sg) * uij2 + (one + sg) * uij1) * half;
    f.yadv = exflux * ((one - sg) * vij2 + (one + sg) * vij1) * half;
  } else {
    // advection_edge_gcn.F:559, 576-577
    R un = vij * dltxc - uij * dltyc;
    R sg = fsign1(un);
    f.xadv = dij * un * ((one - sg) * uij2 + (one + sg) * uij1) * half;
    f.yadv = dij * un * ((one - sg) * vij2 + (one + sg) * vij1) * half;
  }
  return f;
}

// River momentum source on one cell and layer (advection_edge_gcn.F:674-708).
__device__ inline void river3(const Dev& P, int i, int k, double& x, double& y) {
  for (int q = P.cell_riv_ptr[i]; q < P.cell_riv_ptr[i + 1]; ++q) {
    int ii = P.cell_riv[q] >> 1;
    double vq = P.vqdist[(size_t)(k - 1) * (P.numqbc + 1) + ii];
    double vlctyq = P.qdis[ii] / P.qarea[ii];
    double temp;
    if (P.river_location == 0) {
      int j = P.inodeq[ii];
      temp = 0.5 * P.qdis[ii] * vq * vq * vlctyq / P.dz[N3(P, j, k)];
    } else {
      int i1 = P.icellq[ii];
      temp = P.qdis[ii] * vq * vq * vlctyq / P.dz1[C3(P, i1, k)];
    }
    x = x - temp * P.cos_angleq[ii];
    y = y - temp * P.sin_angleq[ii];
  }
}

// The end of ADVECTION_EDGE_GCN for cell i on layer k once its three edges are summed
// into xr, yr (advection_edge_gcn.F:674-708): wet mask, open-boundary cells, rivers.
template <typename R>
__device__ inline void advection3d_tail(const Dev& P, int i, int k, R xr, R yr) {
  double x = (double)xr, y = (double)yr;
  double w = (double)(P.iswetct[i] * P.iswetc[i]);
  x = x * w;
  y = y * w;
  if (P.isbce[i] == 2) { x = 0.0; y = 0.0; }
  river3(P, i, k, x, y);
  P.advx[C3(P, i, k)] = x;
  P.advy[C3(P, i, k)] = y;
}

// -------------------------------------------------------------------------------------
// ADVECTION_EDGE_GCN (advection_edge_gcn.F:397-708): per cell and layer, the cell's three
// edges in ascending edge number.
// -------------------------------------------------------------------------------------
template <typename R, bool LIM>
__global__ void __launch_bounds__(256, (sizeof(R) == 4 && !LIM) ? 4 : 1) k_advection3d(const Dev P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  int kb, ke;
  col_range(P, 1, P.KBM1, kb, ke);
  for (int k = kb; k <= ke; ++k) {
  const size_t n1 = P.N + 1;
  const R epor = (R)P.epor[i], three = (R)3.0;
  R xr = 0, yr = 0;
    // FP32 form without a limiter: the cell's own side of its three edges, once
    constexpr bool OWN = !LIM && sizeof(R) == 4;
    Own3<R> own;
    if constexpr (OWN) {
      own.g = load_g3<R>(P, i, k);
      own.u = (R)P.u[C3(P, i, k)];
      own.v = (R)P.v[C3(P, i, k)];
      own.art = Mesh<R>::art(P, i);
      own.cc = Mesh<R>::cc_hvc(P, i);
    }
  for (int s = 0; s < 3; ++s) {
    const size_t q = (size_t)s * n1 + i;
    const int4 ci = P.ce_i4[q];  // {code, IA, IB, J1}
    const int code = ci.x, side = code & 1, isbc = (code >> 1) & 1;
    const int ia = ci.y, ib = ci.z;
    if (!(P.iswetct[ia] * P.iswetc[ia] == 1 || P.iswetct[ib] * P.iswetc[ib] == 1)) continue;
    const int j1 = ci.w, j2 = P.ce_j2[q];
    R dij = (R)(0.5 * (P.dt[j1] * P.dz[N3(P, j1, k)] + P.dt[j2] * P.dz[N3(P, j2, k)]));
    EdgeFlux<R> f = edge_flux3<R, LIM, OWN>(P, q, ia, ib, k, dij, false, own, side);
    R isb = (R)isbc;
    R tp = (R)((double)(float)(1 - isbc) * P.epor[i]);
    // viscous part: GCN (fxx + 3 fxx ISBC) EPOR; GCY (advection_edge_gcy.F) fxx TPA
    const R vfx = P.gcy ? f.fxx * tp : (f.fxx + three * f.fxx * isb) * epor;
    const R vfy = P.gcy ? f.fyy * tp : (f.fyy + three * f.fyy * isb) * epor;
    if (side == 0) {
      xr = xr + f.xadv * tp + vfx;
      yr = yr + f.yadv * tp + vfy;
    } else {
      xr = xr - f.xadv * tp - vfx;
      yr = yr - f.yadv * tp - vfy;
    }
  }
  advection3d_tail<R>(P, i, k, xr, yr);
  }
}

// -------------------------------------------------------------------------------------
// BAROPG, sigma levels (baropg.F:56-161), then the vertical sums of ADVX/DRHOX into the
// 2-D forcing (internal_step.F:374-384).  One thread per cell column; the density
// anomalies RHO1-RMEAN1 of the three nodes are formed on the fly and the cell's
// RHO = (RHO-RMEAN)+RMEAN round trip is written back as the reference does.
// -------------------------------------------------------------------------------------
__global__ void k_baropg(const Dev P, int do_baropg, int do_sums) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  const size_t n1 = P.N + 1;
  const int KBM1 = P.KBM1;
  if (do_baropg) {
    int nvv[4] = {0, P.nv[i], P.nv[n1 + i], P.nv[2 * n1 + i]};
    double ramp = ramp_int(P);
    bool active = P.iswetct[i] * P.iswetc[i] == 1 &&
                  (P.h[nvv[1]] > P.static_ssh_adj || P.h[nvv[2]] > P.static_ssh_adj || P.h[nvv[3]] > P.static_ssh_adj);
    double dx[4], dyv[4], dij[4];
    for (int j = 1; j <= 3; ++j) {
      int J1 = j + 1 - ((j + 1) / 4) * 3, J2 = j + 2 - ((j + 2) / 4) * 3;
      dyv[j] = P.vy[nvv[J1]] - P.vy[nvv[J2]];
      dx[j] = P.vx[nvv[J2]] - P.vx[nvv[J1]];
      dij[j] = 0.5 * (P.dt[nvv[J1]] + P.dt[nvv[J2]]);
    }
    double rprev[4] = {0, 0, 0, 0}, d1p[4] = {0, 0, 0, 0};
    double d2 = 0.0, rhoc_prev = 0.0, zprev = 0.0;
    double dt1 = P.dt1[i], ge = P.grav_e[i];
    // Layers in batches of kB: every input of a batch is loaded before its vertical
    // integrals run, so the loads of a batch are in flight together.
    constexpr int kB = 4;
    for (int k0 = 1; k0 <= KBM1; k0 += kB) {
      double dn[kB][4], rhoc[kB], zz[kB], dz[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const int k = k0 + b;
        if (k > KBM1) break;
        for (int j = 1; j <= 3; ++j) {
          const size_t q = N3(P, nvv[j], k);
          dn[b][j] = P.rho1[q] - P.rmean1[q];
        }
        const size_t c = C3(P, i, k);
        rhoc[b] = P.rho[c] - P.rmean[c];
        zz[b] = P.zz1[c];
        dz[b] = P.dz1[c];
      }
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const int k = k0 + b;
        if (k > KBM1) break;
        double rij[4];
        for (int j = 1; j <= 3; ++j) {
          int J1 = j + 1 - ((j + 1) / 4) * 3, J2 = j + 2 - ((j + 2) / 4) * 3;
          rij[j] = 0.5 * (dn[b][J1] + dn[b][J2]);
        }
        if (k == 1) {
          for (int j = 1; j <= 3; ++j) d1p[j] = rij[j] * (-zz[b]);
          d2 = 0.0;
        } else {
          const double zkm = zprev, zk = zz[b];
          for (int j = 1; j <= 3; ++j) d1p[j] = 0.5 * (rprev[j] + rij[j]) * (zkm - zk) + d1p[j];
          d2 = d2 + 0.5 * (zkm + zk) * (rhoc[b] - rhoc_prev);
        }
        double drhox = 0.0, drhoy = 0.0;
        if (active) {
          for (int j = 1; j <= 3; ++j) {
            double drho1 = dyv[j] * d1p[j] * dt1;
            double drho2 = dyv[j] * dij[j] * d2;
            drhox = drhox + drho1 + drho2;
            drho1 = dx[j] * d1p[j] * dt1;
            drho2 = dx[j] * dij[j] * d2;
            drhoy = drhoy + drho1 + drho2;
          }
        }
        const size_t c = C3(P, i, k);
        P.drhox[c] = drhox * dt1 * dz[b] * ge * ramp;
        P.drhoy[c] = drhoy * dt1 * dz[b] * ge * ramp;
        for (int j = 1; j <= 3; ++j) rprev[j] = rij[j];
        rhoc_prev = rhoc[b];
        zprev = zz[b];
      }
    }
    for (int k = 1; k <= P.KB; ++k) {
      size_t q = C3(P, i, k);
      P.rho[q] = (P.rho[q] - P.rmean[q]) + P.rmean[q];
    }
  }
  if (do_sums) {
    double ax = 0.0, ay = 0.0, rx = 0.0, ry = 0.0;
    for (int k = 1; k <= KBM1; ++k) {
      size_t q = C3(P, i, k);
      ax = ax + P.advx[q];
      ay = ay + P.advy[q];
      rx = rx + P.drhox[q];
      ry = ry + P.drhoy[q];
    }
    P.adx2d[i] = ax;
    P.ady2d[i] = ay;
    P.drx2d[i] = rx;
    P.dry2d[i] = ry;
  }
}

// internal_step.F:395-416: UARD=VARD=EGF=0, UARD_OBCN=0 before the external loop.
__global__ void k_int_reset(const Dev P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= P.N) { P.uard[i] = 0.0; P.vard[i] = 0.0; }
  if (i <= P.M) P.egf[i] = 0.0;
  if (i >= 1 && i <= P.iobcn) P.uard_obcn[i] = 0.0;
}

// ADJUST2D3D(2) (adjust2d3d.F:65-92), one thread per cell column (AJ_ADJUST), and the
// EXFLUX of VERTVL_EDGE (vertvl_edge.F:68-90) for the cell's three half-edges and every
// layer from the adjusted U, V (AJ_HE_FLUX): DT1*DZ1*(-U*DLTYE + V*DLTXE) into he_vflux,
// which the node kernel sums in half-edge order.
__global__ void k_adjust2(const Dev P, int parts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > P.N) return;
  const bool adj = parts & AJ_ADJUST;
  double ud = 0.0, vd = 0.0;
  if (adj) {
    ud = P.uard[i] / (double)(float)P.isplit;
    vd = P.vard[i] / (double)(float)P.isplit;
    P.uard[i] = ud;
    P.vard[i] = vd;
  }
  if (i == 0) return;
  const bool wet = adj && P.iswetct[i] * P.iswetc[i] == 1;
  const double dt1 = P.dt1[i];
  double ut = 0.0, vt = 0.0;
  if (wet) {
    for (int k = 1; k <= P.KBM1; ++k) {
      size_t q = C3(P, i, k);
      ut = ut + P.u[q] * P.dz1[q];
      vt = vt + P.v[q] * P.dz1[q];
    }
    ut = ut * dt1;
    vt = vt * dt1;
  }
  if (!(parts & AJ_HE_FLUX)) {
    if (!wet) return;
    for (int k = 1; k <= P.KBM1; ++k) {
      size_t q = C3(P, i, k);
      P.u[q] = P.u[q] - (ut - ud) / dt1;
      P.v[q] = P.v[q] - (vt - vd) / dt1;
    }
    return;
  }
  double dy[3], dx[3];
  for (int s = 0; s < 3; ++s) {
    const size_t pos = (size_t)s * P.ns + i;
    dy[s] = Mesh<double>::hg(P, 1, pos);
    dx[s] = Mesh<double>::hg(P, 0, pos);
  }
  for (int k = 1; k <= P.KBM1; ++k) {
    size_t q = C3(P, i, k);
    double uu = P.u[q], vv = P.v[q];
    if (wet) {
      uu = uu - (ut - ud) / dt1;
      vv = vv - (vt - vd) / dt1;
      P.u[q] = uu;
      P.v[q] = vv;
    }
    const double dij = dt1 * P.dz1[q];
    double* F = P.he_vflux + (size_t)(k - 1) * P.ncvs + i;
    for (int s = 0; s < 3; ++s) F[(size_t)s * P.ns] = dij * (-uu * dy[s] + vv * dx[s]);
  }
}

// -------------------------------------------------------------------------------------
// VERTVL_EDGE horizontal divergence (vertvl_edge.F:68-220): per node and layer, the
// node's half-edges in ascending order.  Result in the scratch field.
// -------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_vertvl_flux(const Dev P) {
  // One thread per (node, layer); the 8 layer threads of a node share its list entries
  // in L1, and the entries of 32 consecutive nodes arrive in one load.
  int i = blockIdx.x * 32 + threadIdx.x + 1;
  int k = blockIdx.y * 8 + threadIdx.y + 1;
  if (i > P.M || k > P.KBM1) return;
  {
  double x = 0.0;
  if (P.isonb[i] != 2) {
    const double* F = P.he_vflux + (size_t)(k - 1) * P.ncvs;
    const int* L = P.node_vpos_ell + i;
    const size_t ms = P.ms;
    const int n = P.node_he_ptr[i + 1] - P.node_he_ptr[i];
    int j = 0;
    for (; j + 4 <= n; j += 4) {
      const int e0 = L[j * ms], e1 = L[(j + 1) * ms], e2 = L[(j + 2) * ms], e3 = L[(j + 3) * ms];
      const double f0 = F[e0 >> 1], f1 = F[e1 >> 1], f2 = F[e2 >> 1], f3 = F[e3 >> 1];
      x = (e0 & 1) ? x + f0 : x - f0;
      x = (e1 & 1) ? x + f1 : x - f1;
      x = (e2 & 1) ? x + f2 : x - f2;
      x = (e3 & 1) ? x + f3 : x - f3;
    }
    for (; j < n; ++j) {
      const int e = L[j * ms];
      const double f = F[e >> 1];
      x = (e & 1) ? x + f : x - f;
    }
  }
  for (int q = P.node_riv_ptr[i]; q < P.node_riv_ptr[i + 1]; ++q) {
    int r = P.node_riv[q];
    int j = r >> 1;
    double vq = P.vqdist[(size_t)(k - 1) * (P.numqbc + 1) + j];
    if (P.river_location == 0)
      x = x - P.qdis[j] * vq;
    else
      x = x - P.qdis[j] * P.rdisq[(size_t)(r & 1) * (P.numqbc + 1) + j] * vq;
  }
  P.scr_xflux[N3(P, i, k)] = x;
  }
}

// -------------------------------------------------------------------------------------
// VERTVL_EDGE vertical integration and mass-conservation adjustment
// (vertvl_edge.F:236-539), WD_UPDATE(2) (mod_wd.F:311-317), the RHO1 round trip of BAROPG
// (baropg.F:56,160) and E2N2D of the bottom stress (brough.F:193-206).  Node columns.
// -------------------------------------------------------------------------------------
__global__ void k_vertvl_col(const Dev P, int parts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  const int KB = P.KB, KBM1 = P.KBM1;
  if (parts & VC_WTS) {
    const double ROFVROS = 0.9775171065;
    double wb = 0.0 / P.art1[i];
    double wk = -(0.0 + 0.0) * ROFVROS;
    P.wts[N3(P, i, 1)] = wk;
    if (P.iswetnt[i] * P.iswetn[i] == 1) {
      double dd = P.d[i] - P.dt[i];
      for (int k = 1; k <= KBM1; ++k) {
        wk = wk + P.scr_xflux[N3(P, i, k)] / P.art1[i] + P.dz[N3(P, i, k)] * dd / P.dti;
        P.wts[N3(P, i, k + 1)] = wk;
      }
    } else {
      for (int k = 1; k <= KBM1; ++k) P.wts[N3(P, i, k + 1)] = 0.0;
      wk = 0.0;
    }
    double wkb = wk;
    if (fabs(wkb - wb) > 1.0e-8 && P.isonb[i] != 2) {
      double tmp1 = P.elf[i] * (double)(float)KBM1 - (wkb - wb) * P.dti / P.dz[N3(P, i, 1)];
      tmp1 = tmp1 / (double)(float)KBM1;
      P.dtfa[i] = tmp1 + P.h[i];
      for (int k = 2; k <= KB; ++k) {
        double cur = P.wts[N3(P, i, k)];
        double wkb_now = (k == KB) ? cur : wkb;
        P.wts[N3(P, i, k)] = cur - (double)((float)(k - 1) / (float)KBM1) * (wkb_now - wb);
      }
    }
  }
  if ((parts & VC_WD2) && P.wetting_drying_on) {
    if (P.dtfa[i] - P.min_depth <= 1.0e-5) P.iswetn[i] = 0;
  }
  if (parts & VC_RHO_ROUNDTRIP) {
    for (int k = 1; k <= KBM1; ++k) {
      size_t q = N3(P, i, k);
      P.rho1[q] = (P.rho1[q] - P.rmean1[q]) + P.rmean1[q];
    }
  }
  if (parts & VC_BOT_NODE) {
    double su = 0.0, sv = 0.0;
    int nt = P.ntve[i];
    for (int j = 1; j <= nt; ++j) {
      int c = P.nbve[(size_t)(j - 1) * (P.M + 1) + i];
      su = su + P.wubot[c];
      sv = sv + P.wvbot[c];
    }
    double fn = (double)(float)nt;
    su = su / fn;
    sv = sv / fn;
    P.wubot_n[i] = su;
    P.wvbot_n[i] = sv;
    P.taubm_n[i] = sqrt(su * su + sv * sv);
  }
}

// -------------------------------------------------------------------------------------
// W = N2E(WTS)*ISWETC (vertvl_edge.F:552-563) on cells, and VISCOF_H (viscofh.F:58-122)
// on nodes, one thread per (entity, layer).
// -------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_w_viscofh(const Dev P, int do_w, int do_visc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int kb, ke;
  col_range(P, 1, P.KB, kb, ke);
  for (int k = kb; k <= ke; ++k) {
  const size_t n1 = P.N + 1, m1 = P.M + 1;
  if (do_w && i <= P.N) {
    double w = ONE_THIRD * (P.wts[N3(P, P.nv[i], k)] + P.wts[N3(P, P.nv[n1 + i], k)] + P.wts[N3(P, P.nv[2 * n1 + i], k)]);
    P.w[C3(P, i, k)] = (double)(float)P.iswetc[i] * w;
  }
  if (do_visc && i <= P.M && k <= P.KBM1) {
    const double* U = P.u + C3(P, 0, k);
    const double* V = P.v + C3(P, 0, k);
    double pupx = 0.0, pupy = 0.0, pvpx = 0.0, pvpy = 0.0;
    int nt = P.ntve[i];
    bool bnd = P.isonb[i] != 0;
    // J=1, then J=2..NTVE-1, then J=NTVE (viscofh.F:65-111); a node with one cell adds
    // that cell's edge term twice, as the reference does.
    auto ecec = [&](int j) {
      size_t q = (size_t)(j - 1) * m1 + i;
      int c = P.nbve[q];
      double ey = P.dltyecec[q], ex = P.dltxecec[q];
      pupx = pupx + U[c] * ey;
      pupy = pupy + U[c] * ex;
      pvpx = pvpx + V[c] * ey;
      pvpy = pvpy + V[c] * ex;
    };
    auto nec = [&](int j, double sgn) {
      size_t q = (size_t)(j - 1) * m1 + i;
      int c = P.nbve[q];
      double ny = sgn * P.dltynec[q], nx = sgn * P.dltxnec[q];
      pupx = pupx + U[c] * ny;
      pupy = pupy + U[c] * nx;
      pvpx = pvpx + V[c] * ny;
      pvpy = pvpy + V[c] * nx;
    };
    ecec(1);
    if (bnd) nec(1, 1.0);
    for (int j = 2; j <= nt - 1; ++j) ecec(j);
    ecec(nt);
    if (bnd) nec(nt, -1.0);
    double a1 = P.art1[i];
    pupx = pupx / a1;
    pupy = pupy / a1;
    pvpx = pvpx / a1;
    pvpy = pvpy / a1;
    double tmp1 = pupx * pupx + pvpy * pvpy;
    double tmp2 = 0.5 * ((pupy + pvpx) * (pupy + pvpx));
    P.viscofh[N3(P, i, k)] = sqrt(tmp1 + tmp2) * a1;
  }
  }
}

// The end of ADV_UV_EDGE_GCN for cell i on layer k once its three edges are summed into
// xr, yr, vmr and the pressure-gradient terms into px, py (adv_uv_edge_gcn.F:884-1193):
// wet mask, vertical advection, DRHOX, Coriolis, open-boundary cells, rivers, the update
// to UF, VF and VISCOFM.
template <typename R>
__device__ inline void adv_uv_tail(const Dev& P, int i, int k, R xr, R yr, R vmr, double px, double py,
                                   double dz1i) {
  double x = (double)xr, y = (double)yr, vm = (double)vmr;
  bool wet = P.iswetct[i] * P.iswetc[i] == 1;
  double w = (double)(P.iswetct[i] * P.iswetc[i]);
  x = x * w;
  y = y * w;
  px = px * w;
  py = py * w;
  x = x + px;
  y = y + py;
  size_t q = C3(P, i, k);
  if (wet) {
    const double *U = P.u, *V = P.v, *W = P.w, *DZ1 = P.dz1;
    double xfv, yfv;
    if (k == 1) {
      size_t qp = C3(P, i, k + 1);
      xfv = -W[qp] * (U[q] * DZ1[qp] + U[qp] * DZ1[q]) / (DZ1[q] + DZ1[qp]);
      yfv = -W[qp] * (V[q] * DZ1[qp] + V[qp] * DZ1[q]) / (DZ1[q] + DZ1[qp]);
    } else if (k == P.KBM1) {
      size_t qm = C3(P, i, k - 1);
      xfv = W[q] * (U[q] * DZ1[qm] + U[qm] * DZ1[q]) / (DZ1[q] + DZ1[qm]);
      yfv = W[q] * (V[q] * DZ1[qm] + V[qm] * DZ1[q]) / (DZ1[q] + DZ1[qm]);
    } else {
      size_t qm = C3(P, i, k - 1), qp = C3(P, i, k + 1);
      xfv = W[q] * (U[q] * DZ1[qm] + U[qm] * DZ1[q]) / (DZ1[q] + DZ1[qm]) -
            W[qp] * (U[q] * DZ1[qp] + U[qp] * DZ1[q]) / (DZ1[q] + DZ1[qp]);
      yfv = W[q] * (V[q] * DZ1[qm] + V[qm] * DZ1[q]) / (DZ1[q] + DZ1[qm]) -
            W[qp] * (V[q] * DZ1[qp] + V[qp] * DZ1[q]) / (DZ1[q] + DZ1[qp]);
    }
    x = x + xfv * P.art[i] + P.drhox[q] - P.cor[i] * V[q] * P.dt1[i] * DZ1[q] * P.art[i];
    y = y + yfv * P.art[i] + P.drhoy[q] + P.cor[i] * U[q] * P.dt1[i] * DZ1[q] * P.art[i];
  }
  if (P.isbce[i] == 2) { x = 0.0; y = 0.0; }
  river3(P, i, k, x, y);
  double uf, vf;
  if (wet) {
    double d1 = P.d1[i];
    uf = P.u[q] * P.dt1[i] / d1 - P.dti * x / P.art[i] / (d1 * dz1i);
    vf = P.v[q] * P.dt1[i] / d1 - P.dti * y / P.art[i] / (d1 * dz1i);
  } else {
    uf = 0.0;
    vf = 0.0;
  }
  P.uf[q] = uf;
  P.vf[q] = vf;
  P.viscofm[q] = vm / P.art[i];
}

// -------------------------------------------------------------------------------------
// ADV_UV_EDGE_GCN (adv_uv_edge_gcn.F:124-1193): horizontal advection/diffusion, the
// internal barotropic pressure gradient from EGF, vertical advection, baroclinic
// pressure gradient, Coriolis, river momentum and the explicit update to UF/VF.
// -------------------------------------------------------------------------------------
template <typename R, bool LIM>
__global__ void __launch_bounds__(256, (sizeof(R) == 4 && !LIM) ? 4 : 1) k_adv_uv(const Dev P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  int kb, ke;
  col_range(P, 1, P.KBM1, kb, ke);
  for (int k = kb; k <= ke; ++k) {
  const size_t n1 = P.N + 1;
  double px = 0.0, py = 0.0;
  const R epor = (R)P.epor[i], three = (R)3.0;
  R xr = 0, yr = 0, vmr = 0;
  const double dz1i = P.dz1[C3(P, i, k)];
  const double gdd = P.grav_e[i] * P.dt1[i] * dz1i;
    // FP32 form without a limiter: the cell's own side of its three edges, once
    constexpr bool OWN = !LIM && sizeof(R) == 4;
    Own3<R> own;
    if constexpr (OWN) {
      own.g = load_g3<R>(P, i, k);
      own.u = (R)P.u[C3(P, i, k)];
      own.v = (R)P.v[C3(P, i, k)];
      own.art = Mesh<R>::art(P, i);
      own.cc = Mesh<R>::cc_hvc(P, i);
    }
  for (int s = 0; s < 3; ++s) {
    const size_t q = (size_t)s * n1 + i;
    const int4 ci = P.ce_i4[q];  // {code, IA, IB, J1}
    const int code = ci.x, side = code & 1, isbc = (code >> 1) & 1;
    const int ia = ci.y, ib = ci.z;
    const int j1 = ci.w, j2 = P.ce_j2[q];
    double elij = 0.5 * (P.egf[j1] + P.egf[j2]);
    R dij = (R)(0.5 * (P.dt[j1] * P.dz[N3(P, j1, k)] + P.dt[j2] * P.dz[N3(P, j2, k)]));
    if (P.iswetct[ia] * P.iswetc[ia] == 1 || P.iswetct[ib] * P.iswetc[ib] == 1) {
      EdgeFlux<R> f = edge_flux3<R, LIM, OWN>(P, q, ia, ib, k, dij, true, own, side);
      vmr = vmr + f.viscof;
      R isb = (R)isbc;
      R tp = (R)((double)(float)(1 - isbc) * P.epor[i]);
      const R vfx = P.gcy ? f.fxx * tp : (f.fxx + three * f.fxx * isb) * epor;  // GCY: adv_uv_edge_gcy.F
      const R vfy = P.gcy ? f.fyy * tp : (f.fyy + three * f.fyy * isb) * epor;
      if (side == 0) {
        xr = xr + f.xadv * tp + vfx;
        yr = yr + f.yadv * tp + vfy;
      } else {
        xr = xr - f.xadv * tp - vfx;
        yr = yr - f.yadv * tp - vfy;
      }
    }
    const double edx = P.ce_dx[q], edy = P.ce_dy[q];
    if (side == 0) {
      px = px - gdd * elij * edy;
      py = py + gdd * elij * edx;
    } else {
      px = px + gdd * elij * edy;
      py = py - gdd * elij * edx;
    }
  }
  adv_uv_tail<R>(P, i, k, xr, yr, vmr, px, py, dz1i);
  }
}

// -------------------------------------------------------------------------------------
// Tile-staged ADVECTION_EDGE_GCN (UV = false) and ADV_UV_EDGE_GCN (UV = true), LIMITED_NO
// and GCN.  One CTA per cell tile (struct Tiles) and chunk of layers.  Per layer, the
// tile's cells and their halo -- U, V and the least-squares gradient, with ART, CC_HVC and
// the wet flags staged once -- are loaded into shared memory; every edge of the tile is
// evaluated once from there into shared memory (an interior edge serves both its cells);
// then each own cell sums its three edges in ascending edge number, as the reference's
// scatter adds them, and finishes as the per-cell kernels do.  The edge arithmetic is
// edge_flux3's term by term, so the FP64 instantiation equals the per-cell kernels bit
// for bit.
// -------------------------------------------------------------------------------------
template <typename R>
__device__ inline EdgeFlux<R> edge_flux_staged(const Dev& P, R ua, R va, const R* ga, R ub, R vb, const R* gb,
                                               R arta, R artb, R cca, R ccb, R xija, R yija, R xijb, R yijb,
                                               R dltxc, R dltyc, R dij, bool exflux_form) {
  const R half = (R)0.5, one = (R)1.0;
  // ga, gb: {UX, UY, VX, VY} of IA and IB
  const R uij1 = ua + ga[0] * xija + ga[1] * yija;
  const R vij1 = va + ga[2] * xija + ga[3] * yija;
  const R uij2 = ub + gb[0] * xijb + gb[1] * yijb;
  const R vij2 = vb + gb[2] * xijb + gb[3] * yijb;
  R uij = half * (uij1 + uij2);
  R vij = half * (vij1 + vij2);
  R viscof1 = arta * sqrt(ga[0] * ga[0] + ga[3] * ga[3] + half * ((ga[1] + ga[2]) * (ga[1] + ga[2])));
  R viscof2 = artb * sqrt(gb[0] * gb[0] + gb[3] * gb[3] + half * ((gb[1] + gb[2]) * (gb[1] + gb[2])));
  R viscof = ((R)P.fact * half * (viscof1 * cca + viscof2 * ccb) + (R)P.fm1 * half * (cca + ccb)) / (R)P.hprnu;
  R txx = (ga[0] + gb[0]) * viscof;
  R tyy = (ga[3] + gb[3]) * viscof;
  R txy = half * (ga[1] + gb[1] + ga[2] + gb[2]) * viscof;
  EdgeFlux<R> f;
  f.fxx = dij * (txx * dltyc - txy * dltxc);
  f.fyy = dij * (txy * dltyc - tyy * dltxc);
  f.viscof = viscof;
  if (exflux_form) {
    R exflux = dij * (-uij * dltyc + vij * dltxc);
    R sg = fsign1(exflux);
    f.xadv = exflux * ((one - sg) * uij2 + (one + sg) * uij1) * half;
    f.yadv = exflux * ((one - sg) * vij2 + (one + sg) * vij1) * half;
  } else {
    R un = vij * dltxc - uij * dltyc;
    R sg = fsign1(un);
    f.xadv = dij * un * ((one - sg) * uij2 + (one + sg) * uij1) * half;
    f.yadv = dij * un * ((one - sg) * vij2 + (one + sg) * vij1) * half;
  }
  return f;
}

// Shared memory of one CTA: FP64 DT of both edge nodes (and for UV ELIJ, DLTXC, DLTYC)
// per edge; per cell U, V, UX, UY, VX, VY, ART, CC_HVC; per edge its six metrics and five
// flux values; the cells' wet flags; per edge its two nodes, local cells and wet flag.
template <typename R, bool UV>
__host__ __device__ inline size_t staged_smem_bytes(int cc, int ec) {
  return sizeof(double) * ((size_t)2 * ec + (UV ? (size_t)3 * ec : 0)) + sizeof(R) * ((size_t)8 * cc + (size_t)11 * ec) +
         sizeof(int) * ((size_t)cc + (size_t)4 * ec);
}

template <typename R, bool UV>
__global__ void __launch_bounds__(kTileCells, sizeof(R) == 4 ? 6 : 4) k_mom3d_staged(const Dev P) {
  typedef Mesh<R> Mh;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const Tiles& T = P.tl;
  const int t = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const int c0 = T.ptr[t], nall = T.ptr[t + 1] - c0, nc = T.nc[t];
  const int e0 = T.eptr[t], ne = T.eptr[t + 1] - e0;
  const int CC = T.cap_cells, EC = T.cap_edges;
  double* s_dt = reinterpret_cast<double*>(sm_raw);   // [2][EC]
  double* s_pg = s_dt + 2 * EC;                       // UV: [3][EC] ELIJ, DLTXC, DLTYC
  R* s_c = reinterpret_cast<R*>(s_pg + (UV ? 3 * EC : 0));  // [8][CC]
  R* s_e = s_c + 8 * CC;                              // [6][EC] XOA, YOA, XOB, YOB, DLTXC, DLTYC
  R* s_f = s_e + 6 * EC;                              // [5][EC] XADV, YADV, FXX, FYY, VISCOF
  int* s_w = reinterpret_cast<int*>(s_f + 5 * EC);    // [CC] ISWETCT*ISWETC
  int* s_j = s_w + CC;                                // [3][EC] IENODE1, IENODE2, IA | IB << 16
  int* s_ok = s_j + 3 * EC;                           // [EC] a side of the edge is wet

  // fixed over the layers: the cells' ART, CC_HVC and wet flags, the edges' metrics
  for (int q = tid; q < nall; q += nt) {
    const int c = T.cells[c0 + q];
    s_c[6 * CC + q] = Mh::art(P, c);
    s_c[7 * CC + q] = Mh::cc_hvc(P, c);
    s_w[q] = P.iswetct[c] * P.iswetc[c];
  }
  __syncthreads();
  for (int q = tid; q < ne; q += nt) {
    const int4 ed = T.edges[e0 + q];  // {edge, IA | IB << 16, IENODE1, IENODE2}
    const int e = ed.x, la = ed.y & 0xffff, lb = ed.y >> 16;
    const int ia = T.cells[c0 + la], ib = T.cells[c0 + lb];
    s_e[q] = Mh::xoa(P, e, ia);
    s_e[EC + q] = Mh::yoa(P, e, ia);
    s_e[2 * EC + q] = Mh::xob(P, e, ib);
    s_e[3 * EC + q] = Mh::yob(P, e, ib);
    s_e[4 * EC + q] = Mh::dltxc(P, e);
    s_e[5 * EC + q] = Mh::dltyc(P, e);
    s_dt[q] = P.dt[ed.z];
    s_dt[EC + q] = P.dt[ed.w];
    s_j[q] = ed.z;
    s_j[EC + q] = ed.w;
    s_j[2 * EC + q] = ed.y;
    s_ok[q] = (s_w[la] == 1 || s_w[lb] == 1) ? 1 : 0;
    if (UV) {
      s_pg[q] = 0.5 * (P.egf[ed.z] + P.egf[ed.w]);
      s_pg[EC + q] = P.dltxc[e];
      s_pg[2 * EC + q] = P.dltyc[e];
    }
  }
  const bool own = tid < nc;
  const int4 sl = own ? T.slots[c0 + tid] : make_int4(0, 0, 0, 0);
  const int i = own ? T.cells[c0 + tid] : 0;
  int kb, ke;
  col_range(P, 1, P.KBM1, kb, ke);
  for (int k = kb; k <= ke; ++k) {
    __syncthreads();
    for (int q = tid; q < nall; q += nt) {
      const int c = T.cells[c0 + q];
      const size_t qq = C3(P, c, k);
      s_c[q] = (R)P.u[qq];
      s_c[CC + q] = (R)P.v[qq];
      const G3<R> g = load_g3<R>(P, c, k);
      s_c[2 * CC + q] = g.ux;
      s_c[3 * CC + q] = g.uy;
      s_c[4 * CC + q] = g.vx;
      s_c[5 * CC + q] = g.vy;
    }
    __syncthreads();
    for (int q = tid; q < ne; q += nt) {
      if (!s_ok[q]) continue;
      const int lab = s_j[2 * EC + q], la = lab & 0xffff, lb = lab >> 16;
      const R dij = (R)(0.5 * (s_dt[q] * P.dz[N3(P, s_j[q], k)] + s_dt[EC + q] * P.dz[N3(P, s_j[EC + q], k)]));
      const R ga[4] = {s_c[2 * CC + la], s_c[3 * CC + la], s_c[4 * CC + la], s_c[5 * CC + la]};
      const R gb[4] = {s_c[2 * CC + lb], s_c[3 * CC + lb], s_c[4 * CC + lb], s_c[5 * CC + lb]};
      const EdgeFlux<R> f = edge_flux_staged<R>(P, s_c[la], s_c[CC + la], ga, s_c[lb], s_c[CC + lb], gb,
                                                s_c[6 * CC + la], s_c[6 * CC + lb], s_c[7 * CC + la],
                                                s_c[7 * CC + lb], s_e[q], s_e[EC + q], s_e[2 * EC + q],
                                                s_e[3 * EC + q], s_e[4 * EC + q], s_e[5 * EC + q], dij, UV);
      s_f[q] = f.xadv;
      s_f[EC + q] = f.yadv;
      s_f[2 * EC + q] = f.fxx;
      s_f[3 * EC + q] = f.fyy;
      s_f[4 * EC + q] = f.viscof;
    }
    __syncthreads();
    if (!own) continue;
    const R epor = (R)P.epor[i], three = (R)3.0;
    R xr = 0, yr = 0, vmr = 0;
    double px = 0.0, py = 0.0, dz1i = 0.0, gdd = 0.0;
    if (UV) {
      dz1i = P.dz1[C3(P, i, k)];
      gdd = P.grav_e[i] * P.dt1[i] * dz1i;
    }
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int w = s == 0 ? sl.x : (s == 1 ? sl.y : sl.z);
      const int le = w & 0xffff, side = (w >> 16) & 1, isbc = (w >> 17) & 1;
      if (s_ok[le]) {
        if (UV) vmr = vmr + s_f[4 * EC + le];
        const R isb = (R)isbc;
        const R tp = (R)((double)(float)(1 - isbc) * P.epor[i]);
        const R fxx = s_f[2 * EC + le], fyy = s_f[3 * EC + le];
        const R vfx = (fxx + three * fxx * isb) * epor;
        const R vfy = (fyy + three * fyy * isb) * epor;
        if (side == 0) {
          xr = xr + s_f[le] * tp + vfx;
          yr = yr + s_f[EC + le] * tp + vfy;
        } else {
          xr = xr - s_f[le] * tp - vfx;
          yr = yr - s_f[EC + le] * tp - vfy;
        }
      }
      if (UV) {
        const double elij = s_pg[le], edx = s_pg[EC + le], edy = s_pg[2 * EC + le];
        if (side == 0) {
          px = px - gdd * elij * edy;
          py = py + gdd * elij * edx;
        } else {
          px = px + gdd * elij * edy;
          py = py - gdd * elij * edx;
        }
      }
    }
    if (UV)
      adv_uv_tail<R>(P, i, k, xr, yr, vmr, px, py, dz1i);
    else
      advection3d_tail<R>(P, i, k, xr, yr);
  }
}

constexpr int kStagedSmemMax = 200 * 1024;
template <typename R, bool UV>
static void launch_mom3d_staged(const Dev& P, cudaStream_t s) {
  const size_t smem = staged_smem_bytes<R, UV>(P.tl.cap_cells, P.tl.cap_edges);
  const dim3 grid((unsigned)P.tl.n, (unsigned)((P.KBM1 + P.col_lc - 1) / P.col_lc));
  k_mom3d_staged<R, UV><<<grid, kTileCells, smem, s>>>(P);
}
// Whether the staged kernel of ADVECTION (UV false) or ADV_UV (UV true) runs: LIMITED_NO,
// GCN, a tile table whose shared memory fits one CTA, and P.staged = 2 (every staged
// kernel), or P.staged = 1 (the default: only where it measured faster than the per-cell
// kernel on the 200k-node, 40-layer coastal mesh, which is FP64 ADV_UV: 2.13 against
// 2.52 ms per step; FP64 ADVECTION 1.35 against 1.26, FP32 ADVECTION 1.00 against 0.76,
// FP32 ADV_UV 1.90 against 1.30).
static bool staged_ok(const Dev& P, bool uv) {
  const bool want = P.staged == 2 || (P.staged == 1 && uv && sizeof(RF) == 8);
  return want && !P.limiter && !P.gcy && P.tl.n > 0 &&
         staged_smem_bytes<double, true>(P.tl.cap_cells, P.tl.cap_edges) <= (size_t)kStagedSmemMax;
}
// Allow the staged kernels of this translation unit's arithmetic type up to
// kStagedSmemMax bytes of dynamic shared memory (once, before any launch or capture).
int staged_setup() {
  if (cudaFuncSetAttribute(k_mom3d_staged<RF, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kStagedSmemMax) != cudaSuccess)
    return 1;
  if (cudaFuncSetAttribute(k_mom3d_staged<RF, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kStagedSmemMax) != cudaSuccess)
    return 1;
  return 0;
}

// -------------------------------------------------------------------------------------
// VDIF_UV (vdif_uv.F:56-182), the static-SSH fix and BCOND_GCN(3,0)
// (internal_step.F:660-672, bcond_gcn.F:424-502), WREAL (wreal.F:57-129).
// One thread per cell column; the Thomas sweep keeps its coefficients in registers and
// local memory.
// -------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_vdif_uv(const Dev P, int parts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  const int KB = P.KB, KBM1 = P.KBM1, KBM2 = P.KBM2;
  const double DTI = P.dti;
  // With VU_BC3 in the same launch the sponge and BCOND_GCN(3,0) are applied to each
  // solved value before it is stored (per element they follow in the reference's order),
  // which saves two passes over UF and VF.
  const bool fused = (parts & VU_VDIF) && (parts & VU_BC3);
  const bool fix = P.h1[i] <= P.static_ssh_adj;
  const int b = P.isbce[i];
  const double sp = P.cc_sponge[i];
  auto bc3 = [&](double& uu, double& vv) {
    if (fix) { uu = P.ua[i]; vv = P.va[i]; }
    if (b == 3 && !P.gcy) { uu = 0.0; vv = 0.0; }
    if (b == 1) bc_solid3(P, i, uu, vv);
  };
  // the sponge of vdif_uv.F's end, then (fused) BCOND_GCN(3,0), then the store
  auto finish = [&](int k, double uu, double vv) {
    const size_t q = C3(P, i, k);
    if (fused) {
      uu = uu / (1.0 + sp * (uu * uu));
      vv = vv / (1.0 + sp * (vv * vv));
      bc3(uu, vv);
    }
    P.uf[q] = uu;
    P.vf[q] = vv;
  };
  if (parts & VU_VDIF) {
    if (P.iswetc[i] == 1) {
      double vhu[kMaxKB], vhpu[kMaxKB], vhv[kMaxKB], vhpv[kMaxKB];
      const double d1 = P.d1[i];
      // A(K) uses KM1(K+1) with DZ1(K), DZZ1(K); C(K) uses KM1(K) with DZ1(K), DZZ1(K-1).
      auto Acoef = [&](int kk) {
        return -DTI * (P.km1[C3(P, i, kk + 1)] + P.umol) / (P.dz1[C3(P, i, kk)] * P.dzz1[C3(P, i, kk)] * d1 * d1);
      };
      auto Ccoef = [&](int kk) {
        return -DTI * (P.km1[C3(P, i, kk)] + P.umol) / (P.dz1[C3(P, i, kk)] * P.dzz1[C3(P, i, kk - 1)] * d1 * d1);
      };
      int n1 = P.N + 1;
      int it1 = P.isonb[P.nv[i]], it2 = P.isonb[P.nv[n1 + i]], it3 = P.isonb[P.nv[2 * n1 + i]];
      double tmp = (it1 == 2 || it2 == 2 || it3 == 2) ? 0.0 : 1.0;
      double a1 = Acoef(1);
      double wus = P.wusurf[i], wvs = P.wvsurf[i];
      vhu[1] = a1 / (a1 - 1.0);
      vhv[1] = a1 / (a1 - 1.0);
      vhpu[1] = (-DTI * wus * tmp / (-P.dz1[C3(P, i, 1)] * d1) - P.uf[C3(P, i, 1)]) / (a1 - 1.0);
      vhpv[1] = (-DTI * wvs * tmp / (-P.dz1[C3(P, i, 1)] * d1) - P.vf[C3(P, i, 1)]) / (a1 - 1.0);
      // the forward elimination; the loads of four levels are issued before their steps
      auto step = [&](int k, double ak, double ck, double uk, double vk) {
        double pu = 1.0 / (ak + ck * (1.0 - vhu[k - 1]) - 1.0);
        double pv = 1.0 / (ak + ck * (1.0 - vhv[k - 1]) - 1.0);
        vhu[k] = ak * pu;
        vhv[k] = ak * pv;
        vhpu[k] = (ck * vhpu[k - 1] - uk) * pu;
        vhpv[k] = (ck * vhpv[k - 1] - vk) * pv;
      };
      int k = 2;
      for (; k + 3 <= KBM2; k += 4) {
        double ak[4], ck[4], uk[4], vk[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          ak[u] = Acoef(k + u);
          ck[u] = Ccoef(k + u);
          uk[u] = P.uf[C3(P, i, k + u)];
          vk[u] = P.vf[C3(P, i, k + u)];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) step(k + u, ak[u], ck[u], uk[u], vk[u]);
      }
      for (; k <= KBM2; ++k) step(k, Acoef(k), Ccoef(k), P.uf[C3(P, i, k)], P.vf[C3(P, i, k)]);
      double ub = P.u[C3(P, i, KBM1)], vb = P.v[C3(P, i, KBM1)];
      double tps = P.cbc[i] * sqrt(ub * ub + vb * vb);
      P.tps[i] = tps;
      double cb = Ccoef(KBM1);
      double dzb = P.dz1[C3(P, i, KBM1)];
      double ufk = (cb * vhpu[KBM2] - P.uf[C3(P, i, KBM1)]) / (tps * DTI / (-dzb * d1) - 1.0 - (vhu[KBM2] - 1.0) * cb);
      double vfk = (cb * vhpv[KBM2] - P.vf[C3(P, i, KBM1)]) / (tps * DTI / (-dzb * d1) - 1.0 - (vhv[KBM2] - 1.0) * cb);
      finish(KBM1, ufk, vfk);
      for (int k = 2; k <= KBM1; ++k) {
        int ki = KB - k;
        ufk = (vhu[ki] * ufk + vhpu[ki]);
        vfk = (vhv[ki] * vfk + vhpv[ki]);
        finish(ki, ufk, vfk);
      }
      P.wubot[i] = -tps * ub;
      P.wvbot[i] = -tps * vb;
    } else {
      for (int k = 2; k <= KBM1; ++k) finish(KB - k, 0.0, 0.0);
      if (fused) finish(KBM1, P.uf[C3(P, i, KBM1)], P.vf[C3(P, i, KBM1)]);
      P.wubot[i] = 0.0;
      P.wvbot[i] = 0.0;
    }
    if (!fused) {
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = C3(P, i, k);
        double uu = P.uf[q], vv = P.vf[q];
        P.uf[q] = uu / (1.0 + sp * (uu * uu));
        P.vf[q] = vv / (1.0 + sp * (vv * vv));
      }
    }
  }
  if ((parts & VU_BC3) && !fused) {
    for (int k = 1; k <= KBM1; ++k) {
      size_t q = C3(P, i, k);
      double uu = P.uf[q], vv = P.vf[q];
      bc3(uu, vv);
      P.uf[q] = uu;
      P.vf[q] = vv;
    }
  }
  if (parts & VU_WREAL) {
    if (P.iswetc[i] == 1) {
      const size_t n1 = P.N + 1;
      int j1 = P.nv[i], j2 = P.nv[n1 + i], j3 = P.nv[2 * n1 + i];
      double ax1 = P.awx[i], ax2 = P.awx[n1 + i], ax3 = P.awx[2 * n1 + i];
      double ay1 = P.awy[i], ay2 = P.awy[n1 + i], ay3 = P.awy[2 * n1 + i];
      double dddx = ax1 * P.d[j1] + ax2 * P.d[j2] + ax3 * P.d[j3];
      double dddy = ay1 * P.d[j1] + ay2 * P.d[j2] + ay3 * P.d[j3];
      double dedx = ax1 * P.elf[j1] + ax2 * P.elf[j2] + ax3 * P.elf[j3];
      double dedy = ay1 * P.elf[j1] + ay2 * P.elf[j2] + ay3 * P.elf[j3];
      double etf1aa = ONE_THIRD * (P.el[j1] + P.el[j2] + P.el[j3]);
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = C3(P, i, k);
        double zz = P.zz1[q];
        double ww1 = 0.5 * (P.w[q] + P.w[C3(P, i, k + 1)]) + P.u[q] * (zz * dddx + dedx) + P.v[q] * (zz * dddy + dedy);
        double ww2 = (zz + 1.0) * (etf1aa - P.et1[i]) / DTI;
        P.ww[q] = ww1 + ww2;
      }
    } else {
      for (int k = 1; k <= KBM1; ++k) P.ww[C3(P, i, k)] = 0.0;
    }
  }
}

void launch_cell_pre(const Dev& P, cudaStream_t s, int parts) {
  k_cell_pre<<<nblk(P.N, 128), 128, 0, s>>>(P, parts);
}
void launch_grad3(const Dev& P, cudaStream_t s) {
  FVG_F32_FORWARD(launch_grad3(P, s));
  k_grad3<RF><<<col_grid(P, P.N, P.KBM1), P.col_bc, 0, s>>>(P);
}
static void launch_alfa3(const Dev& P, cudaStream_t s) {
  k_alfa3<RF><<<col_grid(P, P.N, P.KBM1), P.col_bc, 0, s>>>(P);
}
void launch_advection3d(const Dev& P, cudaStream_t s) {
  FVG_F32_FORWARD(launch_advection3d(P, s));
  if (staged_ok(P, false)) {
    launch_mom3d_staged<RF, false>(P, s);
    return;
  }
  if (P.limiter) launch_alfa3(P, s);
  (P.limiter ? k_advection3d<RF, true> : k_advection3d<RF, false>)<<<col_grid(P, P.N, P.KBM1), P.col_bc, 0, s>>>(P);
}
// -------------------------------------------------------------------------------------
// PHY_BAROPG (phy_baropg.F:37-151), BAROCLINIC_PRESSURE_GRADIENT = 'z coordinates'.
// SINTER_EXTRP_DOWN (sinter.F) takes, for each target Y, the last interval J of the
// descending abscissae with X(J+1) <= Y <= X(J); both kernels walk targets and abscissae
// together, which finds the same interval: the largest J with X(J) >= Y.
// -------------------------------------------------------------------------------------
constexpr int kZLevels = 600;

__device__ inline double phy_z(const Dev& P, int k) { return (0.5 - (double)(float)k) * P.deltz; }

// RHO1 of each node column interpolated (extrapolated below) to the 600 z levels.
__global__ void __launch_bounds__(128) k_phy_rhoz(const Dev P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  const int M1 = P.KBM1;
  double X[kMaxKB], A[kMaxKB];
  for (int k = 1; k <= M1; ++k) {
    X[k - 1] = P.zz[N3(P, i, k)] * P.dt[i] + P.et[i];
    A[k - 1] = P.rho1[N3(P, i, k)];
  }
  int j = 0;
  for (int t = 1; t <= kZLevels; ++t) {
    const double Y = phy_z(P, t);
    double b = 0.0;
    if (Y > X[0]) b = A[0];
    if (Y < X[M1 - 1]) b = A[M1 - 1] + (A[M1 - 2] - A[M1 - 1]) * (Y - X[M1 - 1]) / (X[M1 - 2] - X[M1 - 1]);
    while (j + 1 <= M1 - 2 && X[j + 1] >= Y) ++j;
    if (Y <= X[j] && Y >= X[j + 1]) b = A[j] - (A[j] - A[j + 1]) * (X[j] - Y) / (X[j] - X[j + 1]);
    P.rhoz[(size_t)(t - 1) * P.ms + i] = b;
  }
}

// Per cell: the pressure integrals of the three edges down the z levels where all three
// nodes are deeper, their gradient PBXZ, PBYZ per level, and those interpolated back to the
// cell's sigma depths while the levels are walked.
__global__ void __launch_bounds__(128) k_phy_baropg(const Dev P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  const size_t n1 = P.N + 1;
  const int j1 = P.nv[i], j2 = P.nv[n1 + i], j3 = P.nv[2 * n1 + i];
  const int KBM1 = P.KBM1;
  const double deltz = P.deltz, art = P.art[i], dt1 = P.dt1[i], ramp = ramp_int(P);
  const double h1 = P.h[j1], h2 = P.h[j2], h3 = P.h[j3];
  // NTMP: the levels K = 1.. where no node is shallower than K*DELTZ (a leading run)
  int ntmp = 0;
  while (ntmp < kZLevels) {
    const double tmp = (double)(float)(ntmp + 1) * deltz;
    if (h1 < tmp || h2 < tmp || h3 < tmp) break;
    ++ntmp;
  }
  auto emit = [&](int k, double bx, double by) {
    const size_t q = C3(P, i, k);
    const double dz1 = P.dz1[q];
    P.drhox[q] = -bx * dt1 * dz1 * art * ramp;
    P.drhoy[q] = -by * dt1 * dz1 * art * ramp;
  };
  auto target = [&](int k) {
    return (P.zz[N3(P, j1, k)] * P.dt[j1] + P.et[j1] + (P.zz[N3(P, j2, k)] * P.dt[j2] + P.et[j2]) +
            (P.zz[N3(P, j3, k)] * P.dt[j3] + P.et[j3])) / 3.;
  };
  if (ntmp <= 1) {
    double bx = 0.0, by = 0.0;
    if (ntmp == 1) {
      const double g1 = 0.5 * (P.grav_n[j2] + P.grav_n[j3]);
      const double g2 = 0.5 * (P.grav_n[j3] + P.grav_n[j1]);
      const double g3 = 0.5 * (P.grav_n[j1] + P.grav_n[j2]);
      const double r1 = P.rhoz[j1], r2 = P.rhoz[j2], r3 = P.rhoz[j3];
      const double pb1 = 0.0 + g1 * (0.5 * (r2 + r3)) * deltz;
      const double pb2 = 0.0 + g2 * (0.5 * (r3 + r1)) * deltz;
      const double pb3 = 0.0 + g3 * (0.5 * (r1 + r2)) * deltz;
      const double ax1 = (P.vy[j3] - P.vy[j2]) * deltz, ay1 = (P.vx[j2] - P.vx[j3]) * deltz;
      const double ax2 = (P.vy[j1] - P.vy[j3]) * deltz, ay2 = (P.vx[j3] - P.vx[j1]) * deltz;
      const double ax3 = (P.vy[j2] - P.vy[j1]) * deltz, ay3 = (P.vx[j1] - P.vx[j2]) * deltz;
      bx = (ax1 * pb1 + ax2 * pb2 + ax3 * pb3) / art / deltz;
      by = (ay1 * pb1 + ay2 * pb2 + ay3 * pb3) / art / deltz;
    }
    for (int k = 1; k <= KBM1; ++k) emit(k, bx, by);
    return;
  }
  const double g1 = 0.5 * (P.grav_n[j2] + P.grav_n[j3]);
  const double g2 = 0.5 * (P.grav_n[j3] + P.grav_n[j1]);
  const double g3 = 0.5 * (P.grav_n[j1] + P.grav_n[j2]);
  const double ax1 = (P.vy[j3] - P.vy[j2]) * deltz, ay1 = (P.vx[j2] - P.vx[j3]) * deltz;
  const double ax2 = (P.vy[j1] - P.vy[j3]) * deltz, ay2 = (P.vx[j3] - P.vx[j1]) * deltz;
  const double ax3 = (P.vy[j2] - P.vy[j1]) * deltz, ay3 = (P.vx[j1] - P.vx[j2]) * deltz;
  double pb1 = 0.0, pb2 = 0.0, pb3 = 0.0;
  double xprev = 0.0, xcur = 0.0, yprev = 0.0, ycur = 0.0;  // PBXZ, PBYZ at levels K-1, K
  double x0 = 0.0, y0 = 0.0;                                 // at level 1
  int t = 1;
  double Y = target(1);
  for (int K = 1; K <= ntmp; ++K) {
    const double* rz = P.rhoz + (size_t)(K - 1) * P.ms;
    const double r1 = rz[j1], r2 = rz[j2], r3 = rz[j3];
    pb1 = pb1 + g1 * (0.5 * (r2 + r3)) * deltz;
    pb2 = pb2 + g2 * (0.5 * (r3 + r1)) * deltz;
    pb3 = pb3 + g3 * (0.5 * (r1 + r2)) * deltz;
    xprev = xcur;
    yprev = ycur;
    xcur = (ax1 * pb1 + ax2 * pb2 + ax3 * pb3) / art / deltz;
    ycur = (ay1 * pb1 + ay2 * pb2 + ay3 * pb3) / art / deltz;
    if (K == 1) {
      x0 = xcur;
      y0 = ycur;
      continue;
    }
    // interval j = K-2 (0-based) spans levels K-1, K: every pending target whose last
    // interval with X(J) >= Y is this one
    const double Xj = phy_z(P, K - 1), Xj1 = phy_z(P, K);
    while (t <= KBM1) {
      if (Y > phy_z(P, 1)) {
        emit(t, x0, y0);
      } else {
        if (Xj1 >= Y && K < ntmp) break;  // a later interval still has X(J) >= Y
        double bx, by;
        if (Y >= Xj1) {
          bx = xprev - (xprev - xcur) * (Xj - Y) / (Xj - Xj1);
          by = yprev - (yprev - ycur) * (Xj - Y) / (Xj - Xj1);
        } else {  // below the last level: extrapolation from the last two
          bx = xcur + (xprev - xcur) * (Y - Xj1) / (Xj - Xj1);
          by = ycur + (yprev - ycur) * (Y - Xj1) / (Xj - Xj1);
        }
        emit(t, bx, by);
      }
      ++t;
      if (t <= KBM1) Y = target(t);
    }
  }
}

void launch_phy_baropg(const Dev& P, cudaStream_t s) {
  k_phy_rhoz<<<nblk(P.M, 128), 128, 0, s>>>(P);
  k_phy_baropg<<<nblk(P.N, 128), 128, 0, s>>>(P);
}

void launch_baropg(const Dev& P, cudaStream_t s, int do_baropg, int do_sums) {
  k_baropg<<<nblk(P.N, 128), 128, 0, s>>>(P, do_baropg, do_sums);
}
void launch_int_reset(const Dev& P, cudaStream_t s) {
  int n = (P.M > P.N ? P.M : P.N) + 1;
  k_int_reset<<<nblk(n, 256), 256, 0, s>>>(P);
}
void launch_adjust2(const Dev& P, cudaStream_t s, int parts) { k_adjust2<<<nblk(P.N + 1, 128), 128, 0, s>>>(P, parts); }
void launch_vertvl_flux(const Dev& P, cudaStream_t s) {
  k_vertvl_flux<<<dim3(nblk(P.M, 32), nblk(P.KBM1, 8)), dim3(32, 8), 0, s>>>(P);
}
void launch_vertvl_col(const Dev& P, cudaStream_t s, int parts) {
  k_vertvl_col<<<nblk(P.M, 128), 128, 0, s>>>(P, parts);
}
void launch_w_viscofh(const Dev& P, cudaStream_t s, int do_w, int do_visc) {
  int n = P.M > P.N ? P.M : P.N;
  k_w_viscofh<<<col_grid(P, n, P.KB), P.col_bc, 0, s>>>(P, do_w, do_visc);
}
void launch_adv_uv(const Dev& P, cudaStream_t s) {
  FVG_F32_FORWARD(launch_adv_uv(P, s));
  if (staged_ok(P, true)) {
    launch_mom3d_staged<RF, true>(P, s);
    return;
  }
  if (P.limiter) launch_alfa3(P, s);
  (P.limiter ? k_adv_uv<RF, true> : k_adv_uv<RF, false>)<<<col_grid(P, P.N, P.KBM1), P.col_bc, 0, s>>>(P);
}
void launch_vdif_uv(const Dev& P, cudaStream_t s, int parts) {
  k_vdif_uv<<<nblk(P.N, 128), 128, 0, s>>>(P, parts);
}

}  // namespace fvg / fvg_f32
