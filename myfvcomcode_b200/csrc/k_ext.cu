// k_ext.cu - external (2-D) mode kernels: one EXTERNAL_STEP Runge-Kutta stage is
//   k_ext_node   EXTEL_EDGE(K) + BCOND_GCN(1,K) + RK blend      (per node, half-edge gather)
//   k_wet_*      WET_JUDGE                                      (wetting/drying only)
//   k_ext_cell   N2E2D + FLUX_OBN + ADVAVE_EDGE_GCN + EXTUV_EDGE + BCOND_GCN(2,K)  (per cell)
//   k_ext_update external_step.F:333-436 (EL=ELF, D, D1, UA=UAF, UARD/EGF sums)
// Reference: FVCOM_source/external_step.F:30-443 and the routines cited per kernel.
// Arithmetic is kept in the reference's expression order; the library is compiled with
// --fmad=false so no multiply-add is contracted.
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

// Programmatic dependent launch: wait until the previous kernel in the stream has
// completed and its writes are visible (a no-op when the kernel was launched without the
// attribute), then let the next kernel's blocks be scheduled during this one's tail.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... KArgs, typename... Args>
static void launch_maybe_pdl(int pdl, void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, args...);
}

__device__ __constant__ double dAlphaRK[5] = {0.0, 0.25, 1.0 / 3.0, 0.5, 1.0};
#ifndef FVG_F32_TU
const double kAlphaRK[5] = {0.0, 0.25, 1.0 / 3.0, 0.5, 1.0};
#endif
#define ONE_THIRD (1.0 / 3.0)

__device__ inline const double* sched_row(const Dev& P) {
  return P.sched + (size_t)P.ctl[0] * P.sl.len;
}

// -------------------------------------------------------------------------------------
// Least-squares velocity gradient of one cell from itself and its three neighbours
// (advave_edge_gcn.F:634-637, 699-702): COFA1/COFA2 for UA, COFA5/COFA6 for VA.
// -------------------------------------------------------------------------------------
template <typename R>
struct Grad {
  R ux, uy, vx, vy;
};

template <typename R, bool CS = false>
__device__ inline Grad<R> cell_grad(const Dev& P, int c, const double* U, const double* V) {
  typedef Mesh<R> Mh;
  int k1, k2, k3;
  R A[4], B[4];
  lsq_coef<R, CS>(P, c, k1, k2, k3, A, B);
  const R a1 = A[0], a2 = A[1], a3 = A[2], a4 = A[3], b1 = B[0], b2 = B[1], b3 = B[2], b4 = B[3];
  R u0 = (R)U[c], u1 = (R)U[k1], u2 = (R)U[k2], u3 = (R)U[k3];
  R v0 = (R)V[c], v1 = (R)V[k1], v2 = (R)V[k2], v3 = (R)V[k3];
  if (P.gcy && (k1 == 0 || k2 == 0 || k3 == 0)) {
    double gu, gv;
    if (k1 == 0) { ghost_uv(P, U, V, c, 1, gu, gv); u1 = (R)gu; v1 = (R)gv; }
    if (k2 == 0) { ghost_uv(P, U, V, c, 2, gu, gv); u2 = (R)gu; v2 = (R)gv; }
    if (k3 == 0) { ghost_uv(P, U, V, c, 3, gu, gv); u3 = (R)gu; v3 = (R)gv; }
  }
  Grad<R> g;
  g.ux = a1 * u0 + a2 * u1 + a3 * u2 + a4 * u3;
  g.uy = b1 * u0 + b2 * u1 + b3 * u2 + b4 * u3;
  g.vx = a1 * v0 + a2 * v1 + a3 * v2 + a4 * v3;
  g.vy = b1 * v0 + b2 * v1 + b3 * v2 + b4 * v3;
  return g;
}
// Least-squares gradient of UA, VA of cell c (advave_edge_gcn.F:634-637, 699-702), stored
// for the edge loop of the next ADVAVE call in the handle's precision.
template <typename R, bool CS>
__device__ inline void store_grad_t(const Dev& P, int c) {
  Grad<R> g = cell_grad<R, CS>(P, c, P.ua, P.va);
  if constexpr (sizeof(R) == 4) {
    P.f.g2d4[c] = make_float4(g.ux, g.uy, g.vx, g.vy);
  } else {
    Mesh<R>::g2d(P, 0)[c] = g.ux;
    Mesh<R>::g2d(P, 1)[c] = g.uy;
    Mesh<R>::g2d(P, 2)[c] = g.vx;
    Mesh<R>::g2d(P, 3)[c] = g.vy;
  }
}
template <bool CS>
__device__ inline void store_grad(const Dev& P, int c) {
  if (P.prec) store_grad_t<float, CS>(P, c);
  else store_grad_t<double, CS>(P, c);
}
template <typename R>
__device__ inline Grad<R> load_grad(const Dev& P, int c) {
  Grad<R> g;
  if constexpr (sizeof(R) == 4) {
    const float4 a = P.f.g2d4[c];
    g.ux = a.x;
    g.uy = a.y;
    g.vx = a.z;
    g.vy = a.w;
  } else {
    g.ux = Mesh<R>::g2d(P, 0)[c];
    g.uy = Mesh<R>::g2d(P, 1)[c];
    g.vx = Mesh<R>::g2d(P, 2)[c];
    g.vy = Mesh<R>::g2d(P, 3)[c];
  }
  return g;
}
// EXTEL_EDGE half-edge flux EXFLUX = DIJ*(-UIJ*DLTYE+VIJ*DLTXE) (extel_edge.F:86-94) of the
// three half-edges owned by cell c, from the cell's own D1, UA, VA.
__device__ inline void store_exf(const Dev& P, int c) {
  double d1 = P.d1[c], u = P.ua[c], v = P.va[c];
  for (int s = 0; s < 3; ++s) {
    const size_t pos = (size_t)s * P.ns + c;
    P.exf2d[pos] = d1 * (-u * Mesh<double>::hg(P, 1, pos) + v * Mesh<double>::hg(P, 0, pos));
  }
}

// -------------------------------------------------------------------------------------
// EXTEL_EDGE(K) (extel_edge.F:76-180) and BCOND_GCN(1,K) -> BCOND_ASL/BCOND_ASL_CLP
// (mod_obcs.F:509-617) with the Runge-Kutta blend of the specified-elevation nodes
// (external_step.F:262-266).  One thread per node; the node's control-volume half-edges
// are gathered in ascending half-edge number, the order of the reference's scatter.
// Node part of WET_JUDGE for node i from the cell flags cwet of the same judgement.
template <bool CS = false>
__device__ inline void wet_node(const Dev& P, int i, const int* cwet) {
  double e = P.elf[i];
  int wet = ((P.h[i] + e - P.min_depth) < 1.0e-5) ? 0 : 1;
  // the ring's cell flags, four entries' indices and then their flags loaded at a time
  const int nt = ld1<CS>(P.ntve + i);
  const size_t m1 = P.M + 1;
  const int* L = P.nbve + i;
  int s = 0, j = 0;
  for (; j + 4 <= nt; j += 4) {
    const int c0 = ld1<CS>(L + j * m1), c1 = ld1<CS>(L + (j + 1) * m1), c2 = ld1<CS>(L + (j + 2) * m1),
              c3 = ld1<CS>(L + (j + 3) * m1);
    s += cwet[c0] + cwet[c1] + cwet[c2] + cwet[c3];
  }
  for (; j < nt; ++j) s += cwet[ld1<CS>(L + j * m1)];
  if (s == 0) wet = 0;
  P.iswetn[i] = wet;
  P.elf[i] = fmax(e, -P.h[i] + P.min_depth);
}

// -------------------------------------------------------------------------------------
// Node part of the update after stage K (external_step.F:333-436): EL = ELF, D, DTFA, and
// the K == 3 and K == 4 sums.
template <bool CS = false>
__device__ inline void ext_update_node(const Dev& P, int i, int K) {
  double e = P.elf[i];
  P.el[i] = e;
  double dd = P.h[i] + e;
  P.d[i] = dd;
  P.dtfa[i] = dd;
  if (K == 3) P.egf[i] = ld1<CS>(P.egf + i) + e / (double)P.isplit;
  if (K == 4) {
    int ob = ld1<CS>(P.node_obc + i);
    if (ob > 0) {
      double tmp = -(P.elf[i] - P.elrk[i]) * P.art1[i] / P.dte - P.xflux_obcn[ob];
      P.uard_obcn[ob] = P.uard_obcn[ob] + tmp / (double)(float)P.isplit;
    }
  }
}

// Cell part of the update after stage K with the new UA, VA: EL1, D1, the K == 3 sums and
// the half-edge continuity fluxes of the next stage.
__device__ inline void ext_update_cell(const Dev& P, int i, int K, double u, double v) {
  double e1 = P.elf1[i];
  P.el1[i] = e1;
  double dd1 = P.h1[i] + e1;
  P.d1[i] = dd1;
  if (K == 3) {
    P.uard[i] = P.uard[i] + u * dd1;
    P.vard[i] = P.vard[i] + v * dd1;
  }
  for (int s = 0; s < 3; ++s) {
    const size_t pos = (size_t)s * P.ns + i;
    P.exf2d[pos] = dd1 * (-u * Mesh<double>::hg(P, 1, pos) + v * Mesh<double>::hg(P, 0, pos));
  }
}

// Slope limiters UALFA, VALFA of each cell for the limited ADVAVE (advave_edge_gcn.F:141-318):
// the cell's three edges with a wet side, in any order (a minimum), from the cell's own
// gradient and the two cells' UA, VA.  After WET_JUDGE, before the stage's ADVAVE.
template <typename R>
__global__ void k_alfa2(const Dev P) {
  typedef Mesh<R> Mh;
  const int c = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (c > P.N) return;
  const size_t n1 = P.N + 1;
  const Grad<R> g = load_grad<R>(P, c);
  R au = (R)1, av = (R)1;
  for (int s = 0; s < 3; ++s) {
    const size_t q = (size_t)s * n1 + c;
    const int ia = P.ce_ia[q], ib = P.ce_ib[q];
    if (!(P.iswetce[ia] * P.iswetc[ia] == 1 || P.iswetce[ib] * P.iswetc[ib] == 1)) continue;
    const bool a_side = (P.ce_code[q] & 1) == 0;
    const R x = a_side ? Mh::s_xoa(P, q) : Mh::s_xob(P, q);
    const R y = a_side ? Mh::s_yoa(P, q) : Mh::s_yob(P, q);
    lim_alfa<R>(fabs((R)P.ua[ia] - (R)P.ua[ib]), g.ux * x + g.uy * y, au);
    lim_alfa<R>(fabs((R)P.va[ia] - (R)P.va[ib]), g.vx * x + g.vy * y, av);
  }
  Mh::alfa2(P, 0)[c] = au;
  Mh::alfa2(P, 1)[c] = av;
}

// CS: the arrays the kernel reads once per stage (gather lists, pointers, per-node and
// per-cell coefficients) are loaded evict-first (ld1).
template <bool CS>
__device__ __forceinline__ void ext_node_job(const Dev& P, const int i, int iext, int K, int parts) {
  // jobs 1..M are the nodes, jobs M+1..M+N the cells' least-squares gradients of the
  // current UA, VA for ADVAVE of this stage
  if (i > P.M) {
    const int c = i - P.M;
    if ((parts & EN_GRAD) && c <= P.N) store_grad<CS>(P, c);
    return;
  }
  // EXTEL's sum first: its loads (the previous cell kernel's half-edge fluxes) do not
  // depend on the node updates below, which then overlap with them
  double x = 0.0;
  if (parts & EN_EXTEL) {
    // the half-edge fluxes in ascending half-edge order; four entries' codes and then
    // their fluxes are loaded at a time, and added in order
    const int n = ld1<CS>(P.node_he_ptr + i + 1) - ld1<CS>(P.node_he_ptr + i);
    const int* L = P.node_vpos_ell + i;
    const size_t ms = P.ms;
    int j = 0;
    for (; j + 4 <= n; j += 4) {
      const int e0 = ld1<CS>(L + j * ms), e1 = ld1<CS>(L + (j + 1) * ms), e2 = ld1<CS>(L + (j + 2) * ms),
                e3 = ld1<CS>(L + (j + 3) * ms);
      const double f0 = P.exf2d[e0 >> 1], f1 = P.exf2d[e1 >> 1], f2 = P.exf2d[e2 >> 1], f3 = P.exf2d[e3 >> 1];
      x = (e0 & 1) ? x + f0 : x - f0;
      x = (e1 & 1) ? x + f1 : x - f1;
      x = (e2 & 1) ? x + f2 : x - f2;
      x = (e3 & 1) ? x + f3 : x - f3;
    }
    for (; j < n; ++j) {
      const int e = ld1<CS>(L + j * ms);
      const double exflux = P.exf2d[e >> 1];
      x = (e & 1) ? x + exflux : x - exflux;
    }
  }
  // the previous stage's node judgement, its cell flags now in ISWETCE (roles swapped)
  if (parts & EN_WET_PREV) wet_node<CS>(P, i, P.iswetce);
  if (parts & EN_FINISH_PREV) ext_update_node<CS>(P, i, (parts >> 8) & 7);
  if (parts & EN_COPY_ELRK) P.elrk[i] = P.el[i];
  const double alpha = dAlphaRK[K];
  int ob = ld1<CS>(P.node_obc + i);
  if (parts & EN_EXTEL) {
    if (ob > 0) {
      P.xflux_obcn[ob] = x;
      x = 0.0;
    }
    for (int q = P.node_riv_ptr[i]; q < P.node_riv_ptr[i + 1]; ++q) {
      int r = P.node_riv[q];
      int j = r >> 1;
      if (P.river_location == 0)
        x = x - P.qdis[j];
      else
        x = x - P.qdis[j] * P.rdisq[(size_t)(r & 1) * (P.numqbc + 1) + j];
    }
    double dtk = alpha * P.dte;
    P.elf[i] = ld1<CS>(P.elrk + i) - dtk * x / ld1<CS>(P.art1 + i);
  }
  if ((parts & EN_BC) && ob > 0) {
    int kind = P.obc_kind[ob];
    if (kind == 1) {
      if (P.obc_elev_on) {
        const double* row = sched_row(P);
        double force = 0.0;
        for (int j = 0; j < P.ntide; ++j) {
          size_t q = (size_t)j * (P.iobcn + 1) + ob;
          double targ = row[P.sl.targ(iext, K, j)];
          force = P.apt[q] * cos(targ - P.phai_rad[q]) + force;
        }
        force = force + P.emean[ob];
        P.elf[i] = force * row[P.sl.ramp_ext(iext)];
      }
      P.elf[i] = P.elrk[i] + alpha * (P.elf[i] - P.elrk[i]);
    } else if (kind == 2) {
      P.elf[i] = 0.0;
    }
  }
}

// One job per thread, 48 registers (five blocks of 256 per SM; at 40 registers it
// spills).  Measured slower on the 200k-node mesh: a grid of five blocks per SM whose
// threads walk the jobs (1.14 -> 1.29 ms per step), and blocks that each mix three warps
// of node jobs with five of gradient jobs (1.13 -> 1.45 ms).
template <bool CS>
__global__ void __launch_bounds__(256, 5) k_ext_node(const Dev P, int iext, int K, int parts) {
  pdl_enter();
  const int n = (parts & EN_GRAD) ? P.M + P.N : P.M;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i <= n) ext_node_job<CS>(P, i, iext, K, parts);
}

// -------------------------------------------------------------------------------------
// WET_JUDGE (mod_wd.F:193-284) in two passes.  Cells first: the cell flag uses the
// unclamped ELF of its nodes, and ELF1 is the mean of the clamped ELF, which each cell
// forms itself from h and ELF.  Then nodes: the node flag and the clamp of ELF.
// -------------------------------------------------------------------------------------
template <bool CS>
__device__ __forceinline__ void wet_cell(const Dev& P, const int i) {
  int n1 = ld1<CS>(P.nv + i), n2 = ld1<CS>(P.nv + (size_t)(P.N + 1) + i), n3 = ld1<CS>(P.nv + (size_t)2 * (P.N + 1) + i);
  double e1 = P.elf[n1], e2 = P.elf[n2], e3 = P.elf[n3];
  double dtmp = fmax(fmax(e1, e2), e3) + fmin(fmin(P.h[n1], P.h[n2]), P.h[n3]);
  P.iswetc[i] = ((dtmp - P.min_depth) < 1.0e-5) ? 0 : 1;
  double c1 = fmax(e1, -P.h[n1] + P.min_depth);
  double c2 = fmax(e2, -P.h[n2] + P.min_depth);
  double c3 = fmax(e3, -P.h[n3] + P.min_depth);
  P.elf1[i] = ONE_THIRD * (c1 + c2 + c3);
}
template <bool CS>
__global__ void k_wet_cells(const Dev P) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i <= P.N) wet_cell<CS>(P, i);
}

__global__ void k_wet_nodes(const Dev P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  wet_node(P, i, P.iswetc);
}

// ADVAVE_EDGE_GCN for one cell (advave_edge_gcn.F:115-1003, LIMITED_NO branch), over the
// cell's slot table.  The edge fluxes are evaluated in R; the surface-slope pressure
// gradient PSTX/PSTY stays FP64.
template <typename R, bool LIM>
__device__ inline void advave_cell(const Dev& P, int i, double& xfo, double& yfo, double& px, double& py) {
  typedef Mesh<R> Mh;
  const R half = (R)0.5, one = (R)1.0;
  R xf = 0, yf = 0;
  px = 0.0; py = 0.0;
  const size_t n1 = P.N + 1;
  const R epor = (R)P.epor[i], iucp = (R)P.iucp[i];
  // The cell's own side of its three edges is loaded once; per edge only the other
  // cell's gradient, UA, VA, ART, CC_HVC and wet flags are gathered (FP32 form).
  const Grad<R> gi = load_grad<R>(P, i);
  const R ui = (R)P.ua[i], vi = (R)P.va[i], arti = Mh::art(P, i), cci = Mh::cc_hvc(P, i);
  const int weti = P.iswetce[i] * P.iswetc[i];
  const double ged1 = P.grav_e[i] * P.d1[i];
  for (int s = 0; s < 3; ++s) {
    const size_t q = (size_t)s * n1 + i;
    const int4 ci = P.ce_i4[q];  // {code, IA, IB, J1}
    const int code = ci.x;
    const int side = code & 1;
    const int ia = ci.y, ib = ci.z;
    const int j1 = ci.w, j2 = P.ce_j2[q];
    R dij = (R)(0.5 * (P.d[j1] + P.d[j2]));
    double elij = 0.5 * (P.el[j1] + P.el[j2]);
    const int o = side == 0 ? ib : ia;  // the other cell of the edge
    if (weti == 1 || P.iswetce[o] * P.iswetc[o] == 1) {
      R uij1, vij1, uij2, vij2;
      Grad<R> ga, gb;
      R arta, artb, cca, ccb;
      if constexpr (!LIM && sizeof(R) == 8) {
        // FP64: per-edge loads of both sides keep the kernel at 108 registers
        ga = load_grad<R>(P, ia);
        R xij = Mh::s_xoa(P, q);
        R yij = Mh::s_yoa(P, q);
        uij1 = (R)P.ua[ia] + ga.ux * xij + ga.uy * yij;
        vij1 = (R)P.va[ia] + ga.vx * xij + ga.vy * yij;
        gb = load_grad<R>(P, ib);
        xij = Mh::s_xob(P, q);
        yij = Mh::s_yob(P, q);
        uij2 = (R)P.ua[ib] + gb.ux * xij + gb.uy * yij;
        vij2 = (R)P.va[ib] + gb.vx * xij + gb.vy * yij;
        arta = Mh::art(P, ia);
        artb = Mh::art(P, ib);
        cca = Mh::cc_hvc(P, ia);
        ccb = Mh::cc_hvc(P, ib);
      } else if constexpr (!LIM) {
        const Grad<R> go = load_grad<R>(P, o);
        const R uo = (R)P.ua[o], vo = (R)P.va[o];
        ga = side == 0 ? gi : go;
        gb = side == 0 ? go : gi;
        const R uia = side == 0 ? ui : uo, via = side == 0 ? vi : vo;
        const R uib = side == 0 ? uo : ui, vib = side == 0 ? vo : vi;
        const auto G = Mh::s_geo(P, q);  // XOA, YOA, XOB, YOB
        uij1 = uia + ga.ux * G.x + ga.uy * G.y;
        vij1 = via + ga.vx * G.x + ga.vy * G.y;
        uij2 = uib + gb.ux * G.z + gb.uy * G.w;
        vij2 = vib + gb.vx * G.z + gb.vy * G.w;
        const R arto = Mh::art(P, o), cco = Mh::cc_hvc(P, o);
        arta = side == 0 ? arti : arto;
        artb = side == 0 ? arto : arti;
        cca = side == 0 ? cci : cco;
        ccb = side == 0 ? cco : cci;
      } else {
        arta = Mh::art(P, ia);
        artb = Mh::art(P, ib);
        cca = Mh::cc_hvc(P, ia);
        ccb = Mh::cc_hvc(P, ib);
        ga = load_grad<R>(P, ia);
        gb = load_grad<R>(P, ib);
        const R xija = Mh::s_xoa(P, q), yija = Mh::s_yoa(P, q);
        const R xijb = Mh::s_xob(P, q), yijb = Mh::s_yob(P, q);
        lim_faces<R>(P.limiter, (R)P.ua[ia], (R)P.ua[ib], ga.ux * xija + ga.uy * yija, gb.ux * xijb + gb.uy * yijb,
                     Mh::alfa2(P, 0)[ia], Mh::alfa2(P, 0)[ib], uij1, uij2);
        lim_faces<R>(P.limiter, (R)P.va[ia], (R)P.va[ib], ga.vx * xija + ga.vy * yija, gb.vx * xijb + gb.vy * yijb,
                     Mh::alfa2(P, 1)[ia], Mh::alfa2(P, 1)[ib], vij1, vij2);
      }
      R uij = half * (uij1 + uij2);
      R vij = half * (vij1 + vij2);
      const auto DD = Mh::s_dd(P, q);
      const R dltxc = DD.x, dltyc = DD.y;
      R un = -uij * dltyc + vij * dltxc;
      R viscof1 = arta * sqrt(ga.ux * ga.ux + ga.vy * ga.vy + half * ((ga.uy + ga.vx) * (ga.uy + ga.vx)));
      R viscof2 = artb * sqrt(gb.ux * gb.ux + gb.vy * gb.vy + half * ((gb.uy + gb.vx) * (gb.uy + gb.vx)));
      R viscof = ((R)P.fact * half * (viscof1 * cca + viscof2 * ccb) + (R)P.fm1 * half * (cca + ccb)) / (R)P.hprnu;
      R txx = (ga.ux + gb.ux) * viscof;
      R tyy = (ga.vy + gb.vy) * viscof;
      R txy = half * (ga.uy + gb.uy + ga.vx + gb.vx) * viscof;
      R fxx = dij * (txx * dltyc - txy * dltxc);
      R fyy = dij * (txy * dltyc - tyy * dltxc);
      R sg = fsign1(un);
      R xadv = dij * un * ((one - sg) * uij2 + (one + sg) * uij1) * half;
      R yadv = dij * un * ((one - sg) * vij2 + (one + sg) * vij1) * half;
      R nb = one - (R)((code >> 1) & 1);
      if (side == 0) {
        xf = xf + (xadv + fxx * epor) * nb * iucp;
        yf = yf + (yadv + fyy * epor) * nb * iucp;
      } else {
        xf = xf - (xadv + fxx * epor) * nb * iucp;
        yf = yf - (yadv + fyy * epor) * nb * iucp;
      }
    }
    const double edx = P.ce_dx[q], edy = P.ce_dy[q];
    if (side == 0) {
      px = px - ged1 * elij * edy;
      py = py + ged1 * elij * edx;
    } else {
      px = px + ged1 * elij * edy;
      py = py - ged1 * elij * edx;
    }
  }
  R w = (R)weti;
  xfo = (double)(xf * w);
  yfo = (double)(yf * w);
}

// FLUX_OBN (mod_obcs.F:1181-1215) value on one open-boundary cell.
__device__ inline double fluxobn_cell(const Dev& P, int i, int K) {
  double f = 0.0;
  for (int q = P.cell_obc_ptr[i]; q < P.cell_obc_ptr[i + 1]; ++q) {
    int code = P.cell_obc[q];
    int ob = code >> 1, slot = code & 1;
    int j = P.i_obc_n[ob];
    // ELF as WET_JUDGE leaves it (its node part may still be pending in a fused loop;
    // the clamp is idempotent)
    double ej = P.wetting_drying_on ? fmax(P.elf[j], -P.h[j] + P.min_depth) : P.elf[j];
    double flux = -(ej - P.elrk[j]) * P.art1[j] / (dAlphaRK[K] * P.dte) - P.xflux_obcn[ob];
    f = f + P.fluxf_obc[(size_t)slot * (P.iobcn + 1) + ob] * flux;
  }
  return f;
}

// River clamp / tangential projection of a solid-boundary cell (bcond_gcn.F:345-405).
__device__ inline void bc_solid(const Dev& P, int i, int rj, double& uu, double& vv) {
  if (rj > 0) {
    double ca = P.cos_angleq[rj], sa = P.sin_angleq[rj];
    double untmp = uu * ca + vv * sa;
    double vntmp = -uu * sa + vv * ca;
    untmp = fmax(untmp, 0.0);
    uu = untmp * ca - vntmp * sa;
    vv = untmp * sa + vntmp * ca;
  } else {
    double sa = P.sin_alpha[i], ca = P.cos_alpha[i];
    double ui = uu * (sa * sa) - vv * sa * ca;
    double vi = -uu * sa * ca + vv * (ca * ca);
    uu = ui;
    vv = vi;
  }
}

// -------------------------------------------------------------------------------------
// Per-cell part of one RK stage.  EC_INT_ADVAVE is the internal-step call of ADVAVE
// followed by ADX2D -= ADVUA (internal_step.F:387-392).
// -------------------------------------------------------------------------------------
template <typename R, bool LIM>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 8 : 1) k_ext_cell(const Dev P, int iext, int K, int parts) {
  pdl_enter();
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  const size_t n1 = P.N + 1;
  if (parts & EC_COPY_RK) {
    P.uark[i] = P.ua[i];
    P.vark[i] = P.va[i];
    P.elrk1[i] = P.el1[i];
  }
  if (parts & EC_N2E)
    P.elf1[i] = ONE_THIRD * (P.elf[P.nv[i]] + P.elf[P.nv[n1 + i]] + P.elf[P.nv[2 * n1 + i]]);
  double fob = 0.0;
  if (parts & EC_FLUXOBN) {
    fob = fluxobn_cell(P, i, K);
    P.fluxobn[i] = fob;
  } else if (P.isbce[i] == 2) {
    fob = P.fluxobn[i];
  }
  double xf, yf, px, py;
  if (parts & (EC_ADVAVE | EC_INT_ADVAVE)) {
    advave_cell<R, LIM>(P, i, xf, yf, px, py);
    if (P.isbce[i] == 2) {
      if (P.gcy) {  // advave_edge_gcy.F
        xf = xf + fob * P.ua[i] * P.iucp[i];
        yf = yf + fob * P.va[i] * P.iucp[i];
      } else {
        xf = (xf + fob * P.ua[i]) * P.iucp[i];
        yf = (yf + fob * P.va[i]) * P.iucp[i];
      }
    }
    for (int q = P.cell_riv_ptr[i]; q < P.cell_riv_ptr[i + 1]; ++q) {
      int k = P.cell_riv[q] >> 1;
      double vlctyq = P.qdis[k] / P.qarea[k];
      if (P.river_location == 0) {
        xf = xf - 0.5 * P.qdis[k] * vlctyq * P.cos_angleq[k];
        yf = yf - 0.5 * P.qdis[k] * vlctyq * P.sin_angleq[k];
      } else {
        double temp = P.qdis[k] * vlctyq;
        xf = xf - temp * P.cos_angleq[k];
        yf = yf - temp * P.sin_angleq[k];
      }
    }
    P.advua[i] = xf;
    P.advva[i] = yf;
    P.pstx[i] = px;
    P.psty[i] = py;
    if (parts & EC_INT_ADVAVE) {
      P.adx2d[i] = P.adx2d[i] - xf;
      P.ady2d[i] = P.ady2d[i] - yf;
    }
  } else {
    xf = P.advua[i];
    yf = P.advva[i];
    px = P.pstx[i];
    py = P.psty[i];
  }
  if (parts & (EC_EXTUV | EC_BC2)) {
    double uaf, vaf;
    if (parts & EC_EXTUV) {
      // EXTUV_EDGE(K) (extuv_edge.F:106-163)
      if (P.iswetce[i] * P.iswetc[i] == 1) {
        double ramp = sched_row(P)[P.sl.ramp_ext(iext)];
        double wus = P.have_wind ? P.wsx[i] * ramp * 0.001 : 0.0;
        double wvs = P.have_wind ? P.wsy[i] * ramp * 0.001 : 0.0;
        double resx = P.adx2d[i] + xf + P.drx2d[i] + px - P.cor[i] * P.va[i] * P.d1[i] * P.art[i] -
                      (wus + P.wubot[i]) * P.art[i];
        double resy = P.ady2d[i] + yf + P.dry2d[i] + py + P.cor[i] * P.ua[i] * P.d1[i] * P.art[i] -
                      (wvs + P.wvbot[i]) * P.art[i];
        double a = dAlphaRK[K];
        uaf = (P.uark[i] * (P.h1[i] + P.elrk1[i]) - a * P.dte * resx / P.art[i]) / (P.h1[i] + P.elf1[i]);
        vaf = (P.vark[i] * (P.h1[i] + P.elrk1[i]) - a * P.dte * resy / P.art[i]) / (P.h1[i] + P.elf1[i]);
      } else {
        uaf = 0.0;
        vaf = 0.0;
      }
      uaf = uaf / (1.0 + P.cc_sponge[i] * (uaf * uaf));
      vaf = vaf / (1.0 + P.cc_sponge[i] * (vaf * vaf));
    } else {
      uaf = P.uaf[i];
      vaf = P.vaf[i];
    }
    if (parts & EC_BC2) {
      // BCOND_GCN(2,K) (bcond_gcn.F:325-406)
      int b = P.isbce[i];
      // GCY (bcond_gcy.F): the river clamp only, no tangential projection or corner zero
      if (b == 3 && !P.gcy) { uaf = 0.0; vaf = 0.0; }
      if (b == 1 && (!P.gcy || P.cell_bcriv[i] > 0)) bc_solid(P, i, P.cell_bcriv[i], uaf, vaf);
    }
    P.uaf[i] = uaf;
    P.vaf[i] = vaf;
    if (parts & EC_FINISH) ext_update_cell(P, i, K, uaf, vaf);
  }
}

#ifdef FVG_F32_TU
// -------------------------------------------------------------------------------------
// Compact cell kernel of the precision form's stage loop (F32::compact; no limiter, GCN).
// The same steps as k_ext_cell<float, false> -- FLUX_OBN, ADVAVE's edge loop in FP32 with
// the FP64 surface-slope pressure gradient, EXTUV_EDGE and BCOND_GCN(2) in FP64, the cell
// part of the stage's update -- over smaller records:
//   * a slot is {code, other cell, IENODE1, IENODE2}; the edge's geometry is formed in FP64
//     from the node and cell coordinates (XIJC = (VX1+VX2)/2, DLTXC = VX2-VX1, the offsets
//     XIJC-XC rounded once to FP32, DLTXE = XIJC-XC of this cell for the continuity flux),
//     values fvg_set_precision has checked equal, bit for bit, to the mesh's own metrics;
//   * EXTUV's terms that stay fixed over the external loop are summed once per internal
//     step (exc0, exc1, written by the internal-step ADVAVE call of this kernel), so that a
//     stage reads five FP64 values per cell for them instead of thirteen;
//   * ADVUA, ADVVA, PSTX, PSTY, which no later stage reads, are stored by the last stage
//     (EC_LAST) and the internal-step call only.
// -------------------------------------------------------------------------------------
// 64 registers (eight blocks per SM): held to 80 registers, six blocks, it measured slower
// (1.89 against 1.76 ms per step).
// CS: the records the stage reads once (flags, slots, EXTUV's fixed terms, the Runge-Kutta
// start values, the cell's own D1/ELF1/EL1) are loaded evict-first (ld1), so that what
// neighbours gather (UA, VA, the gradients, ART/CC_HVC, XC/YC, the nodes' VX/VY, D, EL,
// the wet flags) keeps its L2 lines between stages.
template <bool CS>
__device__ __forceinline__ void ext_cell_c(const Dev& P, const int i, int iext, int K, int parts) {
  const size_t n1 = P.N + 1;
  const int fl = ld1<CS>(P.f.cflag + i);
  const int isbce = fl & 3;
  const double ua_i = P.ua[i], va_i = P.va[i];
  if (parts & EC_COPY_RK) {
    P.uark[i] = ua_i;
    P.vark[i] = va_i;
    P.elrk1[i] = ld1<CS>(P.el1 + i);
  }
  double elf1 = 0.0;
  if (parts & EC_N2E) {
    elf1 = ONE_THIRD * (P.elf[ld1<CS>(P.nv + i)] + P.elf[ld1<CS>(P.nv + n1 + i)] + P.elf[ld1<CS>(P.nv + 2 * n1 + i)]);
    P.elf1[i] = elf1;
  } else if (parts & (EC_EXTUV | EC_FINISH)) {
    elf1 = ld1<CS>(P.elf1 + i);
  }
  double fob = 0.0;
  if (parts & EC_FLUXOBN) {
    if (fl & 32) fob = fluxobn_cell(P, i, K);
    if ((fl & 32) || isbce == 2) P.fluxobn[i] = fob;
  } else if (isbce == 2) {
    fob = P.fluxobn[i];
  }
  const int weti = P.iswetce[i] * P.iswetc[i];
  const double d1i = ld1<CS>(P.d1 + i);
  // {COR*ART, ART, H1, GRAV_E}: formed by the internal-step call below, read by the stages
  const double4 e1 = (parts & EC_INT_ADVAVE) ? make_double4(0.0, 0.0, 0.0, P.grav_e[i]) : ld1<CS>(P.f.exc1 + i);
  double xf = 0.0, yf = 0.0, px = 0.0, py = 0.0;
  if (parts & (EC_ADVAVE | EC_INT_ADVAVE)) {
    const float half = 0.5f, one = 1.0f;
    const double ged1 = e1.w * d1i;
    const float4 gi4 = P.f.g2d4[i];
    const float2 aci = P.f.artcc[i];
    const double2 xyi = P.f.xyc[i];
    const float ui = (float)ua_i, vi = (float)va_i;
    const float epor = (fl & 8) ? 1.0f : 0.0f, iucp = (fl & 4) ? 1.0f : 0.0f;
    float xr = 0.f, yr = 0.f;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int4 sl = ld1<CS>(P.f.slot4 + (size_t)s * n1 + i);  // {code, other cell, IENODE1, IENODE2}
      const int code = sl.x, side = code & 1, o = sl.y, j1 = sl.z, j2 = sl.w;
      const double2 v1 = P.f.vxy[j1], v2 = P.f.vxy[j2];
      const double xijc = (v1.x + v2.x) / 2.0, yijc = (v1.y + v2.y) / 2.0;
      const double dltxc = v2.x - v1.x, dltyc = v2.y - v1.y;
      const float dij = (float)(0.5 * (P.d[j1] + P.d[j2]));
      const double elij = 0.5 * (P.el[j1] + P.el[j2]);
      if (weti == 1 || P.iswetce[o] * P.iswetc[o] == 1) {
        const float4 go4 = P.f.g2d4[o];
        const float2 aco = P.f.artcc[o];
        const double2 xyo = P.f.xyc[o];
        const float uo = (float)P.ua[o], vo = (float)P.va[o];
        const float xoi = (float)(xijc - xyi.x), yoi = (float)(yijc - xyi.y);
        const float xoo = (float)(xijc - xyo.x), yoo = (float)(yijc - xyo.y);
        // side 0: this cell is IA; side 1: this cell is IB
        const float4 ga = side == 0 ? gi4 : go4, gb = side == 0 ? go4 : gi4;
        const float uia = side == 0 ? ui : uo, via = side == 0 ? vi : vo;
        const float uib = side == 0 ? uo : ui, vib = side == 0 ? vo : vi;
        const float xa = side == 0 ? xoi : xoo, ya = side == 0 ? yoi : yoo;
        const float xb = side == 0 ? xoo : xoi, yb = side == 0 ? yoo : yoi;
        const float arta = side == 0 ? aci.x : aco.x, artb = side == 0 ? aco.x : aci.x;
        const float cca = side == 0 ? aci.y : aco.y, ccb = side == 0 ? aco.y : aci.y;
        // ga = {UX, UY, VX, VY} of IA, gb of IB
        const float uij1 = uia + ga.x * xa + ga.y * ya;
        const float vij1 = via + ga.z * xa + ga.w * ya;
        const float uij2 = uib + gb.x * xb + gb.y * yb;
        const float vij2 = vib + gb.z * xb + gb.w * yb;
        const float uij = half * (uij1 + uij2);
        const float vij = half * (vij1 + vij2);
        const float dx = (float)dltxc, dy = (float)dltyc;
        const float un = -uij * dy + vij * dx;
        const float viscof1 = arta * sqrtf(ga.x * ga.x + ga.w * ga.w + half * ((ga.y + ga.z) * (ga.y + ga.z)));
        const float viscof2 = artb * sqrtf(gb.x * gb.x + gb.w * gb.w + half * ((gb.y + gb.z) * (gb.y + gb.z)));
        const float viscof =
            ((float)P.fact * half * (viscof1 * cca + viscof2 * ccb) + (float)P.fm1 * half * (cca + ccb)) / (float)P.hprnu;
        const float txx = (ga.x + gb.x) * viscof;
        const float tyy = (ga.w + gb.w) * viscof;
        const float txy = half * (ga.y + gb.y + ga.z + gb.z) * viscof;
        const float fxx = dij * (txx * dy - txy * dx);
        const float fyy = dij * (txy * dy - tyy * dx);
        const float sg = fsign1(un);
        const float xadv = dij * un * ((one - sg) * uij2 + (one + sg) * uij1) * half;
        const float yadv = dij * un * ((one - sg) * vij2 + (one + sg) * vij1) * half;
        const float nb = one - (float)((code >> 1) & 1);
        if (side == 0) {
          xr = xr + (xadv + fxx * epor) * nb * iucp;
          yr = yr + (yadv + fyy * epor) * nb * iucp;
        } else {
          xr = xr - (xadv + fxx * epor) * nb * iucp;
          yr = yr - (yadv + fyy * epor) * nb * iucp;
        }
      }
      if (side == 0) {
        px = px - ged1 * elij * dltyc;
        py = py + ged1 * elij * dltxc;
      } else {
        px = px + ged1 * elij * dltyc;
        py = py - ged1 * elij * dltxc;
      }
    }
    const float w = (float)weti;
    xf = (double)(xr * w);
    yf = (double)(yr * w);
    if (isbce == 2) {
      const double iu = (fl & 4) ? 1.0 : 0.0;
      xf = (xf + fob * ua_i) * iu;
      yf = (yf + fob * va_i) * iu;
    }
    if (fl & 16) {
      for (int q = P.cell_riv_ptr[i]; q < P.cell_riv_ptr[i + 1]; ++q) {
        int k = P.cell_riv[q] >> 1;
        double vlctyq = P.qdis[k] / P.qarea[k];
        if (P.river_location == 0) {
          xf = xf - 0.5 * P.qdis[k] * vlctyq * P.cos_angleq[k];
          yf = yf - 0.5 * P.qdis[k] * vlctyq * P.sin_angleq[k];
        } else {
          double temp = P.qdis[k] * vlctyq;
          xf = xf - temp * P.cos_angleq[k];
          yf = yf - temp * P.sin_angleq[k];
        }
      }
    }
    if (parts & (EC_LAST | EC_INT_ADVAVE)) {
      P.advua[i] = xf;
      P.advva[i] = yf;
      P.pstx[i] = px;
      P.psty[i] = py;
    }
    if (parts & EC_INT_ADVAVE) {
      // ADX2D -= ADVUA (internal_step.F:387-392), then EXTUV's fixed terms of the coming
      // external loop
      const double adx = P.adx2d[i] - xf, ady = P.ady2d[i] - yf;
      P.adx2d[i] = adx;
      P.ady2d[i] = ady;
      const double art = P.art[i];
      const double wx = P.have_wind ? 0.001 * P.wsx[i] * art : 0.0;
      const double wy = P.have_wind ? 0.001 * P.wsy[i] * art : 0.0;
      P.f.exc0[i] = make_double4(adx + P.drx2d[i] - P.wubot[i] * art, ady + P.dry2d[i] - P.wvbot[i] * art, wx, wy);
      P.f.exc1[i] = make_double4(P.cor[i] * art, art, P.h1[i], P.grav_e[i]);
    }
  }
  if (parts & (EC_EXTUV | EC_BC2)) {
    double uaf = 0.0, vaf = 0.0;
    if (parts & EC_EXTUV) {
      if (weti == 1) {
        const double4 e0 = ld1<CS>(P.f.exc0 + i);
        const double ramp = sched_row(P)[P.sl.ramp_ext(iext)];
        const double resx = e0.x + xf + px - e1.x * va_i * d1i - ramp * e0.z;
        const double resy = e0.y + yf + py + e1.x * ua_i * d1i - ramp * e0.w;
        const double a = dAlphaRK[K];
        const double uark = (parts & EC_COPY_RK) ? ua_i : ld1<CS>(P.uark + i);
        const double vark = (parts & EC_COPY_RK) ? va_i : ld1<CS>(P.vark + i);
        const double elrk1 = (parts & EC_COPY_RK) ? ld1<CS>(P.el1 + i) : ld1<CS>(P.elrk1 + i);
        uaf = (uark * (e1.z + elrk1) - a * P.dte * resx / e1.y) / (e1.z + elf1);
        vaf = (vark * (e1.z + elrk1) - a * P.dte * resy / e1.y) / (e1.z + elf1);
      }
      if (fl & 64) {
        const double sp = P.cc_sponge[i];
        uaf = uaf / (1.0 + sp * (uaf * uaf));
        vaf = vaf / (1.0 + sp * (vaf * vaf));
      }
    } else {
      uaf = P.uaf[i];
      vaf = P.vaf[i];
    }
    if (parts & EC_BC2) {
      if (isbce == 3) { uaf = 0.0; vaf = 0.0; }
      if (isbce == 1) bc_solid(P, i, P.cell_bcriv[i], uaf, vaf);
    }
    P.uaf[i] = uaf;
    P.vaf[i] = vaf;
    if (parts & EC_FINISH) {
      // cell part of the stage's update (ext_update_cell) with DLTXE, DLTYE = XIJC-XC
      P.el1[i] = elf1;
      const double dd1 = e1.z + elf1;
      P.d1[i] = dd1;
      if (K == 3) {
        P.uard[i] = ld1<CS>(P.uard + i) + uaf * dd1;
        P.vard[i] = ld1<CS>(P.vard + i) + vaf * dd1;
      }
      const double2 xyi = P.f.xyc[i];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const int4 sl = ld1<CS>(P.f.slot4 + (size_t)s * n1 + i);
        const double2 v1 = P.f.vxy[sl.z], v2 = P.f.vxy[sl.w];
        const double dxe = (v1.x + v2.x) / 2.0 - xyi.x, dye = (v1.y + v2.y) / 2.0 - xyi.y;
        P.exf2d[(size_t)s * P.ns + i] = dd1 * (-uaf * dye + vaf * dxe);
      }
    }
  }
}

// One cell per thread (WALK false), or a grid-stride walk over the cells with a grid of
// Dev::ext_grid blocks per SM (WALK true).
template <bool CS, bool WALK>
__global__ void __launch_bounds__(128, 8) k_ext_cell_c(const Dev P, int iext, int K, int parts) {
  pdl_enter();
  if constexpr (WALK) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i <= P.N; i += gridDim.x * blockDim.x)
      ext_cell_c<CS>(P, i, iext, K, parts);
  } else {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i <= P.N) ext_cell_c<CS>(P, i, iext, K, parts);
  }
}
#endif  // FVG_F32_TU

// -------------------------------------------------------------------------------------
// external_step.F:333-436: EL=ELF, EL1=N2E2D(EL), D, D1, UA=UAF, DTFA, the K==3 sums
// for the 3-D correction, the K==4 open-boundary transport and WD_UPDATE(1).
// -------------------------------------------------------------------------------------
__global__ void k_ext_update(const Dev P, int K) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i <= P.M) ext_update_node(P, i, K);
  if (i <= P.N) {
    double u = P.uaf[i], v = P.vaf[i];
    P.ua[i] = u;
    P.va[i] = v;
    if (P.wetting_drying_on) P.iswetce[i] = P.iswetc[i];
    ext_update_cell(P, i, K, u, v);
  }
}

// After the last stage of a fused external loop: the node part of its update, and UAF,
// VAF, ISWETC made equal to UA, VA, ISWETCE as the copying update leaves them.
__global__ void k_ext_finish(const Dev P, int K, int wet_prev) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i <= P.M) {
    if (wet_prev) wet_node(P, i, P.iswetce);
    ext_update_node(P, i, K);
  }
  if (i <= P.N) {
    P.uaf[i] = P.ua[i];
    P.vaf[i] = P.va[i];
    P.iswetc[i] = P.iswetce[i];
  }
}
__global__ void k_ext_prep(const Dev P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.N) return;
  store_grad<false>(P, i);
  store_exf(P, i);
}

// Start of an internal step: advance the schedule slot, then BCOND_GCN(8,0)'s river ramp
// QDIS = QDIS*RAMP (bcond_gcn.F:645-648).
__global__ void k_begin_step(const Dev P, int advance) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int slot = P.ctl[0] + advance;
  P.ctl[0] = slot;
  double ramp = P.sched[(size_t)slot * P.sl.len];
  for (int j = 1; j <= P.numqbc; ++j) P.qdis[j] = P.qdis0[j] * ramp;
}

static inline int nblk(int n, int b) { return (n + b - 1) / b; }

void launch_ext_node(const Dev& P, cudaStream_t s, int iext, int K, int parts, int pdl) {
  const int n = (parts & EN_GRAD) ? P.M + P.N : P.M;
  launch_maybe_pdl(pdl, P.ldcs ? k_ext_node<true> : k_ext_node<false>, dim3(nblk(n, 256)), dim3(256), s, P, iext, K,
                   parts);
}
void launch_ext_prep(const Dev& P, cudaStream_t s) { k_ext_prep<<<nblk(P.N, 256), 256, 0, s>>>(P); }
void launch_alfa2(const Dev& P, cudaStream_t s) {
  FVG_F32_FORWARD(launch_alfa2(P, s));
  k_alfa2<RF><<<nblk(P.N, 128), 128, 0, s>>>(P);
}

// FP32 copies of the mesh metrics the precision form's flux kernels read.
__global__ void k_d2f(const double* __restrict__ src, float* __restrict__ dst, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    dst[q] = (float)src[q];
}
__global__ void k_edge_offsets_f32(const Dev P) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > P.NE) return;
  const size_t e1 = P.NE + 1;
  float xa = 0.f, ya = 0.f, xb = 0.f, yb = 0.f;
  if (e >= 1) {
    int ia = P.iec[e], ib = P.iec[e1 + e];
    xa = (float)(P.xijc[e] - P.xc[ia]);
    ya = (float)(P.yijc[e] - P.yc[ia]);
    xb = (float)(P.xijc[e] - P.xc[ib]);
    yb = (float)(P.yijc[e] - P.yc[ib]);
  }
  P.f.xo[e] = xa;
  P.f.yo[e] = ya;
  P.f.xo[e1 + e] = xb;
  P.f.yo[e1 + e] = yb;
}
// FP32 slot metrics packed per slot, each value rounded once from FP64
__global__ void k_pack_slots_f32(const Dev P) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * (size_t)(P.N + 1)) return;
  P.f.ce_geo[q] = make_float4((float)P.ce_xoa[q], (float)P.ce_yoa[q], (float)P.ce_xob[q], (float)P.ce_yob[q]);
  P.f.ce_dd[q] = make_float2((float)P.ce_dx[q], (float)P.ce_dy[q]);
}
// FP32 half-edge metrics per position and ring-edge metrics, packed, rounded once
__global__ void k_pack_he_f32(const Dev P) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t pl = P.ncvs;
  if (q < pl) {
    P.f.hg4[q] = make_float4((float)P.hg[q], (float)P.hg[pl + q], (float)P.hg[2 * pl + q], (float)P.hg[3 * pl + q]);
    P.f.hg2[q] = make_float2((float)P.hg[4 * pl + q], (float)P.hg[5 * pl + q]);
  }
  if (q < (size_t)P.trie_n) P.f.trie[q] = make_float2((float)P.dltytrie[q], (float)P.dltxtrie[q]);
  const size_t n1 = P.N + 1;
  if (q < n1) {
    P.f.a1u4[q] = make_float4((float)P.a1u[q], (float)P.a1u[n1 + q], (float)P.a1u[2 * n1 + q], (float)P.a1u[3 * n1 + q]);
    P.f.a2u4[q] = make_float4((float)P.a2u[q], (float)P.a2u[n1 + q], (float)P.a2u[2 * n1 + q], (float)P.a2u[3 * n1 + q]);
  }
}
void launch_make_f32(const Dev& P, cudaStream_t s) {
  auto cvt = [&](const double* a, float* b, size_t n) { k_d2f<<<296, 256, 0, s>>>(a, b, n); };
  const size_t n1 = P.N + 1, e1 = P.NE + 1;
  k_edge_offsets_f32<<<nblk(P.NE + 1, 256), 256, 0, s>>>(P);
  cvt(P.dltxc, P.f.dltxc, e1);
  cvt(P.dltyc, P.f.dltyc, e1);
  cvt(P.art, P.f.art, n1);
  cvt(P.cc_hvc, P.f.cc_hvc, n1);
  cvt(P.a1u, P.f.a1u, 4 * n1);
  cvt(P.a2u, P.f.a2u, 4 * n1);
  cvt(P.ce_xoa, P.f.ce_xoa, 3 * n1);
  cvt(P.ce_yoa, P.f.ce_yoa, 3 * n1);
  cvt(P.ce_xob, P.f.ce_xob, 3 * n1);
  cvt(P.ce_yob, P.f.ce_yob, 3 * n1);
  cvt(P.ce_dx, P.f.ce_dx, 3 * n1);
  cvt(P.ce_dy, P.f.ce_dy, 3 * n1);
  k_pack_slots_f32<<<nblk(3 * (P.N + 1), 256), 256, 0, s>>>(P);
  size_t npk = P.ncvs > P.trie_n ? P.ncvs : P.trie_n;
  if ((size_t)P.N + 1 > npk) npk = P.N + 1;
  k_pack_he_f32<<<nblk(npk, 256), 256, 0, s>>>(P);
}
#ifndef FVG_F32_TU
// Records of the compact stage kernel, and the count of mesh metrics that differ from the
// values the kernel forms from the coordinates (then the compact kernel is not used).
__global__ void k_make_compact(const Dev P, int* mismatch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= P.M) P.f.vxy[i] = make_double2(P.vx[i], P.vy[i]);
  if (i > P.N) return;
  P.f.xyc[i] = make_double2(P.xc[i], P.yc[i]);
  P.f.artcc[i] = make_float2((float)P.art[i], (float)P.cc_hvc[i]);
  if (i == 0) return;
  const size_t n1 = P.N + 1;
  int bad = 0;
  for (int s = 0; s < 3; ++s) {
    const size_t q = (size_t)s * n1 + i;
    const int code = P.ce_code[q], ia = P.ce_ia[q], ib = P.ce_ib[q], j1 = P.ce_j1[q], j2 = P.ce_j2[q];
    const int side = code & 1;
    if ((side == 0 ? ia : ib) != i) ++bad;
    P.f.slot4[q] = make_int4(code, side == 0 ? ib : ia, j1, j2);
    const double xijc = (P.vx[j1] + P.vx[j2]) / 2.0, yijc = (P.vy[j1] + P.vy[j2]) / 2.0;
    if (xijc - P.xc[ia] != P.ce_xoa[q] || yijc - P.yc[ia] != P.ce_yoa[q]) ++bad;
    if (xijc - P.xc[ib] != P.ce_xob[q] || yijc - P.yc[ib] != P.ce_yob[q]) ++bad;
    if (P.vx[j2] - P.vx[j1] != P.ce_dx[q] || P.vy[j2] - P.vy[j1] != P.ce_dy[q]) ++bad;
    const size_t pos = (size_t)s * P.ns + i;
    if (P.hg[pos] != xijc - P.xc[i] || P.hg[P.ncvs + pos] != yijc - P.yc[i]) ++bad;
  }
  const double iu = P.iucp[i], ep = P.epor[i];
  if (!(iu == 0.0 || iu == 1.0) || !(ep == 0.0 || ep == 1.0)) ++bad;
  int fl = P.isbce[i] & 3;
  if (iu == 1.0) fl |= 4;
  if (ep == 1.0) fl |= 8;
  if (P.cell_riv_ptr[i + 1] > P.cell_riv_ptr[i]) fl |= 16;
  if (P.cell_obc_ptr[i + 1] > P.cell_obc_ptr[i]) fl |= 32;
  if (P.cc_sponge[i] != 0.0) fl |= 64;
  P.f.cflag[i] = fl;
  if (bad) atomicAdd(mismatch, bad);
}
void launch_make_compact(const Dev& P, cudaStream_t s, int* mismatch) {
  const int n = (P.M > P.N ? P.M : P.N) + 1;
  k_make_compact<<<nblk(n, 256), 256, 0, s>>>(P, mismatch);
}
#endif

void launch_wet_judge(const Dev& P, cudaStream_t s) {
  k_wet_cells<false><<<nblk(P.N, 256), 256, 0, s>>>(P);
  k_wet_nodes<<<nblk(P.M, 256), 256, 0, s>>>(P);
}
void launch_wet_cells(const Dev& P, cudaStream_t s, int pdl) {
  launch_maybe_pdl(pdl, P.ldcs ? k_wet_cells<true> : k_wet_cells<false>, dim3(nblk(P.N, 256)), dim3(256), s, P);
}
void launch_ext_cell(const Dev& P, cudaStream_t s, int iext, int K, int parts, int pdl) {
  FVG_F32_FORWARD(launch_ext_cell(P, s, iext, K, parts, pdl));
  void (*k)(const Dev, int, int, int);
#ifdef FVG_F32_TU
  if ((parts & EC_COMPACT) && P.f.compact && !P.limiter && !P.gcy) {
    const int nb = nblk(P.N, 128);
    if (P.ext_grid > 0 && nb > P.ext_grid * P.nsm) {
      launch_maybe_pdl(pdl, P.ldcs ? k_ext_cell_c<true, true> : k_ext_cell_c<false, true>, dim3(P.ext_grid * P.nsm),
                       dim3(128), s, P, iext, K, parts);
    } else {
      launch_maybe_pdl(pdl, P.ldcs ? k_ext_cell_c<true, false> : k_ext_cell_c<false, false>, dim3(nb), dim3(128), s,
                       P, iext, K, parts);
    }
    return;
  }
#endif
  k = P.limiter ? k_ext_cell<RF, true> : k_ext_cell<RF, false>;
  launch_maybe_pdl(pdl, k, dim3(nblk(P.N, 128)), dim3(128), s, P, iext, K, parts);
}
void launch_ext_update(const Dev& P, cudaStream_t s, int K) {
  int n = P.M > P.N ? P.M : P.N;
  k_ext_update<<<nblk(n, 256), 256, 0, s>>>(P, K);
}
void launch_ext_finish(const Dev& P, cudaStream_t s, int K, int wet_prev) {
  int n = P.M > P.N ? P.M : P.N;
  k_ext_finish<<<nblk(n, 256), 256, 0, s>>>(P, K, wet_prev);
}
void launch_begin_step(const Dev& P, cudaStream_t s) { k_begin_step<<<1, 32, 0, s>>>(P, 1); }
void launch_set_qdis(const Dev& P, cudaStream_t s) { k_begin_step<<<1, 32, 0, s>>>(P, 0); }

}  // namespace fvg / fvg_f32
