// k_scalar.cu - node-centred scalar transport and turbulence of INTERNAL_STEP:
// ADV_Q/FCT_Q2/FCT_Q2L (adv_q.F, fct_q2.F, fct_q2l.F), VDIF_Q with the MY2.5 closure
// (vdif_q.F), ADV_T/ADV_S with FCT_T/FCT_S (adv_t.F, adv_s.F, fct_t.F, fct_s.F), VDIF_TS
// (vdif_ts.F), BCOND_TS (bcond_ts.F, mod_obcs.F:1223-1373), DENS2 (eqs_of_state.F) and the
// end-of-step shifts (internal_step.F:1034-1590).
//
// The node-ring gradients (PTPX.. over NBSN) and the ring extrema of the advected field
// are formed once per (node, layer) by k_grad into scratch fields.  Horizontal advection
// then runs in two phases: k_he_adv evaluates each control-volume half-edge flux once
// (one thread per cell and layer, the cell's three half-edges), and k_gather_q/_ts sum
// each node's half-edge fluxes with their signs in ascending half-edge order, which
// reproduces the reference's scatter sums bit for bit.  T and S (and Q2 and Q2L) are
// transported in the same launches since neither reads the other's update.
#include <cuda_bf16.h>

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
constexpr int kMaxKBs = 64;

static inline int nblk(int n, int b) { return (n + b - 1) / b; }

__device__ inline double F4(double x) { return (double)(float)x; }
__device__ inline int NBSN(const Dev& P, int i, int j) { return P.nbsn[(size_t)(j - 1) * (P.M + 1) + i]; }
__device__ inline double TRIEX(const Dev& P, int i, int j) { return P.dltxtrie[(size_t)(j - 1) * (P.M + 1) + i]; }
__device__ inline double TRIEY(const Dev& P, int i, int j) { return P.dltytrie[(size_t)(j - 1) * (P.M + 1) + i]; }

// One tracer's node data on layer k: value, ring gradients, ring extrema.
template <typename R>
struct TRec {
  R q, px, py, pxd, pyd, rmin, rmax;
  R vf;  // FP32 records: the node's VISCOFH on the record's layer or level (else unused)
};

// Storage of the ring gradients and extrema by arithmetic type.  FP64: six arrays per
// tracer (P.gq, P.gt).  FP32: one 32-byte record per tracer and (node, layer) in P.f.npk,
// record r = (K-1)*ms + I holding {value, PX, PY, PXD, PYD, min, max, VF} for tracer t at
// floats 16r + 8t, read and written as two float4; VF is the node's VISCOFH on the layer
// (T, S) or interpolated to the level (Q2, Q2L) as the half-edge fluxes take it, so that
// they need not gather it.
template <typename R> struct NodeRec;
template <> struct NodeRec<double> {
  __device__ static void store(const Dev& P, int mode, int t, size_t q, double, double px, double py, double pxd,
                               double pyd, double mn, double mx, double) {
    double* const* G = mode == 0 ? P.gq[t] : P.gt[t];
    G[0][q] = px;
    G[1][q] = py;
    G[2][q] = pxd;
    G[3][q] = pyd;
    G[4][q] = mn;
    G[5][q] = mx;
  }
  __device__ static TRec<double> load(const Dev& P, int mode, int t, size_t q, double qv) {
    double* const* G = mode == 0 ? P.gq[t] : P.gt[t];
    return TRec<double>{qv, G[0][q], G[1][q], G[2][q], G[3][q], G[4][q], G[5][q], 0.0};
  }
  __device__ static void minmax(const Dev& P, int mode, int t, size_t q, double& mn, double& mx) {
    double* const* G = mode == 0 ? P.gq[t] : P.gt[t];
    mn = G[4][q];
    mx = G[5][q];
  }
};
template <> struct NodeRec<float> {
  __device__ static float4* rec(const Dev& P, int t, size_t q) {
    return reinterpret_cast<float4*>(P.f.npk + 16 * q + 8 * t);
  }
  __device__ static void store(const Dev& P, int, int t, size_t q, float qv, float px, float py, float pxd,
                               float pyd, float mn, float mx, float vf) {
    float4* r = rec(P, t, q);
    r[0] = make_float4(qv, px, py, pxd);
    r[1] = make_float4(pyd, mn, mx, vf);
  }
  __device__ static TRec<float> load(const Dev& P, int, int t, size_t q, double) {
    const float4* r = rec(P, t, q);
    const float4 a = r[0], b = r[1];
    return TRec<float>{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  }
  __device__ static void minmax(const Dev& P, int, int t, size_t q, double& mn, double& mx) {
    const float4 b = rec(P, t, q)[1];
    mn = (double)b.y;
    mx = (double)b.z;
  }
};

template <typename R, int MODE>
__device__ inline TRec<R> load_trec(const Dev& P, int n, int k, int t) {
  const size_t q = N3(P, n, k);
  if (sizeof(R) == 8) {
    const double* Q = MODE == 0 ? (t == 0 ? P.q2 : P.q2l) : (t == 0 ? P.t1 : P.s1);
    return NodeRec<R>::load(P, MODE, t, q, Q[q]);
  }
  return NodeRec<R>::load(P, MODE, t, q, 0.0);
}

// -------------------------------------------------------------------------------------
// Ring gradients and extrema.  which == 0: Q2 and Q2L on K=2..KBM1 (adv_q.F:161-235);
// which == 1: T1 and S1 on K=1..KBM1 with the wet/dry substitution of adv_t.F:214-376,
// plus PFPXB/PFPYB and AH_BOTTOM at K=KBM1 (adv_t.F:394-408).
// -------------------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_grad(const Dev P, int which) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  int kb, ke;
  col_range(P, which == 0 ? 2 : 1, P.KBM1, kb, ke);
  const int nt = P.ntsn[i];
  const R art2 = (R)P.art2[i];
  const R half = (R)0.5;
  const R qmean = (R)F4(1.e-8);
  // One walk of the ring per layer serves both tracers: the ring node, its wet flag and
  // the ring-edge metrics are loaded once, and each neighbour's values are carried to
  // the next ring edge.  Per tracer the arithmetic is the reference's, term by term.
  for (int k = kb; k <= ke; ++k) {
    const double* Q[2];
    const double* QM[2] = {nullptr, nullptr};
    if (which == 0) {
      Q[0] = P.q2 + N3(P, 0, k);
      Q[1] = P.q2l + N3(P, 0, k);
    } else {
      Q[0] = P.t1 + N3(P, 0, k);
      Q[1] = P.s1 + N3(P, 0, k);
      QM[0] = P.tmean1 + N3(P, 0, k);
      QM[1] = P.smean1 + N3(P, 0, k);
    }
    R qi[2], qmi[2] = {0, 0}, q1[2], qm1[2] = {0, 0};
    R px[2] = {0, 0}, py[2] = {0, 0}, pxd[2] = {0, 0}, pyd[2] = {0, 0}, rmin[2], rmax[2];
    int i1 = NBSN(P, i, 1);
    int w1 = which == 0 ? 1 : P.iswetn[i1];
    for (int t = 0; t < 2; ++t) {
      qi[t] = (R)Q[t][i];
      q1[t] = (R)Q[t][i1];
      if (which != 0) {
        qmi[t] = (R)QM[t][i];
        qm1[t] = (R)QM[t][i1];
      }
      rmin[t] = q1[t];
      rmax[t] = q1[t];
    }
    for (int j = 1; j <= nt - 1; ++j) {
      const int i2 = NBSN(P, i, j + 1);
      const int w2 = which == 0 ? 1 : P.iswetn[i2];
      R ty, tx;
      if constexpr (sizeof(R) == 4) {
        const float2 tr = P.f.trie[(size_t)(j - 1) * (P.M + 1) + i];
        ty = tr.x;
        tx = tr.y;
      } else {
        ty = TRIEY(P, i, j);
        tx = TRIEX(P, i, j);
      }
      for (int t = 0; t < 2; ++t) {
        const R q2 = (R)Q[t][i2];
        if (j >= 2) {
          rmin[t] = fmin(rmin[t], q1[t]);
          rmax[t] = fmax(rmax[t], q1[t]);
        }
        R ffd, ff1;
        if (which == 0) {
          ffd = half * (q1[t] + q2 - qmean - qmean);
          ff1 = half * (q1[t] + q2);
        } else {
          const R qm2 = (R)QM[t][i2];
          R qa = q1[t], qb = q2, qma = qm1[t], qmb = qm2;
          if (w1 == 0 && w2 == 1) { qa = qi[t]; qma = qmi[t]; }
          else if (w1 == 1 && w2 == 0) { qb = qi[t]; qmb = qmi[t]; }
          else if (w1 == 0 && w2 == 0) { qa = qi[t]; qb = qi[t]; qma = qmi[t]; qmb = qmi[t]; }
          ffd = half * (qa + qb - qma - qmb);
          ff1 = half * (qa + qb);
          qm1[t] = qm2;
        }
        px[t] = px[t] + ff1 * ty;
        py[t] = py[t] + ff1 * tx;
        pxd[t] = pxd[t] + ffd * ty;
        pyd[t] = pyd[t] + ffd * tx;
        q1[t] = q2;
      }
      w1 = w2;
    }
    const size_t q = N3(P, i, k);
    // the node's mixing coefficient as the half-edge fluxes take it (FP32 records)
    R vf = 0;
    if (sizeof(R) == 4) {
      if (which == 0) {
        const size_t qm = N3(P, i, k - 1);
        vf = (R)((P.viscofh[q] * P.dz[qm] + P.viscofh[qm] * P.dz[q]) / (P.dz[q] + P.dz[qm]));
      } else {
        vf = (R)P.viscofh[q];
      }
    }
    for (int t = 0; t < 2; ++t) {
      const R gx = px[t] / art2, gy = py[t] / art2, gxd = pxd[t] / art2, gyd = pyd[t] / art2;
      NodeRec<R>::store(P, which, t, q, qi[t], gx, gy, gxd, gyd, rmin[t], rmax[t], vf);
      if (which == 1 && k == P.KBM1) {
        if (t == 0) { P.pfpxb_t[i] = (double)gx; P.pfpyb_t[i] = (double)gy; }
        else { P.pfpxb_s[i] = (double)gx; P.pfpyb_s[i] = (double)gy; }
        double ah = (P.fact * P.viscofh[N3(P, i, P.KBM1)] + P.fm1) * P.nn_hvc[i];
        if (t == 0) P.ah_bottom_t[i] = ah;
        else P.ah_bottom_s[i] = ah;
      }
    }
  }
}

// Vertical-neighbour bound of FCT on sigma layers (fct_t.F:78-97) and on interfaces
// (fct_q2.F:73-92).
__device__ inline void fct_layer_bounds(const Dev& P, int i, int k, const double* F, double& fmax_, double& fmin_) {
  const double* DZ = P.dz;
  size_t q = N3(P, i, k);
  if (k == 1) {
    size_t qp = N3(P, i, k + 1);
    double a = (F[q] * DZ[qp] + F[qp] * DZ[q]) / (DZ[q] + DZ[qp]);
    fmax_ = fmax(fmax_, a);
    fmin_ = fmin(fmin_, a);
  } else if (k == P.KBM1) {
    size_t qm = N3(P, i, k - 1);
    double a = (F[q] * DZ[qm] + F[qm] * DZ[q]) / (DZ[q] + DZ[qm]);
    fmax_ = fmax(fmax_, a);
    fmin_ = fmin(fmin_, a);
  } else {
    size_t qm = N3(P, i, k - 1), qp = N3(P, i, k + 1);
    double a = (F[q] * DZ[qm] + F[qm] * DZ[q]) / (DZ[q] + DZ[qm]);
    double b = (F[q] * DZ[qp] + F[qp] * DZ[q]) / (DZ[q] + DZ[qp]);
    fmax_ = fmax(fmax(fmax_, a), b);
    fmin_ = fmin(fmin(fmin_, a), b);
  }
}
__device__ inline void fct_level_bounds(const Dev& P, int i, int k, const double* F, double& fmax_, double& fmin_) {
  const double* DZZ = P.dzz;
  size_t q = N3(P, i, k), qm = N3(P, i, k - 1), qp = N3(P, i, k + 1);
  if (k == 2) {
    double a = (F[q] * DZZ[q] + F[qp] * DZZ[qm]) / (DZZ[q] + DZZ[qm]);
    fmax_ = fmax(fmax_, a);
    fmin_ = fmin(fmin_, a);
  } else if (k == P.KBM1) {
    size_t qmm = N3(P, i, k - 2);
    double a = (F[q] * DZZ[qmm] + F[qm] * DZZ[qm]) / (DZZ[qm] + DZZ[qmm]);
    fmax_ = fmax(fmax_, a);
    fmin_ = fmin(fmin_, a);
  } else {
    size_t qmm = N3(P, i, k - 2);
    double a = (F[q] * DZZ[qmm] + F[qm] * DZZ[qm]) / (DZZ[qm] + DZZ[qmm]);
    double b = (F[q] * DZZ[q] + F[qp] * DZZ[qm]) / (DZZ[q] + DZZ[qm]);
    fmax_ = fmax(fmax(fmax_, a), b);
    fmin_ = fmin(fmin(fmin_, a), b);
  }
}

// -------------------------------------------------------------------------------------
// Half-edge fluxes of ADV_Q (adv_q.F:250-342) and ADV_T/ADV_S (adv_t.F:411-556).
//
// Phase 1 (k_he_adv, one thread per cell and layer): a cell's three control-volume
// half-edges run from its centroid to its edge midpoints and each separates two of the
// cell's own nodes, so the node data (tracer value, ring gradients and extrema, mixing
// coefficient) is loaded once for the three half-edges.  Each half-edge flux EXFLUX is
// evaluated once, in the reference's expression order, and stored at the half-edge's
// position slot*ns + cell.
// Phase 2 (k_gather_*, one thread per node and layer) sums the node's half-edge fluxes
// with their signs in ascending half-edge order -- the order of the reference's scatter --
// and applies the vertical flux, the update and the FCT clamp.
// MODE 0: Q2 and Q2L on interfaces K=2..KBM1; MODE 1: T and S on layers K=1..KBM1.
// -------------------------------------------------------------------------------------
template <typename R>
struct HeCell {
  R uq, vq, dtij;
  int nd[3];
  R vf[3], nn[3];
};

// The layer-independent part of a cell's half-edge data: its three nodes and their
// NN_HVC, loaded once per thread for the layers it walks.
template <typename R>
__device__ inline void he_cell_static(const Dev& P, int c, HeCell<R>& hc) {
  const size_t n1 = P.N + 1;
  for (int j = 0; j < 3; ++j) {
    const int n = P.nv[j * n1 + c];
    hc.nd[j] = n;
    hc.nn[j] = (R)P.nn_hvc[n];
  }
}
// Cell data of the half-edge fluxes on layer k, formed in FP64 and rounded to R; with
// STATIC false, hc already holds he_cell_static's part.
template <typename R, int MODE, bool STATIC = true>
__device__ inline void he_cell_load(const Dev& P, int c, int k, HeCell<R>& hc) {
  size_t ck = C3(P, c, k);
  if (MODE == 0) {
    size_t ckm = C3(P, c, k - 1);
    hc.uq = (R)((P.u[ck] * P.dz1[ckm] + P.u[ckm] * P.dz1[ck]) / (P.dz1[ck] + P.dz1[ckm]));
    hc.vq = (R)((P.v[ck] * P.dz1[ckm] + P.v[ckm] * P.dz1[ck]) / (P.dz1[ck] + P.dz1[ckm]));
    hc.dtij = (R)(P.dt1[c] * P.dzz1[ckm]);
  } else {
    hc.uq = (R)P.u[ck];
    hc.vq = (R)P.v[ck];
    hc.dtij = (R)(P.dt1[c] * P.dz1[ck]);
  }
  if (STATIC) he_cell_static<R>(P, c, hc);
  for (int j = 0; j < 3; ++j) {
    if (sizeof(R) == 4) continue;  // FP32: VISCOFH travels in the node records
    const int n = hc.nd[j];
    size_t q = N3(P, n, k);
    if (MODE == 0) {
      size_t qm = N3(P, n, k - 1);
      hc.vf[j] = (R)((P.viscofh[q] * P.dz[qm] + P.viscofh[qm] * P.dz[q]) / (P.dz[q] + P.dz[qm]));
    } else {
      hc.vf[j] = (R)P.viscofh[q];
    }
  }
}

// v[j] for a run-time slot j in 0..2, by selects, so v stays in registers.
template <typename R>
__device__ inline R sel3(const R* v, int j) { return j == 0 ? v[0] : (j == 1 ? v[1] : v[2]); }
__device__ inline int sel3i(const int* v, int j) { return j == 0 ? v[0] : (j == 1 ? v[1] : v[2]); }

// Metrics of one half-edge (DLTXE, DLTYE and the DLTXNCVE/DLTYNCVE of both sides), read
// by position (coalesced over the threads of consecutive cells).
template <typename R>
struct HeGeo {
  R dx, dy, xa, ya, xb, yb;
};
template <typename R>
__device__ inline HeGeo<R> he_geo(const Dev& P, size_t pos) {
  typedef Mesh<R> Mh;
  if constexpr (sizeof(R) == 4) {
    const float4 a = P.f.hg4[pos];
    const float2 b = P.f.hg2[pos];
    return HeGeo<R>{a.x, a.y, a.z, a.w, b.x, b.y};
  } else {
    return HeGeo<R>{Mh::hg(P, 0, pos), Mh::hg(P, 1, pos), Mh::hg(P, 2, pos),
                    Mh::hg(P, 3, pos), Mh::hg(P, 4, pos), Mh::hg(P, 5, pos)};
  }
}

// EXFLUX of a half-edge with metrics g for tracer t, in R; a and b are the positions of
// NIEC(he,1) and NIEC(he,2) among the cell's nodes, ra and rb their data.  xadv receives
// EXFLUX-FXX-FYY.
template <typename R, int MODE>
__device__ inline R he_flux(const Dev& P, const HeCell<R>& hc, const HeGeo<R>& g, int a, int b, const TRec<R>& ra,
                            const TRec<R>& rb, R* xadv) {
  const R half = (R)0.5, one = (R)1.0;
  const R dltxe = g.dx, dltye = g.dy;
  R un = hc.vq * dltxe - hc.uq * dltye;
  R fij1 = ra.q + g.xa * ra.px + g.ya * ra.py;
  R fij2 = rb.q + g.xb * rb.px + g.yb * rb.py;
  R q1min = fmin(ra.rmin, ra.q), q1max = fmax(ra.rmax, ra.q);
  R q2min = fmin(rb.rmin, rb.q), q2max = fmax(rb.rmax, rb.q);
  if (fij1 < q1min) fij1 = q1min;
  if (fij1 > q1max) fij1 = q1max;
  if (fij2 < q2min) fij2 = q2min;
  if (fij2 > q2max) fij2 = q2max;
  const R vfa = sizeof(R) == 4 ? ra.vf : sel3(hc.vf, a), vfb = sizeof(R) == 4 ? rb.vf : sel3(hc.vf, b);
  const R nna = sel3(hc.nn, a), nnb = sel3(hc.nn, b);
  R viscof = (R)P.fact * half * (vfa * nna + vfb * nnb) + (R)P.fm1 * half * (nna + nnb);
  if (MODE == 0) viscof = viscof / (R)P.hprnu;
  R txx = half * (ra.pxd + rb.pxd) * viscof;
  R tyy = half * (ra.pyd + rb.pyd) * viscof;
  R fxx = -hc.dtij * txx * dltye;
  R fyy = hc.dtij * tyy * dltxe;
  R sg = fsign1(un);
  R exflux = -un * hc.dtij * ((one + sg) * fij2 + (one - sg) * fij1) * half + fxx + fyy;
  if (xadv) *xadv = exflux - fxx - fyy;
  return exflux;
}

template <typename R>
__device__ inline TRec<R> sel_trec(const TRec<R>& a, const TRec<R>& b, const TRec<R>& c, int j) {
  TRec<R> r;
  r.q = j == 0 ? a.q : (j == 1 ? b.q : c.q);
  r.px = j == 0 ? a.px : (j == 1 ? b.px : c.px);
  r.py = j == 0 ? a.py : (j == 1 ? b.py : c.py);
  r.pxd = j == 0 ? a.pxd : (j == 1 ? b.pxd : c.pxd);
  r.pyd = j == 0 ? a.pyd : (j == 1 ? b.pyd : c.pyd);
  r.rmin = j == 0 ? a.rmin : (j == 1 ? b.rmin : c.rmin);
  r.rmax = j == 0 ? a.rmax : (j == 1 ? b.rmax : c.rmax);
  r.vf = j == 0 ? a.vf : (j == 1 ? b.vf : c.vf);
  return r;
}

template <typename R>
__device__ inline int pos3(const HeCell<R>& hc, int n) { return n == hc.nd[0] ? 0 : (n == hc.nd[1] ? 1 : 2); }

template <typename R, int MODE>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 3 : 2) k_he_adv(const Dev P, int parts) {
  typedef typename Mesh<R>::R2 R2;
  int c = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (c > P.N) return;
  int kb, ke;
  col_range(P, MODE == 0 ? 2 : 1, P.KBM1, kb, ke);
  const size_t v1 = P.NCV + 1;
  const bool do0 = parts & (MODE == 0 ? AD_Q2 : AD_T), do1 = parts & (MODE == 0 ? AD_Q2L : AD_S);
  int pa[3], pb[3];
  {
    int nd0 = P.nv[c], nd1 = P.nv[(size_t)(P.N + 1) + c];
    for (int s = 0; s < 3; ++s) {
      int he = P.cell_he[3 * c + s];
      int na = P.niec[he], nb = P.niec[v1 + he];
      pa[s] = na == nd0 ? 0 : (na == nd1 ? 1 : 2);
      pb[s] = nb == nd0 ? 0 : (nb == nd1 ? 1 : 2);
    }
  }
  // Each of the cell's three nodes ends two of its half-edges: its record is loaded once
  // per tracer and layer and handed to both.  The metrics and the fluxes are by position
  // s*ns + c.  For Q2/Q2L the cell's nodes are loaded once for the layers this thread
  // walks (for T/S, which hold more live values, that spills: they are reloaded per layer).
  HeCell<R> hc;
  if (MODE == 0) he_cell_static<R>(P, c, hc);
  for (int k = kb; k <= ke; ++k) {
    he_cell_load<R, MODE, MODE != 0>(P, c, k, hc);
    R2* EX = Mesh<R>::ex2(P) + (size_t)(k - 1) * P.ncvs + c;
    R e[2][3] = {{0, 0, 0}, {0, 0, 0}};
    for (int t = 0; t < 2; ++t) {
      if (!(t == 0 ? do0 : do1)) continue;
      const TRec<R> r0 = load_trec<R, MODE>(P, hc.nd[0], k, t);
      const TRec<R> r1 = load_trec<R, MODE>(P, hc.nd[1], k, t);
      const TRec<R> r2 = load_trec<R, MODE>(P, hc.nd[2], k, t);
      for (int s = 0; s < 3; ++s)
        e[t][s] = he_flux<R, MODE>(P, hc, he_geo<R>(P, (size_t)s * P.ns + c), pa[s], pb[s],
                                   sel_trec(r0, r1, r2, pa[s]), sel_trec(r0, r1, r2, pb[s]), nullptr);
    }
    for (int s = 0; s < 3; ++s) EX[(size_t)s * P.ns] = mk2(e[0][s], e[1][s]);
  }
}

// XFLUX_ADV of one open-boundary node (adv_t.F:510-511, 572-579): the advective parts of
// its half-edge fluxes, recomputed with the same arithmetic as phase 1.
template <typename R>
__device__ inline double obc_xflux_adv(const Dev& P, int i, int k, int t) {
  const size_t v1 = P.NCV + 1;
  R xa = 0;
  for (int q = P.node_he_ptr[i]; q < P.node_he_ptr[i + 1]; ++q) {
    int code = P.node_he[q];
    int he = code >> 1;
    int c = P.ntrg[he];
    const int sl = P.cell_he[3 * c] == he ? 0 : (P.cell_he[3 * c + 1] == he ? 1 : 2);
    HeCell<R> hc;
    he_cell_load<R, 1>(P, c, k, hc);
    const int na = P.niec[he], nb = P.niec[v1 + he];
    R part;
    he_flux<R, 1>(P, hc, he_geo<R>(P, (size_t)sl * P.ns + c), pos3(hc, na), pos3(hc, nb),
                  load_trec<R, 1>(P, na, k, t), load_trec<R, 1>(P, nb, k, t), &part);
    xa = (code & 1) ? xa - part : xa + part;
  }
  return (double)xa;
}

// Signed sum of a node's half-edge fluxes on layer k, both tracers, in ascending
// half-edge order (the order of the reference's scatter into XFLUX).
// The loads are issued four entries at a time (codes, then fluxes) and added in order.
template <typename R>
__device__ inline double2 gather_he(const Dev& P, int i, int n, int k) {
  typedef typename Mesh<R>::R2 R2;
  const R2* EX = Mesh<R>::ex2(P) + (size_t)(k - 1) * P.ncvs;
  const int* L = P.node_vpos_ell + i;
  const size_t ms = P.ms;
  R x0 = 0, x1 = 0;
  auto add = [&](int code, R2 e) {
    if (code & 1) {
      x0 = x0 - e.x;
      x1 = x1 - e.y;
    } else {
      x0 = x0 + e.x;
      x1 = x1 + e.y;
    }
  };
  int j = 0;
  for (; j + 4 <= n; j += 4) {
    const int c0 = L[j * ms], c1 = L[(j + 1) * ms], c2 = L[(j + 2) * ms], c3 = L[(j + 3) * ms];
    const R2 e0 = EX[c0 >> 1], e1 = EX[c1 >> 1], e2 = EX[c2 >> 1], e3 = EX[c3 >> 1];
    add(c0, e0);
    add(c1, e1);
    add(c2, e2);
    add(c3, e3);
  }
  for (; j < n; ++j) {
    const int c = L[j * ms];
    add(c, EX[c >> 1]);
  }
  return make_double2((double)x0, (double)x1);
}

// Phase 2 of ADV_Q(Q2,Q2F)/ADV_Q(Q2L,Q2LF) (adv_q.F:114-401) with FCT_Q2/FCT_Q2L.
template <typename R>
__global__ void __launch_bounds__(256) k_gather_q(const Dev P, int parts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  int kb, ke;
  col_range(P, 2, P.KBM1, kb, ke);
  const bool wet = P.iswetn[i] * P.iswetnt[i] == 1;
  const int nhe = P.node_he_ptr[i + 1] - P.node_he_ptr[i];
  for (int k = kb; k <= ke; ++k) {
  const double2 xs = gather_he<R>(P, i, nhe, k);
  for (int t = 0; t < 2; ++t) {
    if (!(parts & (t == 0 ? AD_Q2 : AD_Q2L))) continue;
    const double* Q = (t == 0 ? P.q2 : P.q2l);
    double* QF = (t == 0 ? P.q2f : P.q2lf);
    if (k == 2) {
      // QF = 0 on every level before the interior levels are set (adv_q.F:114)
      QF[N3(P, i, 1)] = 0.0;
      QF[N3(P, i, P.KB)] = 0.0;
    }
    double x = t == 0 ? xs.x : xs.y;
    size_t q = N3(P, i, k);
    double qf;
    if (wet) {
      size_t qm = N3(P, i, k - 1), qp = N3(P, i, k + 1);
      double temp = P.wts[qm] * Q[qm] - P.wts[qp] * Q[qp];
      x = x + temp * P.art1[i] * P.dzz[qm] / (P.dz[qm] + P.dz[q]);
      qf = (Q[q] - x / P.art1[i] * (P.dti / (P.dt[i] * P.dzz[qm]))) * (P.dt[i] / P.d[i]);
    } else {
      qf = Q[q];
    }
    if ((parts & AD_FCT) && !P.riv_skip[i]) {
      double qmin, qmax;
      NodeRec<R>::minmax(P, 0, t, q, qmin, qmax);
      fct_level_bounds(P, i, k, Q, qmax, qmin);
      if (qmin - qf > 0.0) qf = qmin;
      if (qf - qmax > 0.0) qf = qmax;
    }
    QF[q] = qf;
  }
  }
}

// FCT_Q2 / FCT_Q2L alone (fct_q2.F:51-99) on QF already in memory.
__global__ void __launch_bounds__(256) k_fct_q(const Dev P, int parts) {
  int i = blockIdx.x * 32 + threadIdx.x + 1;
  int k = blockIdx.y * 8 + threadIdx.y + 2;
  if (i > P.M || k > P.KBM1 || P.riv_skip[i]) return;
  for (int t = 0; t < 2; ++t) {
    if (!(parts & (t == 0 ? AD_Q2 : AD_Q2L))) continue;
    const double* Q = (t == 0 ? P.q2 : P.q2l);
    double* QF = (t == 0 ? P.q2f : P.q2lf);
    size_t q = N3(P, i, k);
    double qmax = Q[N3(P, NBSN(P, i, 1), k)], qmin = qmax;
    for (int j = 2; j <= P.ntsn[i]; ++j) {
      double v = Q[N3(P, NBSN(P, i, j), k)];
      qmax = fmax(qmax, v);
      qmin = fmin(qmin, v);
    }
    fct_level_bounds(P, i, k, Q, qmax, qmin);
    double qf = QF[q];
    if (qmin - qf > 0.0) qf = qmin;
    if (qf - qmax > 0.0) qf = qmax;
    QF[q] = qf;
  }
}

// -------------------------------------------------------------------------------------
// VDIF_Q, MY2.5 (vdif_q.F:119-513), one thread per node column.  With copy_back the
// end-of-closure shift Q2=Q2F, Q2L=Q2LF (internal_step.F:1034-1035) follows.
// -------------------------------------------------------------------------------------
// VDIF_Q in three passes.  The reference's column loop (one node at a time) has only two
// truly sequential parts, the tridiagonal sweeps of the q2 and q2l equations; everything
// else is per level.  k_vdif_q_levels forms, per (node, level), every input of the sweeps
// (the positivity fixes, BOYGR, the shear production PROD, the length scale L and its
// limits, GH, DTEF and the q2l wall-function DTEF); k_vdif_q_sweep runs the two sweeps per
// column; k_vdif_q_coef applies the stability functions per (node, level).  Each value is
// computed with the reference's expression, so the result is bitwise that of the column
// loop.
namespace vq {
constexpr double A1 = 0.92, B1 = 16.6, A2 = 0.74, B2 = 10.1, C1 = 0.08;
constexpr double E1 = 1.80, E2 = 1.33, SEF = 1.00, KAPPA = 0.40;
constexpr double SMALL = 1.e-8, GH_MAX = .0233, GH_MIN = -.281;
constexpr double SURFL = 2.e+5, GHC = -6.0;
}  // namespace vq

// Surface stress magnitude UTAU2 and bottom stress magnitude of node i (vdif_q.F:172-246),
// the NBVE means in ring order.
__device__ inline void vq_stress(const Dev& P, int i, double& utau2, double& wub, double& wvb) {
  const size_t m1 = P.M + 1;
  const int nt = P.ntve[i];
  double wus = 0.0, wvs = 0.0;
  wub = 0.0;
  wvb = 0.0;
  for (int j = 1; j <= nt; ++j) {
    int c = P.nbve[(size_t)(j - 1) * m1 + i];
    wus = wus + P.wusurf[c];
    wvs = wvs + P.wvsurf[c];
  }
  const double fn = (double)(float)nt;
  wus = wus / fn;
  wvs = wvs / fn;
  utau2 = sqrt(wus * wus + wvs * wvs);
  for (int j = 1; j <= nt; ++j) {
    int c = P.nbve[(size_t)(j - 1) * m1 + i];
    wub = wub + P.wubot[c];
    wvb = wvb + P.wvbot[c];
  }
  wub = wub / fn;
  wvb = wvb / fn;
}

// AUX bit 1: the learned closure's inputs are written (P.closure); bit 2: the closure
// samples (P.clos_samp).  Each combination is its own instantiation, so that the plain
// step carries none of the other paths' registers.  Every instantiation is held to 64
// registers (four blocks per SM): with the closure's inputs that spills 20 bytes, and
// still measured faster than 80 registers and three blocks (1.30 against 1.37 ms per
// step for VDIF_Q on the 200k-node mesh).
template <int AUX>
__global__ void __launch_bounds__(256, 4) k_vdif_q_levels(const Dev P) {
  using namespace vq;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  int kb, ke;
  col_range(P, 1, P.KB, kb, ke);
  const int KB = P.KB, KBM1 = P.KBM1;
  const double d = P.d[i];
  const bool wet = P.iswetn[i] == 1;
  double* Q2 = P.q2;
  double* Q2L = P.q2l;
  double* L = P.l;
  auto n3 = [&](int k) { return N3(P, i, k); };
  double utau2, wub, wvb;
  vq_stress(P, i, utau2, wub, wvb);
  const double l0 = SURFL * utau2 / P.grav_n[i];
  if (kb == 1) P.vq_ut[i] = utau2;
  if (ke == KB) P.q2f[n3(KB)] = sqrt(wub * wub + wvb * wvb) * P.const1;
  float* const cs = (AUX & 2) ? P.clos_samp : nullptr;
  const size_t ss = (size_t)P.M * (size_t)(KBM1 - 1);
  auto samp = [&](int f, int k, double v) { cs[(size_t)f * ss + (size_t)(k - 2) * P.M + (i - 1)] = (float)v; };
  // ring means of U, V on the level above the first interior level of the chunk
  const size_t m1 = P.M + 1;
  const int nt = P.ntve[i];
  const double fn = (double)(float)nt;
  auto ring_mean = [&](int k, double& um, double& vm) {
    double su = 0.0, sv = 0.0;
    for (int j = 1; j <= nt; ++j) {
      int c = P.nbve[(size_t)(j - 1) * m1 + i];
      su = su + P.u[C3(P, c, k)];
      sv = sv + P.v[C3(P, c, k)];
    }
    um = su / fn;
    vm = sv / fn;
  };
  double ukm1 = 0.0, vkm1 = 0.0;
  if (wet && kb <= KBM1) ring_mean(kb >= 2 ? kb - 1 : 1, ukm1, vkm1);
  bool chunk_inside = wet;  // every interior level of this chunk inside the closure's envelope
  for (int k = kb; k <= ke; ++k) {
    const size_t q = n3(k);
    // positivity of the previous Q2F/Q2LF (vdif_q.F:144-149)
    if (k >= 2 && k <= KBM1 && (P.q2f[q] <= SMALL || P.q2lf[q] <= SMALL)) {
      P.q2f[q] = SMALL;
      P.q2lf[q] = SMALL;
    }
    const double q2 = fabs(Q2[q] + SMALL);
    double q2l = fabs(Q2L[q]);
    Q2[q] = q2;
    double boygr = 0.0, prod = 0.0, lk;
    if (k >= 2 && k <= KBM1) {
      if (wet) {
        boygr = P.grav_n[i] * (P.rho1[n3(k - 1)] - P.rho1[q]) / (P.dzz[n3(k - 1)] * d);
        prod = P.km[q] * 0.0 * pow(.5 * (-boygr + fabs(boygr)), 1.5);
        double uk, vk;
        ring_mean(k, uk, vk);
        const double den = P.dzz[n3(k - 1)] * d;
        const double shear2 = ((uk - ukm1) * (uk - ukm1) + (vk - vkm1) * (vk - vkm1)) / (den * den);
        if (AUX & 1) {
          // the network's inputs: inside the envelope or not, then transformed,
          // standardised and rounded to BF16 as the MMA takes them
          const float fv[CLOS_IN] = {(float)boygr, (float)shear2, (float)d, (float)P.z[q], (float)sqrt(utau2),
                                     (float)sqrt(sqrt(wub * wub + wvb * wvb)), (float)q2, (float)q2l};
          uint32_t packed[4];
          for (int f = 0; f < CLOS_IN; ++f) {
            if (!(fv[f] >= P.clos_norm.lo[f] && fv[f] <= P.clos_norm.hi[f])) chunk_inside = false;
          }
          for (int f = 0; f < CLOS_IN; f += 2) {
            const __nv_bfloat162 b = __floats2bfloat162_rn(clos_feat_transform(P.clos_norm, f, fv[f]),
                                                           clos_feat_transform(P.clos_norm, f + 1, fv[f + 1]));
            packed[f / 2] = *reinterpret_cast<const uint32_t*>(&b);
          }
          P.clos_feat[(size_t)(k - 2) * P.M + (i - 1)] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        }
        if (AUX & 2) {
          samp(0, k, boygr);
          samp(1, k, shear2);
          samp(2, k, d);
          samp(3, k, P.z[q]);
          samp(4, k, sqrt(utau2));
          samp(5, k, sqrt(sqrt(wub * wub + wvb * wvb)));
          samp(6, k, q2);
          samp(7, k, q2l);
        }
        prod = prod + P.km[q] * SEF * ((uk - ukm1) * (uk - ukm1) + (vk - vkm1) * (vk - vkm1)) / (den * den);
        prod = prod + P.kh[q] * boygr;
        ukm1 = uk;
        vkm1 = vk;
      }
      // length scale and its limits (vdif_q.F:300-331)
      lk = q2l / q2;
      if (P.z[q] > -0.5) lk = fmax(lk, KAPPA * l0);
      if (boygr < 0.0) {
        double lmax = sqrt(fabs(GH_MIN) * q2 / (-boygr + SMALL));
        lk = fmin(lk, lmax);
        q2l = q2 * lk;
      }
    } else {
      lk = k == 1 ? KAPPA * l0 : 0.0;
    }
    Q2L[q] = q2l;
    L[q] = lk;
    double gh = 0.0;
    if (k >= 2 && k <= KBM1) gh = fmin((lk * lk / q2) * boygr, GH_MAX);
    double stf = 1.0;
    if (gh < 0.0) stf = 1.0 - F4(0.9) * pow(gh / GHC, 1.5);
    if (gh < GHC) stf = F4(0.1);
    const double dtef = sqrt(q2) / (B1 * lk + SMALL) * stf;
    P.vq_prod[q] = prod;
    P.vq_gh[q] = gh;
    P.vq_dtef[q] = dtef;
    if (wet && k >= 2 && k <= KBM1) {
      const double x = (1. / fabs(P.z[q] - P.z[n3(1)]) + 1. / fabs(P.z[q] - P.z[n3(KB)])) * lk / (d * KAPPA);
      P.vq_dtefl[q] = dtef * (1. + E2 * (x * x));
    }
  }
  if (AUX & 1) P.clos_envc[(size_t)blockIdx.y * (P.M + 1) + i] = chunk_inside ? 1 : 0;
}

// The q2 and q2l tridiagonal sweeps of one column (vdif_q.F:372-431), and the column's
// envelope flag of the learned closure.  The two sweeps are independent: blockIdx.y = 0
// runs the q2 sweep, 1 the q2l sweep.  The forward elimination loads the coefficients of
// four levels before it runs their (serial) recurrence.
__global__ void __launch_bounds__(128) k_vdif_q_sweep(const Dev P) {
  using namespace vq;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  const int KB = P.KB, KBM1 = P.KBM1;
  const double DTI = P.dti;
  const double d = P.d[i];
  const bool wet = P.iswetn[i] == 1;
  const bool q2l = blockIdx.y == 1;
  auto n3 = [&](int k) { return N3(P, i, k); };
  if (P.closure && !q2l) {
    // the column's envelope flag from the level kernel's per-chunk flags
    bool in_env = wet;
    const int nch = (P.KB + P.col_lc - 1) / P.col_lc;
    for (int c = 0; c < nch && in_env; ++c) in_env = P.clos_envc[(size_t)c * (P.M + 1) + i] != 0;
    P.clos_env[i] = in_env ? 1 : 0;
  }
  if (!wet) return;
  double vh[kMaxKBs], vhp[kMaxKBs];
  vh[1] = 0.0;
  vhp[1] = q2l ? 0.0 : P.vhp1c * P.vq_ut[i];
  double* QF = q2l ? P.q2lf : P.q2f;
  // the coefficients of level k: A, C, the diagonal term and the source of the equation
  auto coef = [&](int k, double& a, double& c, double& e, double& r, double& qf) {
    a = -0.5 * DTI * (P.kq[n3(k + 1)] + P.kq[n3(k)] + 2.0 * P.umol) / (P.dzz[n3(k - 1)] * P.dz[n3(k)] * d * d);
    c = -0.5 * DTI * (P.kq[n3(k - 1)] + P.kq[n3(k)] + 2.0 * P.umol) / (P.dzz[n3(k - 1)] * P.dz[n3(k - 1)] * d * d);
    if (q2l) {
      e = DTI * P.vq_dtefl[n3(k)] + 1.;
      r = DTI * (-P.vq_prod[n3(k)] * P.l[n3(k)] * E1);
    } else {
      e = 2. * DTI * P.vq_dtef[n3(k)] + 1.;
      r = -2. * DTI * P.vq_prod[n3(k)];
    }
    qf = QF[n3(k)];
  };
  auto step = [&](int k, double a, double c, double e, double r, double qf) {
    const double p = 1. / (a + c * (1. - vh[k - 1]) - e);
    vh[k] = a * p;
    vhp[k] = (r + c * vhp[k - 1] - qf) * p;
  };
  int k = 2;
  for (; k + 3 <= KBM1; k += 4) {
    double a[4], c[4], e[4], r[4], qf[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) coef(k + u, a[u], c[u], e[u], r[u], qf[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) step(k + u, a[u], c[u], e[u], r[u], qf[u]);
  }
  for (; k <= KBM1; ++k) {
    double a, c, e, r, qf;
    coef(k, a, c, e, r, qf);
    step(k, a, c, e, r, qf);
  }
  for (int k = 1; k <= KBM1; ++k) {
    int ki = KB - k;
    QF[n3(ki)] = vh[ki] * QF[n3(ki + 1)] + vhp[ki];
  }
}

// Positivity of the new Q2F/Q2LF, the stability functions and KQ, KM, KH
// (vdif_q.F:443-491), per (node, level); then Q2 = Q2F, Q2L = Q2LF.  AUX as for
// k_vdif_q_levels; with the learned closure the interior levels of a column on the network
// skip the stability functions, which k_closure_mlp replaces.
template <int AUX>
__global__ void __launch_bounds__(256) k_vdif_q_coef(const Dev P, int copy_back) {
  using namespace vq;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  int kb, ke;
  col_range(P, 1, P.KB, kb, ke);
  const int KBM1 = P.KBM1;
  const double COEF4 = 18.0 * A1 * A1 + 9.0 * A1 * A2;
  const double COEF5 = 9.0 * A1 * A2;
  const bool wet = P.iswetn[i] == 1;
  float* const cs = (AUX & 2) ? P.clos_samp : nullptr;
  const size_t ss = (size_t)P.M * (size_t)(KBM1 - 1);
  auto samp = [&](int f, int k, double v) { cs[(size_t)f * ss + (size_t)(k - 2) * P.M + (i - 1)] = (float)v; };
  // interior levels of a column inside the envelope are finished by the network kernel
  // (k_closure_mlp); every other column keeps MY2.5 here
  const bool on_network = (AUX & 1) && P.clos_env[i] != 0;
  for (int k = kb; k <= ke; ++k) {
    const size_t q = N3(P, i, k);
    if (k >= 2 && k <= KBM1 && (P.q2f[q] <= SMALL || P.q2lf[q] <= SMALL)) {
      P.q2f[q] = SMALL;
      P.q2lf[q] = SMALL;
    }
    if (!(AUX & 2) && on_network && k >= 2 && k <= KBM1) {
      if (copy_back) {
        P.q2[q] = P.q2f[q];
        P.q2l[q] = P.q2lf[q];
      }
      continue;
    }
    const double gh = P.vq_gh[q];
    double stf = 1.0;
    if (gh < 0.0) stf = 1.0 - F4(0.9) * pow(gh / GHC, 1.5);
    if (gh < GHC) stf = F4(0.1);
    double coef1 = A2 * (1.0 - 6.0 * A1 / B1 * stf);
    double coef2 = 3.0 * A2 * B2 / stf + 18.0 * A1 * A2;
    double coef3 = A1 * (1.0 - 3.0 * C1 - 6.0 * A1 / B1 * stf);
    double sh = coef1 / (1.0 - coef2 * gh);
    double sm = (coef3 + sh * COEF4 * gh) / (1. - COEF5 * gh);
    double kn = P.l[q] * sqrt(P.q2[q]);
    bool interior_by_network = false;
    if (k >= 2 && k <= KBM1) {
      if (AUX & 2) {
        samp(8, k, kn * KAPPA * sm);
        samp(9, k, kn * sm);
        samp(10, k, kn * sh * P.vprnu);
        samp(11, k, wet ? 1.0 : 0.0);
      }
      interior_by_network = on_network;
    }
    if (!interior_by_network) {
      P.kq[q] = 0.5 * (kn * KAPPA * sm + P.kq[q]);
      P.km[q] = 0.5 * (kn * sm + P.km[q]);
      P.kh[q] = 0.5 * (kn * sh * P.vprnu + P.kh[q]);
    }
    if (copy_back) {
      P.q2[q] = P.q2f[q];
      P.q2l[q] = P.q2lf[q];
    }
  }
}

// Q2=Q2F, Q2L=Q2LF on every node and level; N2E3D(KM,KM1) (internal_step.F:1034-1053).
__global__ void __launch_bounds__(256) k_turb_update(const Dev P) {
  int i = blockIdx.x * 32 + threadIdx.x;
  int k = blockIdx.y * 8 + threadIdx.y + 1;
  if (k > P.KB) return;
  if (i <= P.M) {
    size_t q = N3(P, i, k);
    P.q2[q] = P.q2f[q];
    P.q2l[q] = P.q2lf[q];
  }
  if (i >= 1 && i <= P.N) {
    const size_t n1 = P.N + 1;
    P.km1[C3(P, i, k)] = ONE_THIRD * (P.km[N3(P, P.nv[i], k)] + P.km[N3(P, P.nv[n1 + i], k)] + P.km[N3(P, P.nv[2 * n1 + i], k)]);
  }
}

// -------------------------------------------------------------------------------------
// Phase 2 of ADV_T / ADV_S (adv_t.F:124-1042, adv_s.F) with FCT_T / FCT_S (fct_t.F:51-104,
// fct_s.F:50-108) on the same (node, layer) thread.
// -------------------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_gather_ts(const Dev P, int parts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M) return;
  int kb, ke;
  col_range(P, 1, P.KBM1, kb, ke);
  const bool wet = P.iswetn[i] * P.iswetnt[i] == 1;
  const int ob = P.node_obc[i];
  const int nhe = P.node_he_ptr[i + 1] - P.node_he_ptr[i];
  for (int k = kb; k <= ke; ++k) {
  const double2 xs = gather_he<R>(P, i, nhe, k);
  for (int t = 0; t < 2; ++t) {
    if (!(parts & (t == 0 ? AD_T : AD_S))) continue;
    const double* F1 = (t == 0 ? P.t1 : P.s1);
    double* FF1 = (t == 0 ? P.tf1 : P.sf1);
    double x = t == 0 ? xs.x : xs.y;
    if (ob > 0) (t == 0 ? P.xflux_obc_t : P.xflux_obc_s)[(size_t)(k - 1) * (P.iobcn + 1) + ob] = obc_xflux_adv<R>(P, i, k, t);
    size_t q = N3(P, i, k);
    double ff;
    if (wet) {
      const double* DZ = P.dz;
      double temp;
      if (k == 1) {
        size_t qp = N3(P, i, k + 1);
        temp = -P.wts[qp] * (F1[q] * DZ[qp] + F1[qp] * DZ[q]) / (DZ[q] + DZ[qp]);
      } else if (k == P.KBM1) {
        size_t qm = N3(P, i, k - 1);
        temp = P.wts[q] * (F1[q] * DZ[qm] + F1[qm] * DZ[q]) / (DZ[q] + DZ[qm]);
      } else {
        size_t qm = N3(P, i, k - 1), qp = N3(P, i, k + 1);
        temp = P.wts[q] * (F1[q] * DZ[qm] + F1[qm] * DZ[q]) / (DZ[q] + DZ[qm]) -
               P.wts[qp] * (F1[q] * DZ[qp] + F1[qp] * DZ[q]) / (DZ[q] + DZ[qp]);
      }
      if (P.isonb[i] == 2)
        x = temp * P.art1[i];
      else
        x = x + temp * P.art1[i];
      ff = (F1[q] - x / P.art1[i] * (P.dti / (P.dt[i] * DZ[q]))) * (P.dt[i] / P.dtfa[i]);
    } else {
      ff = F1[q];
    }
    if (parts & AD_FCT) {
      if (!P.riv_skip[i]) {
        double fmn, fmx;
        NodeRec<R>::minmax(P, 1, t, q, fmn, fmx);
        fct_layer_bounds(P, i, k, F1, fmx, fmn);
        if (fmn - ff > 0.0) ff = fmn;
        if (ff - fmx > 0.0) ff = fmx;
      }
      if (t == 1 && ff < 0.0) ff = 0.0;
    }
    FF1[q] = ff;
  }
  }
}

// FCT_T / FCT_S alone (fct_t.F:51-104, fct_s.F:50-108) on TF1/SF1 in memory.
__global__ void __launch_bounds__(256) k_fct_ts(const Dev P, int parts) {
  int i = blockIdx.x * 32 + threadIdx.x + 1;
  int k = blockIdx.y * 8 + threadIdx.y + 1;
  if (i > P.M || k > P.KBM1) return;
  for (int t = 0; t < 2; ++t) {
    if (!(parts & (t == 0 ? AD_T : AD_S))) continue;
    const double* F1 = (t == 0 ? P.t1 : P.s1);
    double* FF1 = (t == 0 ? P.tf1 : P.sf1);
    size_t q = N3(P, i, k);
    double ff = FF1[q];
    if (!P.riv_skip[i]) {
      double fmx = F1[N3(P, NBSN(P, i, 1), k)], fmn = fmx;
      for (int j = 2; j <= P.ntsn[i]; ++j) {
        double v = F1[N3(P, NBSN(P, i, j), k)];
        fmx = fmax(fmx, v);
        fmn = fmin(fmn, v);
      }
      fct_layer_bounds(P, i, k, F1, fmx, fmn);
      if (fmn - ff > 0.0) ff = fmn;
      if (ff - fmx > 0.0) ff = fmx;
    }
    if (t == 1 && ff < 0.0) ff = 0.0;
    FF1[q] = ff;
  }
}

// -------------------------------------------------------------------------------------
// VDIF_TS(1,TF1) and VDIF_TS(2,SF1) (vdif_ts.F:78-337), one thread per node column and
// tracer (blockIdx.y 0: T, 1: S).
// With surface heating (HEATING_TYPE 'flux', vdif_ts.F:118-150) the temperature column
// takes the net heat flux WTSURF, held at zero while cooling water at or below -2 C,
// and the short-wave flux RAD(K) = SWRAD*(RHEAT*EXP(Z*D/ZETA1) + (1-RHEAT)*EXP(Z*D/ZETA2))
// absorbed between levels; WTSURF and SWRAD are the forcing in W/m^2 times RAMP over
// -SPCP*ROSEA (BCOND_GCN(8), bcond_gcn.F:683-694).  Without heating every term is zero
// and the kernel is instantiated without them (HEAT = false).
// -------------------------------------------------------------------------------------
template <bool HEAT>
__global__ void __launch_bounds__(128) k_vdif_ts(const Dev P, int parts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > P.M || P.iswetn[i] != 1) return;
  const int KB = P.KB, KBM1 = P.KBM1, KBM2 = P.KBM2;
  const double DTI = P.dti, UMOLPR = P.umol * 1.e0, GW = 0.0;
  const double d = P.d[i];
  auto n3 = [&](int k) { return N3(P, i, k); };
  auto AF = [&](int k) { double fkh = P.kh[n3(k + 1)]; return -DTI * (fkh + UMOLPR) / (P.dz[n3(k)] * P.dzz[n3(k)] * d * d); };
  auto CF = [&](int k) { double fkh = P.kh[n3(k)]; return -DTI * (fkh + UMOLPR) / (P.dz[n3(k)] * P.dzz[n3(k - 1)] * d * d); };
  const double khbottom = P.kh[n3(KBM1)];
  const bool update = P.iswetn[i] * P.iswetnt[i] == 1;
  {
    const int t = blockIdx.y;  // 0: temperature, 1: salinity (independent columns)
    if (!(parts & (t == 0 ? AD_T : AD_S))) return;
    double* F = (t == 0 ? P.tf1 : P.sf1);
    double vhf[kMaxKBs], vhpf[kMaxKBs];
    const double sasurf = 0.0;
    double wfsurf = 0.0, swradf = 0.0;
    const bool heat = HEAT && t == 0;
    if (heat) {
      const double spro = 4.2174E3 * 1.023E3;
      const double ramp = ramp_int(P);
      wfsurf = -(P.wtsurf_w[i] * ramp) / spro;
      swradf = -(P.swrad_w[i] * ramp) / spro;
      const double wftmp1 = -2.0, wftmp2 = wfsurf;
      const double wftmp3 = 0.5 * (1.0 + fsign1(wftmp1 - F[n3(1)]));
      wfsurf = wftmp2 - wftmp3 * 0.5 * (wftmp2 + fabs(wftmp2));
    }
    // RAD at level k; zero without heating
    auto RAD = [&](int k) {
      if (!heat) return 0.0;
      const double zdep = P.z[n3(k)] * d;
      return swradf * (P.rheat * exp(zdep / P.zeta1) + (1 - P.rheat) * exp(zdep / P.zeta2));
    };
    double rad_k = RAD(1), rad_k1 = RAD(2);
    double af1 = AF(1);
    vhf[1] = af1 / (af1 - 1.);
    vhpf[1] = -DTI * (sasurf + wfsurf - swradf + rad_k - rad_k1) / (-P.dz[n3(1)] * d) - F[n3(1)];
    vhpf[1] = vhpf[1] / (af1 - 1.);
    // level k's coefficients and source, then its step of the (serial) recurrence; the
    // loads of four levels are issued before their steps
    auto coef = [&](int k, double& af, double& cf, double& fk, double& r) {
      rad_k = rad_k1;
      rad_k1 = RAD(k + 1);
      af = AF(k);
      cf = CF(k);
      fk = F[n3(k)];
      r = DTI * (rad_k - rad_k1) / (d * P.dz[n3(k)]);
    };
    auto step = [&](int k, double af, double cf, double fk, double r) {
      double p = 1. / (af + cf * (1. - vhf[k - 1]) - 1.);
      vhf[k] = af * p;
      vhpf[k] = (cf * vhpf[k - 1] - fk + r) * p;
    };
    int k = 2;
    for (; k + 3 <= KBM2; k += 4) {
      double af[4], cf[4], fk[4], r[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) coef(k + u, af[u], cf[u], fk[u], r[u]);
#pragma unroll
      for (int u = 0; u < 4; ++u) step(k + u, af[u], cf[u], fk[u], r[u]);
    }
    for (; k <= KBM2; ++k) {
      double af, cf, fk, r;
      coef(k, af, cf, fk, r);
      step(k, af, cf, fk, r);
    }
    if (P.isonb[i] != 2 && update) {
      double pfx = t == 0 ? P.pfpxb_t[i] : P.pfpxb_s[i];
      double pfy = t == 0 ? P.pfpyb_t[i] : P.pfpyb_s[i];
      double ah = t == 0 ? P.ah_bottom_t[i] : P.ah_bottom_s[i];
      double tmp1 = pfx * P.cos_sita[i] + pfy * P.sin_sita[i];
      double tmp2 = ah * P.phpn[i];
      double tmp3 = khbottom + UMOLPR + ah * P.phpn[i] * P.phpn[i];
      double tmp = tmp1 * tmp2 / tmp3 * (khbottom + UMOLPR);
      if (t == 0) {
        if (tmp1 > 0.0) tmp = 0.0;
      } else {
        if (tmp1 < 0.0) tmp = 0.0;
        tmp = -tmp;
      }
      double cfb = CF(KBM1);
      const double rad_b = RAD(KBM1), rad_kb = RAD(KB);
      double ff = (cfb * vhpf[KBM2] - F[n3(KBM1)] - GW + DTI * (rad_b - rad_kb - tmp) / (d * P.dz[n3(KBM1)])) /
                  (cfb * (1. - vhf[KBM2]) - 1.);
      F[n3(KBM1)] = ff;
      for (int k = 2; k <= KBM1; ++k) {
        int ki = KB - k;
        ff = (vhf[ki] * ff + vhpf[ki]);
        F[n3(ki)] = ff;
      }
    }
  }
}

// -------------------------------------------------------------------------------------
// BCOND_TS(1) and BCOND_TS(2) (bcond_ts.F:60-262): river nodes take the river T/S; open
// boundary nodes take the outflow estimate with the radiation perturbation of
// OBC_TS_TYPE and the neighbour clamp, or keep T1/S1 on inflow.  One block.
// -------------------------------------------------------------------------------------
__global__ void k_bcond_ts_riv(const Dev P) {
  const int KBM1 = P.KBM1;
  for (int r = threadIdx.x + 1; r <= P.numqbc; r += blockDim.x) {
    int n1 = P.river_location == 0 ? P.inodeq[r] : P.n_icellq[r];
    int n2 = P.river_location == 0 ? 0 : P.n_icellq[(size_t)(P.numqbc + 1) + r];
    for (int k = 1; k <= KBM1; ++k) {
      P.tf1[N3(P, n1, k)] = P.tdis[r];
      P.sf1[N3(P, n1, k)] = P.sdis[r];
      if (n2 > 0) {
        P.tf1[N3(P, n2, k)] = P.tdis[r];
        P.sf1[N3(P, n2, k)] = P.sdis[r];
      }
    }
  }
}

// Open-boundary part: one thread per (open-boundary node, tracer).  The nodes are
// independent: each reads the old field, its own XFLUX_OBC and TF1/SF1 of its interior
// neighbour NEXT_OBC, which is not an open-boundary node.
__global__ void k_bcond_ts_obc(const Dev P, int parts) {
  const int KBM1 = P.KBM1;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const int ob = id / 2 + 1, t = id % 2;
  if (ob > P.iobcn) return;
  {
    int j = P.i_obc_n[ob], j1 = P.next_obc[ob];
    {
      if (!(parts & (t == 0 ? AD_T : AD_S))) return;
      const double* F1 = t == 0 ? P.t1 : P.s1;
      double* FF1 = t == 0 ? P.tf1 : P.sf1;
      const double* XO = t == 0 ? P.xflux_obc_t : P.xflux_obc_s;
      double t2d = 0.0, t2dn = 0.0, xf2d = 0.0;
      for (int k = 1; k <= KBM1; ++k) {
        t2d = t2d + F1[N3(P, j, k)] * P.dz[N3(P, j, k)];
        t2dn = t2dn + FF1[N3(P, j1, k)] * P.dz[N3(P, j1, k)];
        xf2d = xf2d + XO[(size_t)(k - 1) * (P.iobcn + 1) + ob];
      }
      if (P.uard_obcn[ob] > 0.0) {
        double tmp = xf2d + t2d * P.uard_obcn[ob];
        double t2d_obc = (t2d * P.dt[j] - tmp * P.dti / P.art1[j]) / P.d[j];
        double cc = 0.0, cp = 1.0;
        if (P.obc_ts_type != 1) {
          cc = sqrt(P.grav_n[j] * P.h[j]) * P.dti / P.dltn_obc[ob];
          cp = cc + 1.0;
        }
        for (int k = 1; k <= KBM1; ++k) {
          double ttmp;
          double pert_next = FF1[N3(P, j1, k)] - t2dn;
          if (P.obc_ts_type == 1) {
            ttmp = pert_next;
          } else if (P.obc_ts_type == 2) {
            double pert = F1[N3(P, j, k)] - t2d;
            ttmp = (cc * pert_next + pert) / cp;
          } else {
            double pert = F1[N3(P, j, k)] - t2d;
            ttmp = (cc * pert_next + pert * (1.0 - P.dti / 10800.0)) / cp;
          }
          FF1[N3(P, j, k)] = t2d_obc + ttmp;
        }
        for (int k = 1; k <= KBM1; ++k) {
          double fmx = F1[N3(P, NBSN(P, j, 1), k)], fmn = fmx;
          for (int jj = 2; jj <= P.ntsn[j]; ++jj) {
            double v = F1[N3(P, NBSN(P, j, jj), k)];
            fmx = fmax(fmx, v);
            fmn = fmin(fmn, v);
          }
          fct_layer_bounds(P, j, k, F1, fmx, fmn);
          double ff = FF1[N3(P, j, k)];
          if (fmn - ff > 0.0) ff = fmn;
          if (ff - fmx > 0.0) ff = fmx;
          FF1[N3(P, j, k)] = ff;
        }
      } else {
        for (int k = 1; k <= KBM1; ++k) FF1[N3(P, j, k)] = F1[N3(P, j, k)];
      }
    }
  }
}

// DENS2_2D (eqs_of_state.F:290-319), same operation order.
__device__ inline double dens2(double S, double T) {
  double r = S * S * S * 6.76786136E-6 - S * S * 4.8249614E-4 + S * 8.14876577E-1 - 0.22584586E0;
  r = r * (T * T * T * 1.667E-8 - T * T * 8.164E-7 + T * 1.803E-5);
  r = r + 1.0 - T * T * T * 1.0843E-6 + T * T * 9.8185E-5 - T * 4.786E-3;
  r = r * (S * S * S * 6.76786136E-6 - S * S * 4.8249614E-4 + S * 8.14876577E-1 + 3.895414E-2);
  r = r - (T - 3.98) * (T - 3.98) * (T + 283.0) / (503.57 * (T + 67.26));
  return r * 1.e-3;
}

// -------------------------------------------------------------------------------------
// End of the internal step: T1=TF1, S1=SF1, N2E3D to T/S, DENS2 with N2E3D(RHO1,RHO),
// N2E3D(KM,KM1), U=UF, V=VF, ET=EL, DT=D, ET1=EL1, DT1=D1, WD_UPDATE(3)
// (internal_step.F:1053-1590).  Threads over (max(M,N)+1) x KB.
// -------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_final(const Dev P, int parts) {
  int i = blockIdx.x * 32 + threadIdx.x;
  int k = blockIdx.y * 8 + threadIdx.y + 1;
  if (k > P.KB) return;
  const double* Tn = (parts & FI_T) ? P.tf1 : P.t1;
  const double* Sn = (parts & FI_S) ? P.sf1 : P.s1;
  if (i <= P.M) {
    size_t q = N3(P, i, k);
    if (parts & FI_T) P.t1[q] = P.tf1[q];
    if (parts & FI_S) P.s1[q] = P.sf1[q];
    if (parts & FI_DENS) P.rho1[q] = (k == P.KB || i == 0) ? 0.0 : dens2(Sn[q], Tn[q]);
    if ((parts & FI_SHIFT) && k == 1) {
      P.et[i] = P.el[i];
      P.dt[i] = P.d[i];
      if (P.wetting_drying_on) P.iswetnt[i] = P.iswetn[i];
    }
  }
  if (i >= 1 && i <= P.N) {
    const size_t n1 = P.N + 1;
    int a = P.nv[i], b = P.nv[n1 + i], c = P.nv[2 * n1 + i];
    size_t qa = N3(P, a, k), qb = N3(P, b, k), qc = N3(P, c, k);
    size_t q = C3(P, i, k);
    if (parts & FI_T) P.t[q] = ONE_THIRD * (P.tf1[qa] + P.tf1[qb] + P.tf1[qc]);
    if (parts & FI_S) P.s[q] = ONE_THIRD * (P.sf1[qa] + P.sf1[qb] + P.sf1[qc]);
    if (parts & FI_DENS) {
      double ra = k == P.KB ? 0.0 : dens2(Sn[qa], Tn[qa]);
      double rb = k == P.KB ? 0.0 : dens2(Sn[qb], Tn[qb]);
      double rc = k == P.KB ? 0.0 : dens2(Sn[qc], Tn[qc]);
      P.rho[q] = ONE_THIRD * (ra + rb + rc);
    }
    if (parts & FI_KM1) P.km1[q] = ONE_THIRD * (P.km[qa] + P.km[qb] + P.km[qc]);
    if (parts & FI_SHIFT) {
      P.u[q] = P.uf[q];
      P.v[q] = P.vf[q];
      if (k == 1) {
        P.et1[i] = P.el1[i];
        P.dt1[i] = P.d1[i];
        if (P.wetting_drying_on) P.iswetct[i] = P.iswetc[i];
      }
    }
  }
}

// FP64 budgets over node control volumes, fixed-order two-level reduction.
__global__ void k_budget_partial(const Dev P, double* part) {
  __shared__ double sv[256], sh[256], ss[256];
  int tid = threadIdx.x;
  double v = 0.0, hh = 0.0, s = 0.0;
  for (int i = blockIdx.x * blockDim.x + tid + 1; i <= P.M; i += gridDim.x * blockDim.x) {
    double dd = P.d[i] * P.art1[i];
    double ct = 0.0, cs = 0.0;
    for (int k = 1; k <= P.KBM1; ++k) {
      ct = ct + P.t1[N3(P, i, k)] * P.dz[N3(P, i, k)];
      cs = cs + P.s1[N3(P, i, k)] * P.dz[N3(P, i, k)];
    }
    v = v + dd;
    hh = hh + ct * dd;
    s = s + cs * dd;
  }
  sv[tid] = v; sh[tid] = hh; ss[tid] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (tid < st) { sv[tid] += sv[tid + st]; sh[tid] += sh[tid + st]; ss[tid] += ss[tid + st]; }
    __syncthreads();
  }
  if (tid == 0) { part[3 * blockIdx.x] = sv[0]; part[3 * blockIdx.x + 1] = sh[0]; part[3 * blockIdx.x + 2] = ss[0]; }
}
__global__ void k_budget_final(const double* part, int nb, double* out) {
  if (threadIdx.x != 0) return;
  double a = 0.0, b = 0.0, c = 0.0;
  for (int j = 0; j < nb; ++j) { a += part[3 * j]; b += part[3 * j + 1]; c += part[3 * j + 2]; }
  out[0] = a; out[1] = b; out[2] = c;
}

void launch_grad(const Dev& P, cudaStream_t s, int which) {
  FVG_F32_FORWARD(launch_grad(P, s, which));
  const dim3 g = col_grid(P, P.M, which == 0 ? P.KBM1 - 1 : P.KBM1);
  k_grad<RF><<<g, P.col_bc, 0, s>>>(P, which);
}
void launch_adv_q(const Dev& P, cudaStream_t s, int parts) {
  FVG_F32_FORWARD(launch_adv_q(P, s, parts));
  k_he_adv<RF, 0><<<col_grid(P, P.N, P.KBM1 - 1), P.col_bc, 0, s>>>(P, parts);
  k_gather_q<RF><<<col_grid(P, P.M, P.KBM1 - 1), P.col_bc, 0, s>>>(P, parts);
}
void launch_fct_q(const Dev& P, cudaStream_t s, int parts) {
  dim3 b(32, 8), g(nblk(P.M, 32), nblk(P.KBM1 - 1, 8));
  k_fct_q<<<g, b, 0, s>>>(P, parts);
}
void launch_vdif_q(const Dev& P, cudaStream_t s, int copy_back) {
  const int aux = (P.closure ? 1 : 0) | (P.clos_samp ? 2 : 0);
  void (*lv)(const Dev) = aux == 0 ? k_vdif_q_levels<0> : aux == 1 ? k_vdif_q_levels<1>
                        : aux == 2 ? k_vdif_q_levels<2> : k_vdif_q_levels<3>;
  void (*cf)(const Dev, int) = aux == 0 ? k_vdif_q_coef<0> : aux == 1 ? k_vdif_q_coef<1>
                             : aux == 2 ? k_vdif_q_coef<2> : k_vdif_q_coef<3>;
  lv<<<col_grid(P, P.M, P.KB), P.col_bc, 0, s>>>(P);
  k_vdif_q_sweep<<<dim3(nblk(P.M, 128), 2), 128, 0, s>>>(P);
  cf<<<col_grid(P, P.M, P.KB), P.col_bc, 0, s>>>(P, copy_back);
  if (!P.closure) launch_vdif_q_shallow(P, s);
}
void launch_turb_update(const Dev& P, cudaStream_t s) {
  int n = (P.M > P.N ? P.M : P.N) + 1;
  dim3 b(32, 8), g(nblk(n, 32), nblk(P.KB, 8));
  k_turb_update<<<g, b, 0, s>>>(P);
}
void launch_adv_ts(const Dev& P, cudaStream_t s, int parts) {
  FVG_F32_FORWARD(launch_adv_ts(P, s, parts));
  k_he_adv<RF, 1><<<col_grid(P, P.N, P.KBM1), P.col_bc, 0, s>>>(P, parts);
  k_gather_ts<RF><<<col_grid(P, P.M, P.KBM1), P.col_bc, 0, s>>>(P, parts);
}
void launch_fct_ts(const Dev& P, cudaStream_t s, int parts) {
  dim3 b(32, 8), g(nblk(P.M, 32), nblk(P.KBM1, 8));
  k_fct_ts<<<g, b, 0, s>>>(P, parts);
}
void launch_vdif_ts(const Dev& P, cudaStream_t s, int parts) {
  if (P.heating_on)
    k_vdif_ts<true><<<dim3(nblk(P.M, 128), 2), 128, 0, s>>>(P, parts);
  else
    k_vdif_ts<false><<<dim3(nblk(P.M, 128), 2), 128, 0, s>>>(P, parts);
}
void launch_bcond_ts(const Dev& P, cudaStream_t s, int parts) {
  k_bcond_ts_riv<<<1, 128, 0, s>>>(P);
  if (P.iobcn > 0) k_bcond_ts_obc<<<nblk(2 * P.iobcn, 64), 64, 0, s>>>(P, parts);
}
void launch_final(const Dev& P, cudaStream_t s, int parts) {
  int n = (P.M > P.N ? P.M : P.N) + 1;
  dim3 b(32, 8), g(nblk(n, 32), nblk(P.KB, 8));
  k_final<<<g, b, 0, s>>>(P, parts);
}
void launch_budget(const Dev& P, cudaStream_t s) {
  const int nb = 148;
  k_budget_partial<<<nb, 256, 0, s>>>(P, P.budget + 3);
  k_budget_final<<<1, 32, 0, s>>>(P.budget + 3, nb, P.budget);
}

}  // namespace fvg / fvg_f32
