// fvg_model.h - device data of one fvg_handle and the kernel entry points.
//
// Layout in HBM: every field keeps FVCOM's 1-based index with its ghost slot 0.  3-D
// fields are stored layer-major ("SoA, layer-contiguous"): element (i, k) of a node
// field at a[(k-1)*ms + i], of a cell field at a[(k-1)*ns + i], where the layer strides
// ms >= M+1 and ns >= N+1 are rounded up to 32 elements so every layer starts on a
// 256-byte boundary and a warp's 32 consecutive nodes/cells in one layer are one
// coalesced 256-byte transaction.
//
// Scatter loops of the reference (edge -> cell, half-edge -> node) run as gathers: each
// target owns a list of its contributing edges in ascending edge number (CSR), so every
// sum is accumulated in exactly the reference's order and no atomics are used.
//
// Time-dependent scalars (RAMP of the internal and of each external step, tidal phase
// arguments of each Runge-Kutta stage) are read from a device schedule table indexed by
// a device step counter, so one captured CUDA graph of an internal step replays for any
// step.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include <vector>

#include "../../include/fvg.h"

namespace fvg {

constexpr int kMaxTide = 8;

// Per-step schedule: [ramp_int, ramp_ext[1..isplit], targ[iext][K][j]].
struct SchedLayout {
  int isplit, ntide, len;
  __host__ __device__ int ramp_int() const { return 0; }
  __host__ __device__ int ramp_ext(int iext) const { return iext; }
  __host__ __device__ int targ(int iext, int K, int j) const {
    return 1 + isplit + ((iext - 1) * 4 + (K - 1)) * ntide + j;
  }
};

// FP32 scratch and mesh metrics of the precision form.  Edge offsets are formed in FP64
// and rounded once: xo[e] = XIJC(e)-XC(IEC(e,1)), xo[NE+1+e] = XIJC(e)-XC(IEC(e,2)), the
// same for y.
struct F32 {
  float4* g34;  // least-squares gradient of U, V per cell and layer {UX, UY, VX, VY} (ns x KB)
  float *alfa2[2], *alfa3[2];  // slope limiters UALFA, VALFA (see Dev)
  float* npk;  // node records of the ring gradients, 16 floats per (node, layer)
  float2* ex2;
  float *xo, *yo, *dltxc, *dltyc, *art, *cc_hvc, *a1u, *a2u;
  float *ce_xoa, *ce_yoa, *ce_xob, *ce_yob, *ce_dx, *ce_dy;
  // The slot table's metrics packed per slot: {XOA, YOA, XOB, YOB} and {DX, DY}
  float4* ce_geo;
  float2* ce_dd;
  // The half-edge metrics packed per position: {DLTXE, DLTYE, XNCVE a, YNCVE a} and
  // {XNCVE b, YNCVE b}; the ring-edge metrics per (ring slot, node): {DLTYTRIE, DLTXTRIE}
  float4* hg4;
  float2* hg2;
  float2* trie;
  // A1U and A2U of each cell packed: {A(c,1), A(c,2), A(c,3), A(c,4)}
  float4 *a1u4, *a2u4;
  // Least-squares gradient of UA, VA per cell packed: {UX, UY, VX, VY}
  float4* g2d4;
  // Compact external stage (compact != 0; set up by fvg_set_precision after checking that
  // the mesh's edge metrics are the ones its node and cell coordinates define, bit for
  // bit: DLTXC = VX(IENODE2)-VX(IENODE1), XIJC = (VX(IENODE1)+VX(IENODE2))/2, DLTXE =
  // XIJC-XC of the half-edge's cell, the same in y).  slot4: per (slot s, cell c) at
  // s*(N+1)+c {code, the other cell, IENODE1, IENODE2}; vxy {VX, VY} per node; xyc {XC, YC}
  // per cell; artcc {ART, CC_HVC} in FP32; exc0 per internal step {ADX2D+DRX2D-WUBOT*ART,
  // ADY2D+DRY2D-WVBOT*ART, 0.001*WSX*ART, 0.001*WSY*ART}; exc1 {COR*ART, ART, H1, GRAV_E};
  // cflag: ISBCE in bits 0-1, IUCP = 1 bit 2, EPOR = 1 bit 3, river momentum entries bit
  // 4, open-boundary flux entries bit 5, a sponge coefficient bit 6.
  int compact;
  int4* slot4;
  double2 *vxy, *xyc;
  float2* artcc;
  double4 *exc0, *exc1;
  int* cflag;
};

// Input and output scaling of the learned closure's network, and the training envelope.
// Input f: kind 0 identity, 1 log(x), 2 asinh(x/scale); then (t - mean)/std.  Output c:
// new part = exp(y*tstd + tmean) - teps.  A column uses the network only when every
// interior level's raw inputs lie in [lo, hi] (0.5 and 99.5 percentiles of the training
// samples).
struct ClosNorm {
  int kind[8];
  float scale[8], mean[8], std[8], lo[8], hi[8];
  float tmean[3], tstd[3], teps;
};

// Cell tiles of the staged 3-D momentum flux kernels.  The cells are split by recursive
// coordinate bisection of their centroids into compact tiles of at most kTileCells cells
// (cells ascending within a tile).  Tile t owns entries ptr[t] .. ptr[t+1]-1 of `cells`:
// its nc[t] own cells, then its halo (the other cells of its cells' edges, the ghost cell
// 0 included where an edge has one).  Its edges are entries eptr[t] .. eptr[t+1]-1 of
// `edges`, each {edge number, local IA | local IB << 16, IENODE1, IENODE2}, local indices
// counting from ptr[t]; own cell j's three edges in slot order are slots[ptr[t]+j], each
// {local edge | side << 16 | ISBC << 17} (w unused).
constexpr int kTileCells = 128;
struct Tiles {
  int n, cap_cells, cap_edges;
  const int *ptr, *nc, *eptr, *cells;
  const int4 *edges, *slots;
};

// Device pointers and sizes, passed by value to kernels.
struct Dev {
  int M, N, KB, KBM1, KBM2, NE, NCV, NCV_I, ms, ns;
  int nbsn_cols, nbve_cols, trie_cols;
  int iobcn, numqbc, ntide;
  int isplit;
  double dte, dti, min_depth, static_ssh_adj, hprnu, umol, vprnu, cbcmin;
  double fact, fm1;
  double const1, vhp1c;  // 16.6**0.6666667 and (15.8*100)**0.6666667 (vdif_q.F:172,227)
  int wetting_drying_on, river_location, obc_ts_type, obc_elev_on, have_wind;
  int heating_on;
  double rheat, zeta1, zeta2;
  int limiter;  // 0 LIMITED_NO, 1 LIMITED_1, 2 the slope limiter alone
  int baropg_z;   // BAROCLINIC_PRESSURE_GRADIENT 'z coordinates' (PHY_BAROPG)
  int gcy;        // ghost cells on the solid boundary (GCY); 0: GCN
  const double *gh_cos, *gh_sin;  // GCY: cos, sin of the edge opposite node j, [(j-1)*(N+1)+c]
  double deltz;   // its z spacing HMAX/600
  double* rhoz;   // RHO1 interpolated to the 600 z levels, [(k-1)*ms + node]
  SchedLayout sl;
  const double* sched;  // schedule table
  int* ctl;             // ctl[0] = current schedule slot; ctl[1] = error word

  // ----- mesh, nodes -----
  const double *vx, *vy, *h, *art1, *art2, *grav_n, *nn_hvc, *cos_sita, *sin_sita, *phpn;
  const int *isonb, *ntsn, *ntve, *nbsn, *nbve, *nbvt;
  const double *dltxtrie, *dltytrie, *dltxecec, *dltyecec, *dltxnec, *dltynec;
  int trie_n;  // entries of DLTXTRIE/DLTYTRIE: (M+1) x ring columns
  const double *z, *zz, *dz, *dzz;  // 3-D node (ms stride)
  // ----- mesh, cells -----
  const double *xc, *yc, *art, *cor, *grav_e, *cc_hvc, *cc_sponge, *cc_z0b, *epor, *iucp;
  const double *sin_alpha, *cos_alpha;
  double* h1;  // H1(0) is reset by EXTUV_EDGE
  const int *nv, *nbe, *isbce;
  const int4* nbe4;  // NBE of each cell packed: {NBE(c,1), NBE(c,2), NBE(c,3), 0}
  const double *a1u, *a2u, *awx, *awy;
  const double *z1, *zz1, *dz1, *dzz1;  // 3-D cell (ns stride)
  // ----- edges / half-edges -----
  const int *iec, *ienode, *isbc;
  const double *xijc, *yijc, *dltxc, *dltyc;
  const int *niec, *ntrg;
  const double *dltxe, *dltye, *dltxncve, *dltyncve;
  // ----- gather lists -----
  const int *node_he_ptr, *node_he;   // node -> half-edges (id*2 + side), ascending id
  // Half-edge data by position: half-edge cell_he[3*c + s] (slot s of cell c) sits at
  // pos = s*ns + c, so that the threads of consecutive cells touch consecutive entries.
  // node_vpos_ell: the lists of node_he over positions and transposed, entry j of node i
  // at j*ms + i, code = pos*2 + side, ascending half-edge id (count = ptr[i+1] - ptr[i]);
  // the threads of consecutive nodes read entry j in one coalesced load.
  const int* node_vpos_ell;
  // Metrics by position, plane j at j*ncvs: DLTXE, DLTYE, DLTXNCVE and DLTYNCVE of the
  // NIEC(he,1) side, DLTXNCVE and DLTYNCVE of the NIEC(he,2) side.
  const double* hg;
  const int *cell_edge;               // cell -> its 3 edges (id*2 + side), ascending id
  // Slot table of the cell edge loops, slot s of cell i at s*(N+1) + i (edges in the order
  // of cell_edge): code = edge*4 + ISBC*2 + side, the two cells, the two nodes, the edge
  // offsets XIJC-XC / YIJC-YC of both cells, DLTXC, DLTYC.  Read coalesced by cell.
  const int *ce_code, *ce_ia, *ce_ib, *ce_j1, *ce_j2;
  const int4* ce_i4;  // the same slot as {code, IA, IB, J1} in one 16-byte load
  const double *ce_xoa, *ce_yoa, *ce_xob, *ce_yob, *ce_dx, *ce_dy;
  const int *cell_he;                 // cell -> its 3 control-volume half-edges (NTRG(he) == cell)
  // ----- open boundary -----
  const int *i_obc_n, *next_obc, *node_obc;  // node_obc[node] = OBC index (0 = none)
  const int *obc_kind;                        // 1: specified elevation, 2: clamped
  const double *dltn_obc;
  const int *cell_obc_ptr, *cell_obc;         // cell -> (obc index*2 + slot)
  const double *fluxf_obc;                    // (0:IOBCN, 2)
  const double *apt, *phai_rad, *emean;       // (0:IOBCN, ntide)
  // ----- rivers -----
  const int *node_riv_ptr, *node_riv;         // node -> (river*2 + which) in order
  const int *cell_riv_ptr, *cell_riv;         // cell -> river momentum entries in order
  const int *inodeq, *icellq, *n_icellq;
  const double *rdisq, *qarea, *sin_angleq, *cos_angleq, *vqdist, *qdis0, *tdis, *sdis;
  const int *riv_skip;                        // node is an OBC or river node (FCT skip)
  const int *cell_bcriv;                      // first river whose inflow cell this is (BCOND_GCN 2/3/5)
  // ----- forcing -----
  const double *wsx, *wsy;
  const double *swrad_w, *wtsurf_w;  // surface heating, W/m^2 before RAMP (0:M)

  // ----- state, node 2-D -----
  double *el, *elf, *elrk, *et, *d, *dt, *dtfa, *egf, *wubot_n, *wvbot_n, *taubm_n;
  double *pfpxb_t, *pfpyb_t, *ah_bottom_t, *pfpxb_s, *pfpyb_s, *ah_bottom_s;
  // node 3-D
  double *t1, *s1, *tf1, *sf1, *rho1, *tmean1, *smean1, *rmean1;
  double *q2, *q2l, *q2f, *q2lf, *l, *km, *kh, *kq, *wts, *viscofh;
  // cell 2-D
  double *el1, *elf1, *elrk1, *et1, *d1, *dt1, *ua, *va, *uaf, *vaf, *uark, *vark;
  double *uard, *vard, *adx2d, *ady2d, *drx2d, *dry2d, *advua, *advva, *pstx, *psty;
  double *wubot, *wvbot, *cbc, *tps, *fluxobn, *taubm, *wusurf, *wvsurf;
  // cell 3-D
  double *u, *v, *uf, *vf, *w, *ww, *advx, *advy, *drhox, *drhoy, *rho, *t, *s, *rmean;
  double *km1, *viscofm;
  // wet/dry
  int *iswetn, *iswetnt, *iswetc, *iswetct, *iswetce;
  // open boundary
  double *xflux_obcn, *uard_obcn, *xflux_obc_t, *xflux_obc_s;
  // river discharge after the ramp
  double* qdis;
  // scratch (node 3-D)
  double *scr_xflux;                         // VERTVL flux
  double *gq[2][6];  // ADV_Q of Q2 / Q2L: PQPX, PQPY, PQPXD, PQPYD, ring min, ring max
  double *gt[2][6];  // ADV_T / ADV_S: the same six per tracer
  double* budget;                            // 3 doubles
  // VDIF_Q between its passes: PROD, GH, DTEF, the q2l DTEF (node 3-D) and UTAU2 (node)
  double *vq_prod, *vq_gh, *vq_dtef, *vq_dtefl, *vq_ut;
  double2* ex2;                              // half-edge fluxes of both tracers (ncvs x KB, by position)
  // VERTVL_EDGE's EXFLUX of each half-edge position and layer, at (k-1)*ncvs + pos; it
  // lives in the allocation of ex2, which is free between ADJUST2D3D and the next advection.
  double* he_vflux;
  double* g2d[4];                            // least-squares gradient of UA, VA per cell (COFA1/2/5/6)
  // Slope limiters of the limited schemes, UALFA and VALFA: per cell of the 2-D mode
  // (N+1) and per cell and layer of the 3-D mode (ns x KB); index 0 holds 1.
  double *alfa2[2], *alfa3[2];
  double* exf2d;                             // EXTEL_EDGE flux of each half-edge position (ncvs)
  double* g3[4];                             // least-squares gradient of U, V per cell and layer (ns x KB)
  int ncvs;                                  // layer stride of the half-edge arrays by position (3*ns)
  // Precision form (fvg_set_precision): 0 = FP64 everywhere; 1 = the edge fluxes and
  // advection (ADVAVE's edge loop, the 3-D momentum edge fluxes, ADV_Q/ADV_T/ADV_S with
  // FCT) in FP32 arithmetic over FP32 scratch and FP32 copies of their mesh metrics.
  int prec;
  F32 f;
  // Closure samples (fvg_closure_sample): when set, VDIF_Q writes for every node and
  // interior level K=2..KBM1 at index (K-2)*M + (I-1) of each plane of CLOS_PLANES:
  // N^2 (BOYGR), S^2, D, sigma Z, u*_surf, u*_bot, Q2, Q2L, the new parts KN*KAPPA*SM,
  // KN*SM, KN*SH*VPRNU that MY2.5 averages into KQ, KM, KH, and 1 for a wet node.
  float* clos_samp;
  // Learned closure (fvg_set_closure): 0 = MY2.5; 1 = the network with MY2.5 as the
  // per-column fallback.  clos_feat: per row r = (K-2)*M + (I-1) the eight network inputs
  // already transformed and standardised, in BF16 (16 bytes, the MMA's A-operand row);
  // clos_envc: per level chunk of VDIF_Q's level kernel and node, 1 if every interior
  // level of the chunk lies inside the training envelope (chunk c at c*(M+1) + I);
  // clos_env: per node 1 = wet and inside the envelope on every interior level; clos_w:
  // the BF16 weight image, clos_b: biases (64 + 64 + 16).
  int closure;
  ClosNorm clos_norm;
  const void* clos_w;
  const float* clos_b;
  uint4* clos_feat;
  unsigned char* clos_envc;
  int* clos_env;
  // clos_list: [0] the number of columns on the network, [1..] their nodes ascending
  // (compacted from clos_env each step); clos_cnt: per-block counts of the compaction
  int *clos_list, *clos_cnt;
  int* clos_err;
  Tiles tl;
  // 1: ADVECTION_EDGE_GCN and ADV_UV_EDGE_GCN run as the tile-staged kernels (no limiter,
  // GCN); 0: one thread per cell gathering its neighbours (tuning key "staged").
  int staged;
  // Column tiling of the 3-D gather kernels: col_bc threads (entities) per block, each
  // walking col_lc consecutive layers, so the entity's index chain (cell -> edge ->
  // neighbour) is resolved from cache after the first layer.  Results do not depend on it.
  int col_bc, col_lc;
  // 1: the external loop's stage kernels load what a stage reads once evict-first (ld1),
  // so that the arrays gathered from neighbours stay in L2 between stages (tuning key
  // "stream_hints"); results do not depend on it.
  int ldcs;
  // Blocks per SM of the compact stage kernel's grid-stride launch (tuning key
  // "ext_grid", default 8: one full wave whose threads walk the cells); 0: one thread per
  // cell.  nsm: the device's SM count.
  int ext_grid, nsm;
};

// Grid of a column-tiled kernel over n entities and nl layers.
inline dim3 col_grid(const Dev& P, int n, int nl) {
  return dim3((unsigned)((n + P.col_bc - 1) / P.col_bc), (unsigned)((nl + P.col_lc - 1) / P.col_lc));
}
// First and last layer of this thread's chunk, layers k0..klast.
__device__ inline void col_range(const Dev& P, int k0, int klast, int& kb, int& ke) {
  kb = k0 + (int)blockIdx.y * P.col_lc;
  ke = kb + P.col_lc - 1;
  if (ke > klast) ke = klast;
}


constexpr int CLOS_IN = 8, CLOS_OUT = 3, CLOS_PLANES = CLOS_IN + CLOS_OUT + 1;

// The learned closure's input transform of feature f: kind 0 identity, 1 log(x),
// 2 asinh(x / scale); then standardised.  The result is rounded to BF16 (8 significant
// bits) for the tensor cores, so the hardware logarithm (__logf, a few ulp of FP32) is
// used, and asinh(y) = sign(y) log(|y| + sqrt(y^2 + 1)) through it, except for |y| < 2^-6
// where asinh(y) = y (1 - y^2/6) to well below BF16's resolution, and |y| > 1e18, where
// it is log(|y|) + log(2).
__device__ inline float clos_feat_transform(const ClosNorm& nm, int f, float x) {
  float t = x;
  const int kind = nm.kind[f];
  if (kind == 1) {
    t = __logf(fmaxf(x, 1e-30f));
  } else if (kind == 2) {
    const float y = x / nm.scale[f], a = fabsf(y);
    const float s = a < 0.015625f ? a * (1.0f - a * a * (1.0f / 6.0f))
                    : (a > 1.0e18f ? __logf(a) + 0.6931472f : __logf(a + sqrtf(a * a + 1.0f)));
    t = copysignf(s, y);
  }
  return (t - nm.mean[f]) / nm.std[f];
}

// index helpers
__host__ __device__ inline size_t N3(const Dev& P, int i, int k) { return (size_t)(k - 1) * P.ms + i; }
__host__ __device__ inline size_t C3(const Dev& P, int i, int k) { return (size_t)(k - 1) * P.ns + i; }
// Velocity of neighbour j (1..3, cell index k) of cell c for the least-squares gradient
// under GCY where the neighbour is missing (k == 0): GHOSTUV2/GHOSTUV3 (ghostuv.F:32-223),
// the cell's velocity projected on the boundary edge opposite node j, or on an
// open-boundary cell the cell's own velocity.  The angle's cos and sin come from the host.
__device__ inline void ghost_uv(const Dev& P, const double* U, const double* V, int c, int j, double& uk,
                                double& vk) {
  if (P.isbce[c] != 2) {
    const size_t q = (size_t)(j - 1) * (P.N + 1) + c;
    const double ca = P.gh_cos[q], sa = P.gh_sin[q];
    const double utmp = U[c] * ca + V[c] * sa;
    const double vtmp = 0.0;
    uk = utmp * ca - vtmp * sa;
    vk = utmp * sa + vtmp * ca;
  } else {
    uk = U[c];
    vk = V[c];
  }
}

// RAMP of the current internal step, from its schedule row.
__device__ inline double ramp_int(const Dev& P) { return P.sched[(size_t)P.ctl[0] * P.sl.len]; }

// A load of an array that one pass reads once (CS: evict-first in L2, ld.global.cs), so
// that the arrays the pass gathers from neighbours keep their L2 lines from one
// Runge-Kutta stage to the next; a plain load otherwise.
template <bool CS, class T>
__device__ __forceinline__ T ld1(const T* p) {
  if constexpr (!CS) {
    return *p;
  } else if constexpr (std::is_same<T, double4>::value) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p)), b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
  } else {
    return __ldcs(p);
  }
}

// Mesh metrics and scratch of the edge-flux kernels by arithmetic type R.  The FP64
// instantiation reads the FP64 arrays and forms the edge offsets as the reference does;
// the FP32 one reads the FP32 copies of the precision form.
template <typename R> struct Mesh;
template <> struct Mesh<double> {
  typedef double2 R2;
  __device__ static double xoa(const Dev& P, int e, int ia) { return P.xijc[e] - P.xc[ia]; }
  __device__ static double yoa(const Dev& P, int e, int ia) { return P.yijc[e] - P.yc[ia]; }
  __device__ static double xob(const Dev& P, int e, int ib) { return P.xijc[e] - P.xc[ib]; }
  __device__ static double yob(const Dev& P, int e, int ib) { return P.yijc[e] - P.yc[ib]; }
  __device__ static double s_xoa(const Dev& P, size_t q) { return P.ce_xoa[q]; }
  __device__ static double s_yoa(const Dev& P, size_t q) { return P.ce_yoa[q]; }
  __device__ static double s_xob(const Dev& P, size_t q) { return P.ce_xob[q]; }
  __device__ static double s_yob(const Dev& P, size_t q) { return P.ce_yob[q]; }
  __device__ static double s_dx(const Dev& P, size_t q) { return P.ce_dx[q]; }
  __device__ static double s_dy(const Dev& P, size_t q) { return P.ce_dy[q]; }
  __device__ static double4 s_geo(const Dev& P, size_t q) {
    return make_double4(P.ce_xoa[q], P.ce_yoa[q], P.ce_xob[q], P.ce_yob[q]);
  }
  __device__ static double2 s_dd(const Dev& P, size_t q) { return make_double2(P.ce_dx[q], P.ce_dy[q]); }
  __device__ static double dltxc(const Dev& P, int e) { return P.dltxc[e]; }
  __device__ static double dltyc(const Dev& P, int e) { return P.dltyc[e]; }
  __device__ static double art(const Dev& P, int c) { return P.art[c]; }
  __device__ static double2 artcc(const Dev& P, int c) { return make_double2(P.art[c], P.cc_hvc[c]); }
  __device__ static double cc_hvc(const Dev& P, int c) { return P.cc_hvc[c]; }
  __device__ static double a1u(const Dev& P, size_t q) { return P.a1u[q]; }
  __device__ static double a2u(const Dev& P, size_t q) { return P.a2u[q]; }
  __device__ static double* g2d(const Dev& P, int q) { return P.g2d[q]; }
  __device__ static double* alfa2(const Dev& P, int q) { return P.alfa2[q]; }
  __device__ static double* alfa3(const Dev& P, int q) { return P.alfa3[q]; }
  __device__ static double* g3(const Dev& P, int q) { return P.g3[q]; }
  __device__ static double2* ex2(const Dev& P) { return P.ex2; }
  __device__ static double hg(const Dev& P, int j, size_t pos) { return P.hg[(size_t)j * P.ncvs + pos]; }
};
template <> struct Mesh<float> {
  typedef float2 R2;
  __device__ static float xoa(const Dev& P, int e, int) { return P.f.xo[e]; }
  __device__ static float yoa(const Dev& P, int e, int) { return P.f.yo[e]; }
  __device__ static float xob(const Dev& P, int e, int) { return P.f.xo[(size_t)P.NE + 1 + e]; }
  __device__ static float yob(const Dev& P, int e, int) { return P.f.yo[(size_t)P.NE + 1 + e]; }
  __device__ static float s_xoa(const Dev& P, size_t q) { return P.f.ce_xoa[q]; }
  __device__ static float s_yoa(const Dev& P, size_t q) { return P.f.ce_yoa[q]; }
  __device__ static float s_xob(const Dev& P, size_t q) { return P.f.ce_xob[q]; }
  __device__ static float s_yob(const Dev& P, size_t q) { return P.f.ce_yob[q]; }
  __device__ static float s_dx(const Dev& P, size_t q) { return P.f.ce_dx[q]; }
  __device__ static float s_dy(const Dev& P, size_t q) { return P.f.ce_dy[q]; }
  __device__ static float4 s_geo(const Dev& P, size_t q) { return P.f.ce_geo[q]; }
  __device__ static float2 s_dd(const Dev& P, size_t q) { return P.f.ce_dd[q]; }
  __device__ static float dltxc(const Dev& P, int e) { return P.f.dltxc[e]; }
  __device__ static float dltyc(const Dev& P, int e) { return P.f.dltyc[e]; }
  __device__ static float art(const Dev& P, int c) { return P.f.art[c]; }
  __device__ static float2 artcc(const Dev& P, int c) { return P.f.artcc[c]; }  // {ART, CC_HVC}
  __device__ static float cc_hvc(const Dev& P, int c) { return P.f.cc_hvc[c]; }
  __device__ static float a1u(const Dev& P, size_t q) { return P.f.a1u[q]; }
  __device__ static float a2u(const Dev& P, size_t q) { return P.f.a2u[q]; }
  __device__ static float* alfa2(const Dev& P, int q) { return P.f.alfa2[q]; }
  __device__ static float* alfa3(const Dev& P, int q) { return P.f.alfa3[q]; }
  __device__ static float2* ex2(const Dev& P) { return P.f.ex2; }
};
// The cell's NBE and its least-squares coefficients A1U(c,1..4), A2U(c,1..4) in the
// form's type (FP32: one packed load each).
template <typename R, bool CS = false>
__device__ inline void lsq_coef(const Dev& P, int c, int& k1, int& k2, int& k3, R* a, R* b) {
  const int4 nb = ld1<CS>(P.nbe4 + c);
  k1 = nb.x;
  k2 = nb.y;
  k3 = nb.z;
  if constexpr (sizeof(R) == 4) {
    const float4 A = ld1<CS>(P.f.a1u4 + c), B = ld1<CS>(P.f.a2u4 + c);
    a[0] = A.x; a[1] = A.y; a[2] = A.z; a[3] = A.w;
    b[0] = B.x; b[1] = B.y; b[2] = B.z; b[3] = B.w;
  } else {
    const size_t n1 = P.N + 1;
    for (int j = 0; j < 4; ++j) {
      a[j] = P.a1u[j * n1 + c];
      b[j] = P.a2u[j * n1 + c];
    }
  }
}
// Limited schemes (advave_edge_gcn.F:226-229, 300-303, 340-357): the slope limiter of one
// cell and edge, min(ALFA, min(1, |U(IA)-U(IB)| / |U'+EPSILON|)), EPSILON of the form's type.
template <typename R>
__device__ inline void lim_alfa(R num, R ext, R& a) {
  R t = num / fabs(ext + (R)(sizeof(R) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07));
  if (t > (R)1) t = (R)1;
  a = t < a ? t : a;
}
// Face values U + ALFA*U' of both cells; under LIMITED_1 both revert to the cell values
// when either leaves their range.
template <typename R>
__device__ inline void lim_faces(int limiter, R ua, R ub, R ea, R eb, R alfa_a, R alfa_b, R& f1, R& f2) {
  f1 = ua + alfa_a * ea;
  f2 = ub + alfa_b * eb;
  if (limiter == 1) {
    R hi = ua > ub ? ua : ub, lo = ua < ub ? ua : ub;
    if (f1 > hi || f1 < lo || f2 > hi || f2 < lo) {
      f1 = ua;
      f2 = ub;
    }
  }
}
__device__ inline double2 mk2(double a, double b) { return make_double2(a, b); }
__device__ inline float2 mk2(float a, float b) { return make_float2(a, b); }

// Fortran SIGN(1.0, x) for a processor that does not distinguish negative zero.
__host__ __device__ inline double fsign1(double x) { return x >= 0.0 ? 1.0 : -1.0; }
__host__ __device__ inline float fsign1(float x) { return x >= 0.0f ? 1.0f : -1.0f; }

extern const double kAlphaRK[5];

// ---------------- external mode (k_ext.cu) ----------------
// EN_FINISH_PREV: first finish the node part of the previous stage's update (EL = ELF,
// D, DTFA, the stage sums), that stage's K in bits 8-10 of parts.
// EN_WET_PREV: before that, the node part of the previous stage's WET_JUDGE (ISWETN and the
// ELF clamp, mod_wd.F:222-284) from that stage's cell flags, then in ISWETCE.
enum ExtNodeParts { EN_EXTEL = 1, EN_BC = 2, EN_COPY_ELRK = 4, EN_GRAD = 8, EN_FINISH_PREV = 16, EN_WET_PREV = 32 };
// EC_FINISH: end with the cell part of the stage's update (EL1, D1, the stage sums, the
// next stage's continuity fluxes from the new UAF, VAF), UA/VA being swapped with
// UAF/VAF between stages instead of copied.
// EC_COMPACT: the stage loop of an internal step may use the compact FP32 kernel (when
// F32::compact is set); EC_LAST: the last stage of that loop (the compact kernel writes
// ADVUA, ADVVA, PSTX, PSTY only there and in the internal-step ADVAVE call).
enum ExtCellParts { EC_N2E = 1, EC_FLUXOBN = 2, EC_ADVAVE = 4, EC_EXTUV = 8, EC_BC2 = 16, EC_COPY_RK = 32,
                    EC_INT_ADVAVE = 64, EC_FINISH = 128, EC_COMPACT = 256, EC_LAST = 512 };
void launch_ext_finish(const Dev& P, cudaStream_t s, int K, int wet_prev);
// pdl: launched as a programmatic dependent of the previous kernel in the stream (the
// fused external loop); the kernel waits for that kernel's completion before it touches
// memory, while its blocks are scheduled during the previous kernel's tail.
void launch_ext_node(const Dev& P, cudaStream_t s, int iext, int K, int parts, int pdl = 0);
void launch_wet_judge(const Dev& P, cudaStream_t s);
void launch_wet_cells(const Dev& P, cudaStream_t s, int pdl = 0);
void launch_ext_cell(const Dev& P, cudaStream_t s, int iext, int K, int parts, int pdl = 0);
void launch_alfa2(const Dev& P, cudaStream_t s);
void launch_ext_update(const Dev& P, cudaStream_t s, int K);
void launch_begin_step(const Dev& P, cudaStream_t s);
void launch_ext_prep(const Dev& P, cudaStream_t s);
void launch_make_f32(const Dev& P, cudaStream_t s);
// Fill the compact external stage's records and count (into *mismatch, device memory)
// the mesh metrics that differ from the ones the coordinates define.
void launch_make_compact(const Dev& P, cudaStream_t s, int* mismatch);
void launch_closure(const Dev& P, cudaStream_t s, int* err, int grid);
void launch_vdif_q_shallow(const Dev& P, cudaStream_t s);
size_t closure_smem_bytes();
int closure_ctas_per_sm();
size_t closure_weight_image_bytes();
int closure_setup_attrs();
void launch_mlp_tc_forward(const void* wimg, const float* bias, const float* x, int n, float* out, int* err, int grid,
                           cudaStream_t s);
void closure_weight_image(const float* params, std::vector<uint8_t>& img, std::vector<float>& bias);
void launch_set_qdis(const Dev& P, cudaStream_t s);

// ---------------- 3-D momentum (k_mom3d.cu) ----------------
enum CellPreParts { CP_ADJUST1 = 1, CP_BC5 = 2, CP_BCOND8 = 4, CP_BROUGH = 8 };
void launch_cell_pre(const Dev& P, cudaStream_t s, int parts);
void launch_grad3(const Dev& P, cudaStream_t s);
void launch_advection3d(const Dev& P, cudaStream_t s);
void launch_baropg(const Dev& P, cudaStream_t s, int do_baropg, int do_sums);
void launch_phy_baropg(const Dev& P, cudaStream_t s);
void launch_int_reset(const Dev& P, cudaStream_t s);
// ADJUST2D3D(2) (AJ_ADJUST) and the half-edge fluxes of VERTVL_EDGE (AJ_HE_FLUX)
enum Adjust2Parts { AJ_ADJUST = 1, AJ_HE_FLUX = 2 };
void launch_adjust2(const Dev& P, cudaStream_t s, int parts);
void launch_vertvl_flux(const Dev& P, cudaStream_t s);
enum VertvlColParts { VC_WTS = 1, VC_WD2 = 2, VC_RHO_ROUNDTRIP = 4, VC_BOT_NODE = 8 };
void launch_vertvl_col(const Dev& P, cudaStream_t s, int parts);
void launch_w_viscofh(const Dev& P, cudaStream_t s, int do_w, int do_visc);
void launch_adv_uv(const Dev& P, cudaStream_t s);
int staged_setup();  // shared-memory limit of the tile-staged momentum kernels; 0 on success
enum VdifUvParts { VU_VDIF = 1, VU_BC3 = 2, VU_WREAL = 4 };
void launch_vdif_uv(const Dev& P, cudaStream_t s, int parts);

// ---------------- scalars and turbulence (k_scalar.cu) ----------------
void launch_grad(const Dev& P, cudaStream_t s, int which);  // 0: q2+q2l, 1: T+S
enum AdvParts { AD_Q2 = 1, AD_Q2L = 2, AD_FCT = 4, AD_T = 8, AD_S = 16 };
void launch_adv_q(const Dev& P, cudaStream_t s, int parts);
void launch_fct_q(const Dev& P, cudaStream_t s, int parts);
void launch_vdif_q(const Dev& P, cudaStream_t s, int copy_back);
void launch_turb_update(const Dev& P, cudaStream_t s);
void launch_adv_ts(const Dev& P, cudaStream_t s, int parts);
void launch_fct_ts(const Dev& P, cudaStream_t s, int parts);
void launch_vdif_ts(const Dev& P, cudaStream_t s, int parts);
void launch_bcond_ts(const Dev& P, cudaStream_t s, int parts);
enum FinalParts { FI_T = 1, FI_S = 2, FI_DENS = 4, FI_KM1 = 8, FI_SHIFT = 16 };
void launch_final(const Dev& P, cudaStream_t s, int parts);
void launch_budget(const Dev& P, cudaStream_t s);

}  // namespace fvg

// The precision form's FP32 flux kernels, compiled separately with multiply-add
// contraction (the FP64 kernels keep --fmad=false for their bitwise parity).  Launchers
// of kernels that have an FP32 instantiation forward to these when P.prec is set.
namespace fvg_f32 {
using fvg::Dev;
void launch_alfa2(const Dev& P, cudaStream_t s);
void launch_ext_cell(const Dev& P, cudaStream_t s, int iext, int K, int parts, int pdl);
void launch_grad3(const Dev& P, cudaStream_t s);
void launch_advection3d(const Dev& P, cudaStream_t s);
void launch_adv_uv(const Dev& P, cudaStream_t s);
void launch_grad(const Dev& P, cudaStream_t s, int which);
void launch_adv_q(const Dev& P, cudaStream_t s, int parts);
void launch_adv_ts(const Dev& P, cudaStream_t s, int parts);
int staged_setup();
}  // namespace fvg_f32

// RF: the arithmetic type of the flux kernels this translation unit launches.
#ifdef FVG_F32_TU
using RF = float;
#define FVG_F32_FORWARD(call)
#else
using RF = double;
#define FVG_F32_FORWARD(call) \
  do {                          \
    if (P.prec) {               \
      fvg_f32::call;            \
      return;                   \
    }                           \
  } while (0)
#endif
