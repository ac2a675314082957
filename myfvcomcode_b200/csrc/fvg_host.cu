// fvg_host.cu - C ABI (include/fvg.h) of the B200 mode-split step.
//
// fvg_create copies FVCOM's mesh arrays to the device, builds the gather lists that turn
// the reference's scatter loops into ordered per-target sums, and allocates the state.
// fvg_internal_step / fvg_run enqueue one INTERNAL_STEP (FVCOM_source/internal_step.F:29)
// as a fixed kernel sequence; the sequence is captured once into a CUDA graph and
// replayed, with the per-step scalars (RAMP, tidal phase arguments) supplied through a
// device schedule table that the host fills ahead of each batch of steps.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "fvg_model.h"

using namespace fvg;

namespace {

const double kPI2 = 2.0 * 3.141592653589793238;

struct FieldDesc {
  void* d = nullptr;
  int64_t rows = 0;   // len+1
  int layers = 1;
  int64_t stride = 0; // device elements between layers
  bool is_int = false;
};

}  // namespace

struct fvg_handle {
  Dev P{};
  fvg_params prm{};
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  std::map<std::string, FieldDesc> fields;
  std::string err;
  int32_t iint = 0;
  double ext_time = 0.0;
  double ramp = 0.0;
  int ntide = 0;
  std::vector<double> period;
  int sched_cap = 0;
  double* d_sched = nullptr;
  double* h_sched = nullptr;  // pinned
  int* h_ctl = nullptr;       // pinned
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  bool use_graph = true;
  int clos_grid = 148;
  // compact external stage of the precision form: allowed (tuning key "compact") and
  // possible (the mesh check of fvg_set_precision passed)
  int compact_allowed = 1;
  int compact_ok = 0;
};

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
      return FVG_ERR_CUDA;                                                            \
    }                                                                                 \
  } while (0)

namespace {

template <class T>
int dalloc(fvg_handle* h, T** p, size_t n) {
  void* q = nullptr;
  size_t bytes = (n == 0 ? 1 : n) * sizeof(T);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return FVG_ERR_NOMEM;
  }
  cudaMemset(q, 0, bytes);
  h->allocs.push_back(q);
  *p = (T*)q;
  return FVG_OK;
}

template <class T>
int upload(fvg_handle* h, T** p, const T* src, size_t n) {
  int rc = dalloc(h, p, n);
  if (rc) return rc;
  if (src && n) CK(cudaMemcpy(*p, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return FVG_OK;
}

// (0:len, 1:KB) Fortran array -> layer-strided device array
int upload3(fvg_handle* h, double** p, const double* src, size_t rows, int kb, size_t stride) {
  int rc = dalloc(h, p, stride * kb);
  if (rc) return rc;
  if (src)
    CK(cudaMemcpy2D(*p, stride * sizeof(double), src, rows * sizeof(double), rows * sizeof(double), kb,
                    cudaMemcpyHostToDevice));
  return FVG_OK;
}

inline size_t pad32(size_t n) { return (n + 31) / 32 * 32; }

// Cell tiles of the staged momentum kernels (struct Tiles): recursive coordinate bisection
// of the cell centroids, the larger extent split at a multiple of the tile size.  cl[i]:
// cell i's edges (edge*2 + side) in ascending edge order; iec: IEC (NE+1, 2) column-major.
struct TileBuild {
  std::vector<int> ptr, nc, eptr, cells;
  std::vector<int> edges, slots;  // 4 ints per entry
  int cap_cells = 0, cap_edges = 0;
};
void rcb(std::vector<int>& ids, size_t b, size_t e, const double* xc, const double* yc, std::vector<size_t>& cuts) {
  const size_t n = e - b;
  if (n <= (size_t)fvg::kTileCells) {
    cuts.push_back(e);
    return;
  }
  double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
  for (size_t q = b; q < e; ++q) {
    x0 = std::min(x0, xc[ids[q]]); x1 = std::max(x1, xc[ids[q]]);
    y0 = std::min(y0, yc[ids[q]]); y1 = std::max(y1, yc[ids[q]]);
  }
  const bool byx = (x1 - x0) >= (y1 - y0);
  const size_t ntile = (n + fvg::kTileCells - 1) / fvg::kTileCells;
  const size_t mid = b + ((ntile + 1) / 2) * fvg::kTileCells;
  auto key = [&](int c) { return byx ? std::make_pair(xc[c], c) : std::make_pair(yc[c], c); };
  std::nth_element(ids.begin() + b, ids.begin() + mid, ids.begin() + e,
                   [&](int a, int c) { return key(a) < key(c); });
  rcb(ids, b, mid, xc, yc, cuts);
  rcb(ids, mid, e, xc, yc, cuts);
}
void build_tiles(int N, int NE, const double* xc, const double* yc, const int* iec, const int* ienode,
                 const int* isbc, const std::vector<std::vector<int>>& cl, TileBuild& tb) {
  const size_t e1 = (size_t)NE + 1;
  std::vector<int> ids(N);
  for (int i = 0; i < N; ++i) ids[i] = i + 1;
  std::vector<size_t> cuts;
  rcb(ids, 0, ids.size(), xc, yc, cuts);
  std::vector<int> local((size_t)N + 1, -1), elocal(e1, -1);
  size_t b = 0;
  tb.ptr.push_back(0);
  tb.eptr.push_back(0);
  for (size_t cut : cuts) {
    std::vector<int> own(ids.begin() + b, ids.begin() + cut);
    b = cut;
    std::sort(own.begin(), own.end());
    std::vector<int> all(own), elist;
    for (size_t j = 0; j < own.size(); ++j) local[own[j]] = (int)j;
    for (int c : own)
      for (int code : cl[c]) {
        const int e = code >> 1, side = code & 1;
        const int o = side == 0 ? iec[e1 + e] : iec[e];
        if (local[o] < 0) {
          local[o] = (int)all.size();
          all.push_back(o);
        }
        if (elocal[e] < 0) {
          elocal[e] = (int)elist.size();
          elist.push_back(e);
        }
      }
    for (int e : elist) {
      tb.edges.push_back(e);
      tb.edges.push_back(local[iec[e]] | (local[iec[e1 + e]] << 16));
      tb.edges.push_back(ienode[e]);
      tb.edges.push_back(ienode[e1 + e]);
    }
    for (int c : own) {
      for (int sl = 0; sl < 3; ++sl) {
        const int code = cl[c][sl], e = code >> 1;
        tb.slots.push_back(elocal[e] | ((code & 1) << 16) | ((isbc[e] != 0 ? 1 : 0) << 17));
      }
      tb.slots.push_back(0);
    }
    for (int c : all) tb.cells.push_back(c);
    tb.nc.push_back((int)own.size());
    tb.ptr.push_back((int)tb.cells.size());
    // own cells' slot entries are padded to the tile's cell count (halo entries unused)
    for (size_t j = own.size(); j < all.size(); ++j)
      for (int w = 0; w < 4; ++w) tb.slots.push_back(0);
    tb.eptr.push_back((int)(tb.edges.size() / 4));
    tb.cap_cells = std::max(tb.cap_cells, (int)all.size());
    tb.cap_edges = std::max(tb.cap_edges, (int)elist.size());
    for (int c : all) local[c] = -1;
    for (int e : elist) elocal[e] = -1;
  }
}

int build_csr(const std::vector<std::vector<int>>& lists, std::vector<int>& ptr, std::vector<int>& ent) {
  ptr.assign(lists.size() + 1, 0);
  for (size_t i = 0; i < lists.size(); ++i) ptr[i + 1] = ptr[i] + (int)lists[i].size();
  ent.clear();
  for (auto& l : lists) ent.insert(ent.end(), l.begin(), l.end());
  return FVG_OK;
}

// Schedule row for internal step iint (1-based) whose ExtTime before the step is t0.
void fill_sched_row(const fvg_handle* h, double* row, int32_t iint, double t0) {
  const fvg_params& p = h->prm;
  const SchedLayout& sl = h->P.sl;
  row[sl.ramp_int()] = p.iramp != 0 ? std::tanh((double)iint / (double)p.iramp) : 1.0;
  double ext = t0;
  for (int iext = 1; iext <= p.isplit; ++iext) {
    ext = ext + p.dte;
    if (p.iramp != 0) {
      double tmp = (double)(iint - 1) + (double)iext / (double)p.isplit;
      row[sl.ramp_ext(iext)] = std::tanh(tmp / (double)p.iramp);
    } else {
      row[sl.ramp_ext(iext)] = 1.0;
    }
    for (int K = 1; K <= 4; ++K) {
      double rktime = ext + p.dte * (kAlphaRK[K] - 1.0);
      double te = rktime - p.tide_ref_time;
      for (int j = 0; j < h->ntide; ++j) row[sl.targ(iext, K, j)] = te * kPI2 / h->period[j];
    }
  }
}

// Row used by fvg_run_routine: current RAMP everywhere, phases from the current ExtTime.
void fill_routine_row(const fvg_handle* h, double* row) {
  const fvg_params& p = h->prm;
  const SchedLayout& sl = h->P.sl;
  for (int q = 0; q < sl.len; ++q) row[q] = 0.0;
  row[sl.ramp_int()] = h->ramp;
  for (int iext = 1; iext <= p.isplit; ++iext) {
    row[sl.ramp_ext(iext)] = h->ramp;
    for (int K = 1; K <= 4; ++K) {
      double rktime = h->ext_time + p.dte * (kAlphaRK[K] - 1.0);
      double te = rktime - p.tide_ref_time;
      for (int j = 0; j < h->ntide; ++j) row[sl.targ(iext, K, j)] = te * kPI2 / h->period[j];
    }
  }
}

// Kernel groups reported by fvg_profile (order of enqueue_internal_step).
const char* kGroupNames[] = {"cell_pre", "advection3d", "baropg", "int_advave", "ext_node", "wet_judge",
                             "ext_cell", "ext_update", "adjust2", "vertvl_flux", "vertvl_col", "w_viscofh",
                             "adv_uv", "vdif_uv", "grad_q", "adv_q", "vdif_q", "grad_ts", "adv_ts",
                             "vdif_ts", "bcond_ts", "final", "closure"};
enum { G_CELL_PRE, G_ADV3D, G_BAROPG, G_INT_ADVAVE, G_EXT_NODE, G_WET, G_EXT_CELL, G_EXT_UPD, G_ADJ2,
       G_VV_FLUX, G_VV_COL, G_W_VISC, G_ADV_UV, G_VDIF_UV, G_GRAD_Q, G_ADV_Q, G_VDIF_Q, G_GRAD_TS,
       G_ADV_TS, G_VDIF_TS, G_BCOND_TS, G_FINAL, G_CLOSURE, G_COUNT };

struct Marker {
  std::vector<cudaEvent_t>* ev = nullptr;
  std::vector<int>* grp = nullptr;
  void mark(cudaStream_t s, int g) {
    if (!ev) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    ev->push_back(e);
    grp->push_back(g);
  }
};

// One INTERNAL_STEP as a kernel sequence (internal_step.F:115-1590).
void enqueue_internal_step(fvg_handle* h, cudaStream_t s, Marker mk = Marker()) {
  const Dev& P = h->P;
  const fvg_params& p = h->prm;
  const int spc = p.scalar_positivity_control ? AD_FCT : 0;
  mk.mark(s, -1);
  launch_begin_step(P, s);
  launch_cell_pre(P, s, CP_ADJUST1 | CP_BC5 | CP_BCOND8 | CP_BROUGH);
  mk.mark(s, G_CELL_PRE);
  launch_grad3(P, s);
  launch_advection3d(P, s);
  mk.mark(s, G_ADV3D);
  if (!p.barotropic && P.baropg_z) {
    launch_phy_baropg(P, s);
    launch_baropg(P, s, 0, 1);
  } else {
    launch_baropg(P, s, !p.barotropic, 1);
  }
  launch_ext_prep(P, s);
  if (P.limiter) launch_alfa2(P, s);
  mk.mark(s, G_BAROPG);
  launch_ext_cell(P, s, 1, 1, EC_INT_ADVAVE | EC_COMPACT);
  launch_int_reset(P, s);
  mk.mark(s, G_INT_ADVAVE);
  // The ISPLIT x 4 Runge-Kutta stages.  Instead of copying UAF to UA and ISWETC to
  // ISWETCE after each stage (external_step.F:333-436), the stage reads and writes swapped
  // arrays: stage n+1's UA is stage n's UAF, its ISWETCE stage n's ISWETC.  The update's
  // cell part ends the cell kernel, its node part starts the next stage's node kernel,
  // and k_ext_finish closes the last stage (an even number of stages leaves the arrays in
  // their own roles).  With wetting and drying, WET_JUDGE's node part (ISWETN, the ELF
  // clamp) moves the same way to the head of the next node kernel; FLUX_OBN, the one
  // reader of ELF in between, applies the clamp itself.
  int stage = 0;
  for (int iext = 1; iext <= p.isplit; ++iext) {
    for (int K = 1; K <= 4; ++K, ++stage) {
      Dev Q = P;
      if (stage & 1) {
        std::swap(Q.ua, Q.uaf);
        std::swap(Q.va, Q.vaf);
        std::swap(Q.iswetce, Q.iswetc);
      }
      const int prev =
          stage > 0 ? (EN_FINISH_PREV | (p.wetting_drying_on ? EN_WET_PREV : 0) | ((K == 1 ? 4 : K - 1) << 8)) : 0;
      // stage > 0: each kernel of the loop overlaps its launch with the previous one's tail
      const int pdl = stage > 0 ? 1 : 0;
      launch_ext_node(Q, s, iext, K, EN_EXTEL | EN_BC | EN_GRAD | (K == 1 ? EN_COPY_ELRK : 0) | prev, pdl);
      mk.mark(s, G_EXT_NODE);
      if (p.wetting_drying_on) {
        launch_wet_cells(Q, s, 1);  // its node part opens the next stage's node kernel
        mk.mark(s, G_WET);
      }
      if (P.limiter) launch_alfa2(Q, s);
      launch_ext_cell(Q, s, iext, K,
                      (p.wetting_drying_on ? 0 : EC_N2E) | EC_FLUXOBN | EC_ADVAVE | EC_EXTUV | EC_BC2 |
                          (K == 1 ? EC_COPY_RK : 0) | EC_FINISH | EC_COMPACT |
                          (iext == p.isplit && K == 4 ? EC_LAST : 0),
                      P.limiter ? 0 : 1);
      mk.mark(s, G_EXT_CELL);
    }
  }
  launch_ext_finish(P, s, 4, p.wetting_drying_on);
  mk.mark(s, G_EXT_UPD);
  launch_adjust2(P, s, AJ_ADJUST | AJ_HE_FLUX);
  mk.mark(s, G_ADJ2);
  launch_vertvl_flux(P, s);
  mk.mark(s, G_VV_FLUX);
  launch_vertvl_col(P, s, VC_WTS | VC_WD2 | (p.barotropic || P.baropg_z ? 0 : VC_RHO_ROUNDTRIP) | VC_BOT_NODE);
  mk.mark(s, G_VV_COL);
  launch_w_viscofh(P, s, 1, 1);
  mk.mark(s, G_W_VISC);
  launch_grad3(P, s);
  launch_adv_uv(P, s);
  mk.mark(s, G_ADV_UV);
  launch_vdif_uv(P, s, VU_VDIF | VU_BC3 | VU_WREAL);
  mk.mark(s, G_VDIF_UV);
  launch_grad(P, s, 0);
  mk.mark(s, G_GRAD_Q);
  launch_adv_q(P, s, AD_Q2 | AD_Q2L | spc);
  mk.mark(s, G_ADV_Q);
  launch_vdif_q(P, s, 1);
  mk.mark(s, G_VDIF_Q);
  if (P.closure) {
    launch_closure(P, s, P.clos_err, h->clos_grid);
    mk.mark(s, G_CLOSURE);
  }
  int ts = (p.temperature_active ? AD_T : 0) | (p.salinity_active ? AD_S : 0);
  if (ts) {
    launch_grad(P, s, 1);
    mk.mark(s, G_GRAD_TS);
    launch_adv_ts(P, s, ts | spc);
    mk.mark(s, G_ADV_TS);
    launch_vdif_ts(P, s, ts);
    mk.mark(s, G_VDIF_TS);
    launch_bcond_ts(P, s, ts);
    mk.mark(s, G_BCOND_TS);
  }
  int fin = FI_KM1 | FI_SHIFT | (p.temperature_active ? FI_T : 0) | (p.salinity_active ? FI_S : 0) |
            (p.barotropic ? 0 : FI_DENS);
  launch_final(P, s, fin);
  mk.mark(s, G_FINAL);
}

}  // namespace

extern "C" {

const char* fvg_build_info(void) {
  return "fvg: B200 mode-split step, sm_100a, FP64, --fmad=false, gather-by-target (no atomics)";
}

const char* fvg_last_error(const fvg_handle* h) { return h ? h->err.c_str() : "null handle"; }

int fvg_create(const fvg_mesh* m, const fvg_params* prm, const fvg_forcing* f, fvg_handle** out) {
  if (!m || !prm || !out) return FVG_ERR_ARG;
  *out = nullptr;
  if (m->m < 3 || m->n < 1 || m->kb < 3 || m->kb > 64) return FVG_ERR_ARG;
  if (prm->isplit < 1 || prm->dte <= 0.0) return FVG_ERR_ARG;
  if (prm->vertical_mixing != 0 || prm->river_ts_setting != 0) return FVG_ERR_UNSUPPORTED;
  if (prm->obc_ts_type < 1 || prm->obc_ts_type > 3) return FVG_ERR_UNSUPPORTED;
  if (f && f->ntide > kMaxTide) return FVG_ERR_UNSUPPORTED;
  if (prm->heating_on && !(prm->rheat >= 0.0 && prm->zeta1 > 0.0 && prm->zeta2 > 0.0)) return FVG_ERR_ARG;
  if (prm->limiter < 0 || prm->limiter > 2) return FVG_ERR_ARG;
  if (prm->ghost_cells < 0 || prm->ghost_cells > 1) return FVG_ERR_ARG;
  fvg_handle* h = new fvg_handle();
  h->prm = *prm;
  Dev& P = h->P;
  const int M = m->m, N = m->n, KB = m->kb;
  P.M = M; P.N = N; P.KB = KB; P.KBM1 = KB - 1; P.KBM2 = KB - 2;
  P.NE = m->ne; P.NCV = m->ncv; P.NCV_I = m->ncv_i;
  P.ms = (int)pad32(M + 1);
  P.ns = (int)pad32(N + 1);
  P.col_bc = 128;
  P.ldcs = 1;
  P.ext_grid = 8;
  P.nsm = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&P.nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      P.nsm = 148;
  }
  P.col_lc = 8;
  P.prec = FVG_PREC_FP64;
  P.nbsn_cols = m->nbsn_cols; P.nbve_cols = m->nbve_cols; P.trie_cols = m->trie_cols;
  P.iobcn = m->iobcn; P.numqbc = m->numqbc;
  P.isplit = prm->isplit;
  P.dte = prm->dte;
  P.dti = prm->dte * (double)prm->isplit;
  P.min_depth = prm->min_depth;
  P.static_ssh_adj = prm->static_ssh_adj;
  P.hprnu = prm->hprnu; P.umol = prm->umol; P.vprnu = prm->vprnu; P.cbcmin = prm->cbcmin;
  P.fact = prm->horizontal_mixing == 0 ? 1.0 : 0.0;
  P.fm1 = prm->horizontal_mixing == 0 ? 0.0 : 1.0;
  P.const1 = std::pow(16.6, .6666667) * 1.00;
  P.vhp1c = std::pow(15.8 * 100.0, 0.6666667);
  P.wetting_drying_on = prm->wetting_drying_on;
  P.river_location = prm->river_location;
  P.obc_ts_type = prm->obc_ts_type;
  h->ntide = (f && m->iobcn > 0) ? f->ntide : 0;
  P.ntide = h->ntide;
  P.obc_elev_on = prm->obc_elevation_forcing_on && h->ntide > 0;
  P.have_wind = f && f->wstress_x && f->wstress_y;
  P.heating_on = prm->heating_on != 0;
  P.limiter = prm->limiter;
  P.baropg_z = prm->baropg_z != 0;
  P.gcy = prm->ghost_cells != 0;
  {
    double hmax = m->h[1];
    for (int i = 2; i <= M; ++i) hmax = std::max(hmax, m->h[i]);
    P.deltz = hmax / (double)(float)600;
  }
  P.rheat = prm->rheat; P.zeta1 = prm->zeta1; P.zeta2 = prm->zeta2;
  P.sl.isplit = prm->isplit;
  P.sl.ntide = h->ntide;
  P.sl.len = 1 + prm->isplit + prm->isplit * 4 * h->ntide;
  for (int j = 0; j < h->ntide; ++j) h->period.push_back(f->period[j]);

  int rc = FVG_OK;
  auto fail = [&](int code) {
    fvg_destroy(h);
    return code;
  };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return FVG_ERR_CUDA;
  }
  const size_t m1 = M + 1, n1 = N + 1, e1 = m->ne + 1, v1 = m->ncv + 1, vi1 = m->ncv_i + 1;
  const size_t o1 = m->iobcn + 1, q1 = m->numqbc + 1;
  const size_t ms = P.ms, ns = P.ns;

  // ---- index validation (FVG_ERR_BOUNDS instead of a device fault) ----
  for (size_t i = 1; i < n1; ++i)
    for (int j = 0; j < 3; ++j) {
      int v = m->nv[j * n1 + i], b = m->nbe[j * n1 + i];
      if (v < 1 || v > M || b < 0 || b > N) { h->err = "NV/NBE out of range"; return fail(FVG_ERR_BOUNDS); }
    }
  for (size_t e = 1; e < e1; ++e) {
    int a = m->iec[e], b = m->iec[e1 + e], j1 = m->ienode[e], j2 = m->ienode[e1 + e];
    if (a < 1 || a > N || b < 0 || b > N || j1 < 1 || j1 > M || j2 < 1 || j2 > M) {
      h->err = "IEC/IENODE out of range";
      return fail(FVG_ERR_BOUNDS);
    }
  }
  for (size_t e = 1; e < v1; ++e) {
    int a = m->niec[e], b = m->niec[v1 + e], c = m->ntrg[e];
    if (a < 1 || a > M || b < 1 || b > M || c < 1 || c > N) { h->err = "NIEC/NTRG out of range"; return fail(FVG_ERR_BOUNDS); }
  }
  for (size_t i = 1; i < m1; ++i) {
    int nt = m->ntsn[i], nv = m->ntve[i];
    if (nt < 2 || nt > m->nbsn_cols || nv < 1 || nv + 1 > m->nbve_cols || nt - 1 > m->trie_cols || nv > m->trie_cols) {
      h->err = "NTSN/NTVE out of range";
      return fail(FVG_ERR_BOUNDS);
    }
    for (int j = 0; j < nt; ++j) {
      int v = m->nbsn[j * m1 + i];
      if (v < 1 || v > M) { h->err = "NBSN out of range"; return fail(FVG_ERR_BOUNDS); }
    }
    for (int j = 0; j < nv; ++j) {
      int v = m->nbve[j * m1 + i];
      if (v < 1 || v > N) { h->err = "NBVE out of range"; return fail(FVG_ERR_BOUNDS); }
    }
  }

  // ---- mesh upload ----
#define UPD(dst, src, n) if ((rc = upload(h, (double**)&P.dst, src, n))) return fail(rc)
#define UPI(dst, src, n) if ((rc = upload(h, (int**)&P.dst, src, n))) return fail(rc)
#define UP3(dst, src, rows, str) if ((rc = upload3(h, (double**)&P.dst, src, rows, KB, str))) return fail(rc)
  UPD(vx, m->vx, m1); UPD(vy, m->vy, m1); UPD(h, m->h, m1); UPD(art1, m->art1, m1); UPD(art2, m->art2, m1);
  UPD(grav_n, m->grav_n, m1); UPD(nn_hvc, m->nn_hvc, m1); UPD(phpn, m->phpn, m1);
  UPI(isonb, m->isonb, m1); UPI(ntsn, m->ntsn, m1); UPI(ntve, m->ntve, m1);
  UPI(nbsn, m->nbsn, m1 * m->nbsn_cols); UPI(nbve, m->nbve, m1 * m->nbve_cols); UPI(nbvt, m->nbvt, m1 * m->nbve_cols);
  UPD(dltxtrie, m->dltxtrie, m1 * m->trie_cols); UPD(dltytrie, m->dltytrie, m1 * m->trie_cols);
  P.trie_n = (int)(m1 * m->trie_cols);
  UPD(dltxecec, m->dltxecec, m1 * m->trie_cols); UPD(dltyecec, m->dltyecec, m1 * m->trie_cols);
  UPD(dltxnec, m->dltxnec, m1 * m->trie_cols); UPD(dltynec, m->dltynec, m1 * m->trie_cols);
  UP3(z, m->z, m1, ms); UP3(zz, m->zz, m1, ms); UP3(dz, m->dz, m1, ms); UP3(dzz, m->dzz, m1, ms);
  UPD(xc, m->xc, n1); UPD(yc, m->yc, n1); UPD(art, m->art, n1); UPD(cor, m->cor, n1);
  UPD(grav_e, m->grav_e, n1); UPD(cc_hvc, m->cc_hvc, n1); UPD(cc_sponge, m->cc_sponge, n1);
  UPD(cc_z0b, m->cc_z0b, n1); UPD(epor, m->epor, n1); UPD(iucp, m->iucp, n1);
  {
    std::vector<double> h1(m->h1, m->h1 + n1);
    h1[0] = h1[1];  // extuv_edge.F:73
    UPD(h1, h1.data(), n1);
  }
  UPI(nv, m->nv, n1 * 3); UPI(nbe, m->nbe, n1 * 3); UPI(isbce, m->isbce, n1);
  {
    std::vector<int> nb4(4 * n1, 0);
    for (size_t c = 0; c < n1; ++c)
      for (int j = 0; j < 3; ++j) nb4[4 * c + j] = m->nbe[j * n1 + c];
    UPI(nbe4, nb4.data(), nb4.size());
  }
  UPD(a1u, m->a1u, n1 * 4); UPD(a2u, m->a2u, n1 * 4); UPD(awx, m->awx, n1 * 3); UPD(awy, m->awy, n1 * 3);
  UP3(z1, m->z1, n1, ns); UP3(zz1, m->zz1, n1, ns); UP3(dz1, m->dz1, n1, ns); UP3(dzz1, m->dzz1, n1, ns);
  UPI(iec, m->iec, e1 * 2); UPI(ienode, m->ienode, e1 * 2); UPI(isbc, m->isbc, e1);
  UPD(xijc, m->xijc, e1); UPD(yijc, m->yijc, e1); UPD(dltxc, m->dltxc, e1); UPD(dltyc, m->dltyc, e1);
  UPI(niec, m->niec, v1 * 2); UPI(ntrg, m->ntrg, v1); UPD(dltxe, m->dltxe, v1); UPD(dltye, m->dltye, v1);
  UPD(dltxncve, m->dltxncve, vi1 * 2); UPD(dltyncve, m->dltyncve, vi1 * 2);
  // Loop-invariant transcendental factors, formed on the host with the C library so they
  // equal the values the reference recomputes each call.
  {
    std::vector<double> sa(n1), ca(n1), cs(m1), ss(m1);
    for (size_t i = 0; i < n1; ++i) { sa[i] = std::sin(m->alpha[i]); ca[i] = std::cos(m->alpha[i]); }
    for (size_t i = 0; i < m1; ++i) { cs[i] = std::cos(m->sita_gd[i]); ss[i] = std::sin(m->sita_gd[i]); }
    UPD(sin_alpha, sa.data(), n1); UPD(cos_alpha, ca.data(), n1);
    UPD(cos_sita, cs.data(), m1); UPD(sin_sita, ss.data(), m1);
  }

  // ---- gather lists ----
  {
    std::vector<std::vector<int>> nl(m1), cl(n1);
    for (int he = 1; he <= m->ncv; ++he) {
      nl[m->niec[he]].push_back(he * 2 + 0);
      nl[m->niec[v1 + he]].push_back(he * 2 + 1);
    }
    for (int e = 1; e <= m->ne; ++e) {
      cl[m->iec[e]].push_back(e * 2 + 0);
      int b = m->iec[e1 + e];
      if (b > 0) cl[b].push_back(e * 2 + 1);
    }
    std::vector<int> ptr, ent;
    build_csr(nl, ptr, ent);
    UPI(node_he_ptr, ptr.data(), ptr.size()); UPI(node_he, ent.data(), ent.size());
    std::vector<int> ce(3 * n1, 0);
    for (size_t i = 1; i < n1; ++i) {
      if (cl[i].size() != 3) { h->err = "cell without exactly three edges"; return fail(FVG_ERR_BOUNDS); }
      for (int s = 0; s < 3; ++s) ce[3 * i + s] = cl[i][s];
    }
    UPI(cell_edge, ce.data(), ce.size());
    // Slot table of the edge loops: slot s of cell i at s*(N+1) + i, the edges in the
    // order of cell_edge.  code = edge*4 + ISBC*2 + side; offsets XIJC-XC of both ends.
    {
      const size_t S3 = 3 * n1;
      std::vector<int> cc(S3, 0), ca(S3, 0), cb(S3, 0), cj1(S3, 0), cj2(S3, 0);
      std::vector<double> xa(S3, 0.0), ya(S3, 0.0), xb(S3, 0.0), yb(S3, 0.0), dx(S3, 0.0), dy(S3, 0.0);
      for (size_t i = 1; i < n1; ++i)
        for (int sl = 0; sl < 3; ++sl) {
          const int code = cl[i][sl], e = code >> 1, side = code & 1;
          const size_t q = (size_t)sl * n1 + i;
          const int ia = m->iec[e], ib = m->iec[e1 + e];
          cc[q] = e * 4 + (m->isbc[e] != 0 ? 2 : 0) + side;
          ca[q] = ia;
          cb[q] = ib;
          cj1[q] = m->ienode[e];
          cj2[q] = m->ienode[e1 + e];
          xa[q] = m->xijc[e] - m->xc[ia];
          ya[q] = m->yijc[e] - m->yc[ia];
          xb[q] = m->xijc[e] - m->xc[ib];
          yb[q] = m->yijc[e] - m->yc[ib];
          dx[q] = m->dltxc[e];
          dy[q] = m->dltyc[e];
        }
      UPI(ce_code, cc.data(), S3); UPI(ce_ia, ca.data(), S3); UPI(ce_ib, cb.data(), S3);
      std::vector<int> c4(4 * S3);
      for (size_t q = 0; q < S3; ++q) {
        c4[4 * q] = cc[q];
        c4[4 * q + 1] = ca[q];
        c4[4 * q + 2] = cb[q];
        c4[4 * q + 3] = cj1[q];
      }
      UPI(ce_i4, c4.data(), c4.size());
      UPI(ce_j1, cj1.data(), S3); UPI(ce_j2, cj2.data(), S3);
      UPD(ce_xoa, xa.data(), S3); UPD(ce_yoa, ya.data(), S3); UPD(ce_xob, xb.data(), S3);
      UPD(ce_yob, yb.data(), S3); UPD(ce_dx, dx.data(), S3); UPD(ce_dy, dy.data(), S3);
    }
    // cell tiles of the staged momentum flux kernels
    {
      TileBuild tb;
      build_tiles(N, m->ne, m->xc, m->yc, m->iec, m->ienode, m->isbc, cl, tb);
      if (tb.cap_edges >= (1 << 16) || tb.cap_cells >= (1 << 16)) {
        h->err = "tile builder: a tile with too many edges";
        return fail(FVG_ERR_BOUNDS);
      }
      P.tl.n = (int)tb.nc.size();
      P.tl.cap_cells = tb.cap_cells;
      P.tl.cap_edges = tb.cap_edges;
      UPI(tl.ptr, tb.ptr.data(), tb.ptr.size());
      UPI(tl.nc, tb.nc.data(), tb.nc.size());
      UPI(tl.eptr, tb.eptr.data(), tb.eptr.size());
      UPI(tl.cells, tb.cells.data(), tb.cells.size());
      UPI(tl.edges, tb.edges.data(), tb.edges.size());
      UPI(tl.slots, tb.slots.data(), tb.slots.size());
      P.staged = 1;
      if (staged_setup() || fvg_f32::staged_setup()) {
        h->err = "cannot configure the staged momentum kernels";
        return fail(FVG_ERR_CUDA);
      }
    }
    std::vector<std::vector<int>> ch(n1);
    for (int he = 1; he <= m->ncv; ++he) ch[m->ntrg[he]].push_back(he);
    std::vector<int> chv(3 * n1, 0);
    for (size_t i = 1; i < n1; ++i) {
      if (ch[i].size() != 3) { h->err = "cell without exactly three half-edges"; return fail(FVG_ERR_BOUNDS); }
      for (int s2 = 0; s2 < 3; ++s2) {
        int he = ch[i][s2];
        int a = m->niec[he], b = m->niec[v1 + he];
        bool ok_a = false, ok_b = false;
        for (int j = 0; j < 3; ++j) {
          ok_a |= m->nv[j * n1 + i] == a;
          ok_b |= m->nv[j * n1 + i] == b;
        }
        if (!ok_a || !ok_b) { h->err = "half-edge nodes not on its cell"; return fail(FVG_ERR_BOUNDS); }
        chv[3 * i + s2] = he;
      }
    }
    UPI(cell_he, chv.data(), chv.size());
    // Half-edge positions pos = slot*ns + cell; the node lists over positions, entry j of
    // node i at j*ms + i, code = pos*2 + side, ascending half-edge id; the metrics by position
    std::vector<int> slot(v1, 0);
    std::vector<double> hg(18 * ns, 0.0);
    for (size_t i = 1; i < n1; ++i)
      for (int s2 = 0; s2 < 3; ++s2) {
        const int he = chv[3 * i + s2];
        slot[he] = s2;
        const size_t pos = (size_t)s2 * ns + i, pl = 3 * ns;
        hg[pos] = m->dltxe[he];
        hg[pl + pos] = m->dltye[he];
        hg[2 * pl + pos] = m->dltxncve[he];
        hg[3 * pl + pos] = m->dltyncve[he];
        hg[4 * pl + pos] = m->dltxncve[vi1 + he];
        hg[5 * pl + pos] = m->dltyncve[vi1 + he];
      }
    UPD(hg, hg.data(), hg.size());
    std::vector<std::vector<int>> vl(m1);
    for (int he = 1; he <= m->ncv; ++he) {
      const long pos = (long)slot[he] * (long)ns + m->ntrg[he];
      vl[m->niec[he]].push_back((int)(pos * 2 + 0));
      vl[m->niec[v1 + he]].push_back((int)(pos * 2 + 1));
    }
    size_t w = 1;
    for (auto& l : vl) w = std::max(w, l.size());
    std::vector<int> ell(w * ms, 0);
    for (size_t i = 0; i < m1; ++i)
      for (size_t j = 0; j < vl[i].size(); ++j) ell[j * ms + i] = vl[i][j];
    UPI(node_vpos_ell, ell.data(), ell.size());
  }
  // open boundary
  {
    std::vector<int> node_obc(m1, 0), kind(o1, 0);
    std::vector<std::vector<int>> co(n1);
    for (int ob = 1; ob <= m->iobcn; ++ob) {
      int nd = m->i_obc_n[ob];
      if (nd < 1 || nd > M) { h->err = "I_OBC_N out of range"; return fail(FVG_ERR_BOUNDS); }
      node_obc[nd] = ob;
      int t = m->type_obc[ob];
      if (t == 1 || t == 2) kind[ob] = 1;
      else if (t == 3 || t == 4) kind[ob] = 2;
      else { h->err = "open-boundary TYPE_OBC 5-10 not supported"; return fail(FVG_ERR_UNSUPPORTED); }
      int na = m->nadjc_obc[ob];
      for (int s = 0; s < na && s < 2; ++s) {
        int c = m->adjc_obc[s * o1 + ob];
        if (c < 1 || c > N) { h->err = "ADJC_OBC out of range"; return fail(FVG_ERR_BOUNDS); }
        co[c].push_back(ob * 2 + s);
      }
      int nx = m->next_obc[ob];
      if (nx < 1 || nx > M) { h->err = "NEXT_OBC out of range"; return fail(FVG_ERR_BOUNDS); }
    }
    std::vector<int> ptr, ent;
    build_csr(co, ptr, ent);
    UPI(node_obc, node_obc.data(), m1); UPI(obc_kind, kind.data(), o1);
    UPI(cell_obc_ptr, ptr.data(), ptr.size()); UPI(cell_obc, ent.data(), ent.size());
    UPI(i_obc_n, m->i_obc_n, o1); UPI(next_obc, m->next_obc, o1);
    UPD(dltn_obc, m->dltn_obc, o1); UPD(fluxf_obc, m->fluxf_obc, o1 * 2);
    size_t nt = h->ntide;
    std::vector<double> apt(o1 * (nt ? nt : 1), 0.0), ph(o1 * (nt ? nt : 1), 0.0), em(o1, 0.0);
    if (nt) {
      for (size_t q = 0; q < o1 * nt; ++q) { apt[q] = f->apt[q]; ph[q] = f->phai[q] * kPI2 / 360.0; }
      for (size_t q = 0; q < o1; ++q) em[q] = f->emean ? f->emean[q] : 0.0;
    }
    UPD(apt, apt.data(), apt.size()); UPD(phai_rad, ph.data(), ph.size()); UPD(emean, em.data(), o1);
  }
  // rivers
  {
    const int nq = m->numqbc;
    std::vector<std::vector<int>> nr(m1), cr(n1);
    std::vector<int> bcriv(n1, 0), skip(m1, 0);
    for (int ob = 1; ob <= m->iobcn; ++ob) skip[m->i_obc_n[ob]] = 1;
    for (int j = 1; j <= nq; ++j) {
      if (prm->river_location == 0) {
        int nd = m->inodeq[j];
        if (nd < 1 || nd > M) { h->err = "INODEQ out of range"; return fail(FVG_ERR_BOUNDS); }
        nr[nd].push_back(j * 2);
        skip[nd] = 1;
        int i1 = m->nbve[nd], i2 = m->nbve[(m->ntve[nd] - 1) * m1 + nd];
        cr[i1].push_back(j * 2);
        cr[i2].push_back(j * 2 + 1);
      } else {
        int c = m->icellq[j], a = m->n_icellq[j], b = m->n_icellq[q1 + j];
        if (c < 1 || c > N || a < 1 || a > M || b < 1 || b > M) { h->err = "river cell out of range"; return fail(FVG_ERR_BOUNDS); }
        nr[a].push_back(j * 2);
        nr[b].push_back(j * 2 + 1);
        skip[a] = 1;
        skip[b] = 1;
        cr[c].push_back(j * 2);
      }
    }
    for (size_t i = 1; i < n1; ++i)
      for (int j = 1; j <= nq && !bcriv[i]; ++j) {
        bool hit;
        if (prm->river_location == 0) {
          int i1 = m->inodeq[j];
          hit = (int)i == m->nbve[i1] || (int)i == m->nbve[(m->ntve[i1] - 1) * m1 + i1];
        } else {
          hit = (int)i == m->icellq[j];
        }
        if (hit) bcriv[i] = j;
      }
    std::vector<int> ptr, ent;
    build_csr(nr, ptr, ent);
    UPI(node_riv_ptr, ptr.data(), ptr.size()); UPI(node_riv, ent.data(), ent.size());
    build_csr(cr, ptr, ent);
    UPI(cell_riv_ptr, ptr.data(), ptr.size()); UPI(cell_riv, ent.data(), ent.size());
    UPI(cell_bcriv, bcriv.data(), n1); UPI(riv_skip, skip.data(), m1);
    UPI(inodeq, m->inodeq, q1); UPI(icellq, m->icellq, q1); UPI(n_icellq, m->n_icellq, q1 * 2);
    UPD(rdisq, m->rdisq, q1 * 2); UPD(qarea, m->qarea, q1); UPD(vqdist, m->vqdist, q1 * (KB - 1));
    std::vector<double> sq(q1), cq(q1);
    for (size_t j = 0; j < q1; ++j) { sq[j] = std::sin(m->angleq[j]); cq[j] = std::cos(m->angleq[j]); }
    UPD(sin_angleq, sq.data(), q1); UPD(cos_angleq, cq.data(), q1);
    UPD(qdis0, f ? f->qdis : nullptr, q1); UPD(tdis, f ? f->tdis : nullptr, q1); UPD(sdis, f ? f->sdis : nullptr, q1);
  }
  UPD(wsx, P.have_wind ? f->wstress_x : nullptr, n1);
  UPD(wsy, P.have_wind ? f->wstress_y : nullptr, n1);
  UPD(swrad_w, P.heating_on && f ? f->swrad : nullptr, m1);
  UPD(wtsurf_w, P.heating_on && f ? f->wtsurf : nullptr, m1);

  // ---- state ----
  auto reg = [&](const char* name, double** p, size_t rows, int layers, size_t stride) -> int {
    int r = dalloc(h, p, layers == 1 ? rows : stride * layers);
    if (r) return r;
    h->fields[name] = FieldDesc{*p, (int64_t)rows, layers, (int64_t)(layers == 1 ? rows : stride), false};
    return FVG_OK;
  };
  auto regi = [&](const char* name, int** p, size_t rows) -> int {
    int r = dalloc(h, p, rows);
    if (r) return r;
    std::vector<int> ones(rows, 1);
    cudaMemcpy(*p, ones.data(), rows * sizeof(int), cudaMemcpyHostToDevice);
    h->fields[name] = FieldDesc{*p, (int64_t)rows, 1, (int64_t)rows, true};
    return FVG_OK;
  };
#define RN2(x) if ((rc = reg(#x, &P.x, m1, 1, 0))) return fail(rc)
#define RN3(x) if ((rc = reg(#x, &P.x, m1, KB, ms))) return fail(rc)
#define RC2(x) if ((rc = reg(#x, &P.x, n1, 1, 0))) return fail(rc)
#define RC3(x) if ((rc = reg(#x, &P.x, n1, KB, ns))) return fail(rc)
  RN2(el); RN2(elf); RN2(elrk); RN2(et); RN2(d); RN2(dt); RN2(dtfa); RN2(egf); RN2(wubot_n); RN2(wvbot_n); RN2(taubm_n);
  RN2(pfpxb_t); RN2(pfpyb_t); RN2(ah_bottom_t); RN2(pfpxb_s); RN2(pfpyb_s); RN2(ah_bottom_s);
  RN3(t1); RN3(s1); RN3(tf1); RN3(sf1); RN3(rho1); RN3(tmean1); RN3(smean1); RN3(rmean1);
  RN3(q2); RN3(q2l); RN3(q2f); RN3(q2lf); RN3(l); RN3(km); RN3(kh); RN3(kq); RN3(wts); RN3(viscofh);
  RC2(el1); RC2(elf1); RC2(elrk1); RC2(et1); RC2(d1); RC2(dt1); RC2(ua); RC2(va); RC2(uaf); RC2(vaf);
  RC2(uark); RC2(vark); RC2(uard); RC2(vard); RC2(adx2d); RC2(ady2d); RC2(drx2d); RC2(dry2d);
  RC2(advua); RC2(advva); RC2(pstx); RC2(psty); RC2(wubot); RC2(wvbot); RC2(cbc); RC2(tps); RC2(fluxobn);
  RC2(taubm); RC2(wusurf); RC2(wvsurf);
  RC3(u); RC3(v); RC3(uf); RC3(vf); RC3(w); RC3(ww); RC3(advx); RC3(advy); RC3(drhox); RC3(drhoy);
  RC3(rho); RC3(t); RC3(s); RC3(rmean); RC3(km1); RC3(viscofm);
  if ((rc = regi("iswetn", &P.iswetn, m1))) return fail(rc);
  if ((rc = regi("iswetnt", &P.iswetnt, m1))) return fail(rc);
  if ((rc = regi("iswetc", &P.iswetc, n1))) return fail(rc);
  if ((rc = regi("iswetct", &P.iswetct, n1))) return fail(rc);
  if ((rc = regi("iswetce", &P.iswetce, n1))) return fail(rc);
  if ((rc = reg("xflux_obcn", &P.xflux_obcn, o1, 1, 0))) return fail(rc);
  if ((rc = reg("uard_obcn", &P.uard_obcn, o1, 1, 0))) return fail(rc);
  if ((rc = reg("xflux_obc_t", &P.xflux_obc_t, o1, KB - 1, o1))) return fail(rc);
  if ((rc = reg("xflux_obc_s", &P.xflux_obc_s, o1, KB - 1, o1))) return fail(rc);
  if ((rc = reg("qdis", &P.qdis, q1, 1, 0))) return fail(rc);
  h->fields["h1"] = FieldDesc{P.h1, (int64_t)n1, 1, (int64_t)n1, false};
  // surface stress before the RAMP*0.001 scaling: a per-step forcing input
  h->fields["wstress_x"] = FieldDesc{(void*)P.wsx, (int64_t)n1, 1, (int64_t)n1, false};
  h->fields["wstress_y"] = FieldDesc{(void*)P.wsy, (int64_t)n1, 1, (int64_t)n1, false};
  h->fields["swrad_watts"] = FieldDesc{(void*)P.swrad_w, (int64_t)m1, 1, (int64_t)m1, false};
  h->fields["wtsurf_watts"] = FieldDesc{(void*)P.wtsurf_w, (int64_t)m1, 1, (int64_t)m1, false};
  if ((rc = dalloc(h, &P.scr_xflux, ms * KB))) return fail(rc);
  for (int t = 0; t < 2; ++t)
    for (int g = 0; g < 6; ++g) {
      if ((rc = dalloc(h, &P.gq[t][g], ms * KB))) return fail(rc);
      if ((rc = dalloc(h, &P.gt[t][g], ms * KB))) return fail(rc);
    }
  if ((rc = dalloc(h, &P.budget, 3 + 3 * 148))) return fail(rc);
  for (double** pp : {&P.vq_prod, &P.vq_gh, &P.vq_dtef, &P.vq_dtefl})
    if ((rc = dalloc(h, pp, ms * KB))) return fail(rc);
  if ((rc = dalloc(h, &P.vq_ut, ms))) return fail(rc);
  P.ncvs = (int)(3 * ns);  // half-edge arrays by position, pos = slot*ns + cell
  for (int q = 0; q < 4; ++q) {
    if ((rc = dalloc(h, &P.g2d[q], n1))) return fail(rc);
  }
  if (P.baropg_z && (rc = dalloc(h, &P.rhoz, (size_t)P.ms * 600))) return fail(rc);
  if (P.gcy) {
    // GHOSTUV2/3's ATAN2, COS, SIN of the edge opposite node j, once on the host
    std::vector<double> gc(3 * n1, 1.0), gs(3 * n1, 0.0);
    for (size_t i = 1; i < n1; ++i)
      for (int j = 1; j <= 3; ++j) {
        const int J1 = j + 1 - ((j + 1) / 4) * 3, J2 = j + 2 - ((j + 2) / 4) * 3;
        const int na = m->nv[(size_t)(J1 - 1) * n1 + i], nb = m->nv[(size_t)(J2 - 1) * n1 + i];
        const double a = std::atan2(m->vy[na] - m->vy[nb], m->vx[na] - m->vx[nb]);
        gc[(size_t)(j - 1) * n1 + i] = std::cos(a);
        gs[(size_t)(j - 1) * n1 + i] = std::sin(a);
      }
    UPD(gh_cos, gc.data(), 3 * n1);
    UPD(gh_sin, gs.data(), 3 * n1);
  }
  if (P.limiter) {
    std::vector<double> ones(std::max(n1, (size_t)P.ns * KB), 1.0);
    for (int q = 0; q < 2; ++q) {
      if ((rc = upload(h, &P.alfa2[q], ones.data(), n1))) return fail(rc);
      if ((rc = upload(h, &P.alfa3[q], ones.data(), (size_t)P.ns * KB))) return fail(rc);
    }
  }
  if ((rc = dalloc(h, &P.exf2d, 3 * ns))) return fail(rc);
  for (int q = 0; q < 4; ++q)
    if ((rc = dalloc(h, &P.g3[q], ns * KB))) return fail(rc);
  if ((rc = dalloc(h, (double**)&P.ex2, (size_t)P.ncvs * KB * 2))) return fail(rc);
  P.he_vflux = (double*)P.ex2;

  // ---- schedule ----
  h->sched_cap = 256;
  if ((rc = dalloc(h, &h->d_sched, (size_t)(h->sched_cap + 1) * P.sl.len))) return fail(rc);
  if (cudaMallocHost(&h->h_sched, (size_t)(h->sched_cap + 1) * P.sl.len * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&h->h_ctl, 4 * sizeof(int)) != cudaSuccess) {
    h->err = "cudaMallocHost failed";
    return fail(FVG_ERR_NOMEM);
  }
  {
    int* ctl;
    if ((rc = dalloc(h, &ctl, 4))) return fail(rc);
    P.ctl = ctl;
  }
  P.sched = h->d_sched;
  if (cudaDeviceSynchronize() != cudaSuccess) {
    h->err = "device synchronize failed after create";
    return fail(FVG_ERR_CUDA);
  }
  *out = h;
  return FVG_OK;
}

void fvg_destroy(fvg_handle* h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  for (void* p : h->allocs) cudaFree(p);
  if (h->h_sched) cudaFreeHost(h->h_sched);
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int64_t fvg_field_size(const fvg_handle* h, const char* name) {
  if (!h || !name) return -1;
  auto it = h->fields.find(name);
  if (it == h->fields.end()) return -1;
  return it->second.rows * it->second.layers;
}

static int field_copy(fvg_handle* h, const char* name, void* host, int64_t count, bool to_dev, bool is_int) {
  if (!h || !name || !host) return FVG_ERR_ARG;
  auto it = h->fields.find(name);
  if (it == h->fields.end()) { h->err = std::string("unknown field ") + name; return FVG_ERR_ARG; }
  const FieldDesc& fd = it->second;
  if (fd.is_int != is_int || count != fd.rows * fd.layers) {
    h->err = std::string("size/type mismatch for field ") + name;
    return FVG_ERR_ARG;
  }
  size_t es = is_int ? sizeof(int32_t) : sizeof(double);
  CK(cudaStreamSynchronize(h->stream));
  if (fd.layers == 1) {
    CK(cudaMemcpy(to_dev ? fd.d : host, to_dev ? host : fd.d, fd.rows * es,
                  to_dev ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost));
  } else if (to_dev) {
    CK(cudaMemcpy2D(fd.d, fd.stride * es, host, fd.rows * es, fd.rows * es, fd.layers, cudaMemcpyHostToDevice));
  } else {
    CK(cudaMemcpy2D(host, fd.rows * es, fd.d, fd.stride * es, fd.rows * es, fd.layers, cudaMemcpyDeviceToHost));
  }
  return FVG_OK;
}

int fvg_set_field(fvg_handle* h, const char* name, const double* src, int64_t count) {
  return field_copy(h, name, (void*)src, count, true, false);
}
int fvg_get_field(fvg_handle* h, const char* name, double* dst, int64_t count) {
  return field_copy(h, name, dst, count, false, false);
}
int fvg_set_ifield(fvg_handle* h, const char* name, const int32_t* src, int64_t count) {
  return field_copy(h, name, (void*)src, count, true, true);
}
int fvg_get_ifield(fvg_handle* h, const char* name, int32_t* dst, int64_t count) {
  return field_copy(h, name, dst, count, false, true);
}

int fvg_set_clock(fvg_handle* h, int32_t iint, double ext_time) {
  if (!h) return FVG_ERR_ARG;
  h->iint = iint;
  h->ext_time = ext_time;
  return FVG_OK;
}
int fvg_get_clock(const fvg_handle* h, int32_t* iint, double* ext_time) {
  if (!h || !iint || !ext_time) return FVG_ERR_ARG;
  *iint = h->iint;
  *ext_time = h->ext_time;
  return FVG_OK;
}
int fvg_set_ramp(fvg_handle* h, double ramp) {
  if (!h) return FVG_ERR_ARG;
  h->ramp = ramp;
  return FVG_OK;
}

// mode 0: graph replay (or plain launches when graphs are off); mode 1: plain launches
// with events between kernel groups, accumulated into group_ms; total_ms gets the device
// time of all steps measured with events on the handle's stream.
// Schedule rows of the next c internal steps (RAMP, tidal phase arguments) and the device
// slot counter, on the handle's stream; the stream must be idle.
static int prep_chunk(fvg_handle* h, int c) {
  const int len = h->P.sl.len;
  int32_t iint = h->iint;
  double t = h->ext_time;
  for (int s = 0; s < c; ++s) {
    fill_sched_row(h, h->h_sched + (size_t)s * len, iint + 1, t);
    iint += 1;
    for (int iext = 1; iext <= h->prm.isplit; ++iext) t = t + h->prm.dte;
  }
  CK(cudaMemcpyAsync(h->d_sched, h->h_sched, (size_t)c * len * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  h->h_ctl[0] = -1;
  CK(cudaMemcpyAsync(h->P.ctl, h->h_ctl, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  return FVG_OK;
}

// Advance the host clock by c internal steps exactly as the reference accumulates ExtTime.
static void finish_chunk(fvg_handle* h, int c) {
  for (int s = 0; s < c; ++s) {
    h->iint += 1;
    for (int iext = 1; iext <= h->prm.isplit; ++iext) h->ext_time = h->ext_time + h->prm.dte;
  }
  h->ramp = h->prm.iramp != 0 ? std::tanh((double)h->iint / (double)h->prm.iramp) : 1.0;
}

// The learned closure's error word, read after the steps have run: a bounded wait of the
// tensor-core kernel that ran out (its rows then took MY2.5's values) fails the call.
static int closure_check(fvg_handle* h) {
  if (!h->P.closure || !h->P.clos_err) return FVG_OK;
  int e = 0;
  CK(cudaMemcpy(&e, h->P.clos_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e == 0) return FVG_OK;
  h->err = "learned closure: a bounded tensor-core wait ran out (error word " + std::to_string(e) +
           "); the affected rows took MY2.5's values";
  return FVG_ERR_TIMEOUT;
}

static int run_steps(fvg_handle* h, int32_t nsteps, int mode, double* group_ms, double* total_ms) {
  if (!h || nsteps < 0) return FVG_ERR_ARG;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (total_ms) {
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
  }
  double total = 0.0;
  int done = 0;
  while (done < nsteps) {
    int c = std::min(h->sched_cap, nsteps - done);
    CK(cudaStreamSynchronize(h->stream));
    { int rc = prep_chunk(h, c); if (rc) return rc; }
    if (total_ms) CK(cudaEventRecord(t0, h->stream));
    std::vector<cudaEvent_t> ev;
    std::vector<int> grp;
    for (int s = 0; s < c; ++s) {
      if (mode == 1) {
        Marker mk;
        mk.ev = &ev;
        mk.grp = &grp;
        enqueue_internal_step(h, h->stream, mk);
      } else if (h->use_graph) {
        if (!h->gexec) {
          CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
          enqueue_internal_step(h, h->stream);
          cudaError_t e = cudaStreamEndCapture(h->stream, &h->graph);
          if (e != cudaSuccess) { h->err = std::string("graph capture: ") + cudaGetErrorString(e); return FVG_ERR_CUDA; }
          CK(cudaGraphInstantiate(&h->gexec, h->graph, 0));
        }
        CK(cudaGraphLaunch(h->gexec, h->stream));
      } else {
        enqueue_internal_step(h, h->stream);
      }
    }
    CK(cudaGetLastError());
    if (total_ms) {
      CK(cudaEventRecord(t1, h->stream));
      CK(cudaEventSynchronize(t1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, t0, t1));
      total += ms;
    }
    if (mode == 1) {
      CK(cudaStreamSynchronize(h->stream));
      for (size_t q = 1; q < ev.size(); ++q) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[q - 1], ev[q]);
        if (grp[q] >= 0 && group_ms) group_ms[grp[q]] += ms;
      }
      for (auto e : ev) cudaEventDestroy(e);
    }
    finish_chunk(h, c);
    done += c;
  }
  CK(cudaStreamSynchronize(h->stream));
  if (total_ms) {
    *total_ms = total;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
  }
  return closure_check(h);
}

int fvg_run(fvg_handle* h, int32_t nsteps) { return run_steps(h, nsteps, 0, nullptr, nullptr); }

int fvg_internal_step(fvg_handle* h) { return fvg_run(h, 1); }

int fvg_time_steps(fvg_handle* h, int32_t nsteps, double* ms) {
  if (!ms) return FVG_ERR_ARG;
  return run_steps(h, nsteps, 0, nullptr, ms);
}

int32_t fvg_profile_groups(void) { return G_COUNT; }

int32_t fvg_kernels_per_step(const fvg_handle* h) {
  if (!h) return -1;
  const fvg_params& p = h->prm;
  int n = 1 + 1 + 2 + 2 + 2;                                // begin, cell_pre, grad3+adv3d, baropg+prep, int advave+reset
  n += p.isplit * 4 * (2 + (p.wetting_drying_on ? 1 : 0)) + 1; // RK stages, closing update
  if (p.limiter) n += p.isplit * 4 + 1 + 2;                  // slope limiters: stages, ADVAVE, 3-D
  if (p.baropg_z && !p.barotropic) n += 2;                   // PHY_BAROPG's two kernels
  n += 1 + 1 + 1 + 1 + 2 + 1;                              // adjust2, vertvl x2, w/viscofh, grad3+adv_uv, vdif_uv
  n += 7;                                                  // grad_q, adv_q (2 phases), vdif_q (4 passes)
  if (h->P.closure) n += 3;                                // learned closure (compaction x2, network)
  if (p.temperature_active || p.salinity_active)           // grad_ts, adv_ts (2 phases), vdif_ts,
    n += 5 + (h->P.iobcn > 0 ? 1 : 0);                     // bcond_ts (rivers, open boundary)
  n += 1;                                                  // final
  return n;
}
const char* fvg_profile_group_name(int32_t g) { return (g >= 0 && g < G_COUNT) ? kGroupNames[g] : ""; }

int fvg_profile(fvg_handle* h, int32_t nsteps, double* group_ms, double* total_ms) {
  if (!group_ms) return FVG_ERR_ARG;
  for (int g = 0; g < G_COUNT; ++g) group_ms[g] = 0.0;
  return run_steps(h, nsteps, 1, group_ms, total_ms);
}

int fvg_sync(fvg_handle* h) {
  if (!h) return FVG_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  return FVG_OK;
}

int fvg_use_graph(fvg_handle* h, int32_t on) {
  if (!h) return FVG_ERR_ARG;
  h->use_graph = on != 0;
  return FVG_OK;
}

int fvg_external_step(fvg_handle* h, int32_t iext) {
  if (!h || iext < 1 || iext > h->prm.isplit) return FVG_ERR_ARG;
  return fvg_run_routine(h, FVG_R_EXTERNAL_STEP, iext);
}

int fvg_set_forcing(fvg_handle* h, const fvg_forcing* f) {
  if (!h || !f) return FVG_ERR_ARG;
  Dev& P = h->P;
  if (f->ntide != h->ntide) { h->err = "fvg_set_forcing: ntide differs from fvg_create"; return FVG_ERR_ARG; }
  const bool wind = f->wstress_x && f->wstress_y;
  if (wind && !P.have_wind) { h->err = "fvg_set_forcing: the model was created without wind stress"; return FVG_ERR_UNSUPPORTED; }
  CK(cudaStreamSynchronize(h->stream));
  const size_t o1 = (size_t)P.iobcn + 1, q1 = (size_t)P.numqbc + 1, n1 = (size_t)P.N + 1;
  const size_t nt = h->ntide;
  if (nt) {
    std::vector<double> apt(o1 * nt), ph(o1 * nt), em(o1, 0.0);
    for (size_t q = 0; q < o1 * nt; ++q) { apt[q] = f->apt[q]; ph[q] = f->phai[q] * kPI2 / 360.0; }
    for (size_t q = 0; q < o1; ++q) em[q] = f->emean ? f->emean[q] : 0.0;
    for (size_t j = 0; j < nt; ++j) h->period[j] = f->period[j];
    CK(cudaMemcpy((void*)P.apt, apt.data(), apt.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void*)P.phai_rad, ph.data(), ph.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void*)P.emean, em.data(), em.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (P.numqbc > 0) {
    if (f->qdis) CK(cudaMemcpy((void*)P.qdis0, f->qdis, q1 * sizeof(double), cudaMemcpyHostToDevice));
    if (f->tdis) CK(cudaMemcpy((void*)P.tdis, f->tdis, q1 * sizeof(double), cudaMemcpyHostToDevice));
    if (f->sdis) CK(cudaMemcpy((void*)P.sdis, f->sdis, q1 * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (wind) {
    CK(cudaMemcpy((void*)P.wsx, f->wstress_x, n1 * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void*)P.wsy, f->wstress_y, n1 * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (P.heating_on) {
    const size_t m1 = (size_t)P.M + 1;
    if (f->swrad) CK(cudaMemcpy((void*)P.swrad_w, f->swrad, m1 * sizeof(double), cudaMemcpyHostToDevice));
    if (f->wtsurf) CK(cudaMemcpy((void*)P.wtsurf_w, f->wtsurf, m1 * sizeof(double), cudaMemcpyHostToDevice));
  }
  return FVG_OK;
}

int fvg_set_precision(fvg_handle* h, int32_t mode) {
  if (!h) return FVG_ERR_ARG;
  if (mode != FVG_PREC_FP64 && mode != FVG_PREC_FP32_FLUX) { h->err = "unknown precision mode"; return FVG_ERR_ARG; }
  Dev& P = h->P;
  CK(cudaStreamSynchronize(h->stream));
  if (mode == FVG_PREC_FP32_FLUX && !P.f.ex2) {
    int rc;
    const size_t ms = P.ms, ns = P.ns, KB = P.KB, n1 = P.N + 1, e1 = P.NE + 1;
    F32& f = P.f;
    auto fail = [&](int r) { return r; };
    if ((rc = dalloc(h, (float**)&f.g34, 4 * ns * KB))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.g2d4, 4 * n1))) return fail(rc);
    if (P.limiter) {
      std::vector<float> ones(std::max(n1, ns * KB), 1.0f);
      for (int q = 0; q < 2; ++q) {
        if ((rc = dalloc(h, &f.alfa2[q], n1))) return fail(rc);
        if ((rc = dalloc(h, &f.alfa3[q], ns * KB))) return fail(rc);
        CK(cudaMemcpy(f.alfa2[q], ones.data(), n1 * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(f.alfa3[q], ones.data(), ns * KB * sizeof(float), cudaMemcpyHostToDevice));
      }
    }
    if ((rc = dalloc(h, &f.npk, ms * KB * 16))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.ex2, (size_t)P.ncvs * KB * 2))) return fail(rc);
    if ((rc = dalloc(h, &f.xo, 2 * e1))) return fail(rc);
    if ((rc = dalloc(h, &f.yo, 2 * e1))) return fail(rc);
    if ((rc = dalloc(h, &f.dltxc, e1))) return fail(rc);
    if ((rc = dalloc(h, &f.dltyc, e1))) return fail(rc);
    if ((rc = dalloc(h, &f.art, n1))) return fail(rc);
    if ((rc = dalloc(h, &f.cc_hvc, n1))) return fail(rc);
    if ((rc = dalloc(h, &f.a1u, 4 * n1))) return fail(rc);
    if ((rc = dalloc(h, &f.a2u, 4 * n1))) return fail(rc);
    for (float** pp : {&f.ce_xoa, &f.ce_yoa, &f.ce_xob, &f.ce_yob, &f.ce_dx, &f.ce_dy})
      if ((rc = dalloc(h, pp, 3 * n1))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.ce_geo, 4 * 3 * n1))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.ce_dd, 2 * 3 * n1))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.hg4, 4 * (size_t)P.ncvs))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.hg2, 2 * (size_t)P.ncvs))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.trie, 2 * (size_t)P.trie_n))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.a1u4, 4 * n1))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.a2u4, 4 * n1))) return fail(rc);
    launch_make_f32(P, h->stream);
    CK(cudaGetLastError());
    // records of the compact stage kernel, used where the mesh's edge metrics are the ones
    // its coordinates define (checked here, bit for bit)
    if ((rc = dalloc(h, (int**)&f.slot4, 4 * 3 * n1))) return fail(rc);
    if ((rc = dalloc(h, (double**)&f.vxy, 2 * ((size_t)P.M + 1)))) return fail(rc);
    if ((rc = dalloc(h, (double**)&f.xyc, 2 * n1))) return fail(rc);
    if ((rc = dalloc(h, (float**)&f.artcc, 2 * n1))) return fail(rc);
    if ((rc = dalloc(h, (double**)&f.exc0, 4 * n1))) return fail(rc);
    if ((rc = dalloc(h, (double**)&f.exc1, 4 * n1))) return fail(rc);
    if ((rc = dalloc(h, &f.cflag, n1))) return fail(rc);
    int* d_bad = nullptr;
    if ((rc = dalloc(h, &d_bad, 1))) return fail(rc);
    launch_make_compact(P, h->stream, d_bad);
    CK(cudaGetLastError());
    int bad = -1;
    CK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->compact_ok = (bad == 0 && !P.limiter && !P.gcy) ? 1 : 0;
  }
  P.prec = mode;
  P.f.compact = (mode == FVG_PREC_FP32_FLUX && h->compact_ok) ? h->compact_allowed : 0;
  // The captured step holds the other precision's kernels: capture again.
  CK(cudaStreamSynchronize(h->stream));
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  return FVG_OK;
}

int32_t fvg_get_precision(const fvg_handle* h) { return h ? h->P.prec : -1; }

int fvg_set_closure(fvg_handle* h, int32_t mode, const float* params, int32_t nparams, const float* norm,
                    int32_t nnorm) {
  if (!h) return FVG_ERR_ARG;
  Dev& P = h->P;
  CK(cudaStreamSynchronize(h->stream));
  auto regraph = [&]() {
    if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  };
  if (mode == 0) { P.closure = 0; regraph(); return FVG_OK; }
  if (mode != 1 || !params || nparams != fvg_mlp_num_params() || !norm || nnorm != FVG_CLOSURE_NORM_FLOATS) {
    h->err = "fvg_set_closure: bad mode, parameter or scaling vector";
    return FVG_ERR_ARG;
  }
  if (P.KBM1 < 2) { h->err = "fvg_set_closure: no interior levels"; return FVG_ERR_ARG; }
  const size_t S = (size_t)P.M * (P.KBM1 - 1);
  int rc;
  if (!P.clos_feat) {
    if (closure_setup_attrs()) { h->err = "cannot configure the closure kernel"; return FVG_ERR_CUDA; }
    if ((rc = dalloc(h, &P.clos_feat, S))) return rc;
    // one flag per level chunk and node: at most KB chunks (one level per thread)
    if ((rc = dalloc(h, &P.clos_envc, (size_t)P.KB * ((size_t)P.M + 1)))) return rc;
    if ((rc = dalloc(h, &P.clos_env, (size_t)P.M + 1))) return rc;
    if ((rc = dalloc(h, &P.clos_list, (size_t)P.M + 1))) return rc;
    if ((rc = dalloc(h, &P.clos_cnt, (size_t)P.M / 1024 + 2))) return rc;
    if ((rc = dalloc(h, &P.clos_err, 1))) return rc;
    float* b = nullptr;
    if ((rc = dalloc(h, &b, 144))) return rc;
    P.clos_b = b;
    uint8_t* w = nullptr;
    if ((rc = dalloc(h, &w, closure_weight_image_bytes()))) return rc;
    P.clos_w = w;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    h->clos_grid = closure_ctas_per_sm() * nsm;
  }
  std::vector<uint8_t> img;
  std::vector<float> bias;
  closure_weight_image(params, img, bias);
  CK(cudaMemcpy((void*)P.clos_w, img.data(), img.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy((void*)P.clos_b, bias.data(), bias.size() * sizeof(float), cudaMemcpyHostToDevice));
  CK(cudaMemset(P.clos_err, 0, sizeof(int)));
  ClosNorm nm{};
  for (int f = 0; f < 8; ++f) {
    nm.kind[f] = (int)norm[f];
    nm.scale[f] = norm[8 + f];
    nm.mean[f] = norm[16 + f];
    nm.std[f] = norm[24 + f];
    nm.lo[f] = norm[32 + f];
    nm.hi[f] = norm[40 + f];
  }
  for (int c = 0; c < 3; ++c) {
    nm.tmean[c] = norm[48 + c];
    nm.tstd[c] = norm[51 + c];
  }
  nm.teps = norm[54];
  P.clos_norm = nm;
  P.closure = 1;
  regraph();
  return FVG_OK;
}

int fvg_closure_status(fvg_handle* h, int32_t* columns_on_network, int32_t* wait_timeouts) {
  if (!h) return FVG_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  if (columns_on_network) {
    *columns_on_network = 0;
    if (h->P.clos_env) {
      std::vector<int> env(h->P.M + 1);
      CK(cudaMemcpy(env.data(), h->P.clos_env, env.size() * sizeof(int), cudaMemcpyDeviceToHost));
      int c = 0;
      for (int i = 1; i <= h->P.M; ++i) c += env[i] != 0;
      *columns_on_network = c;
    }
  }
  if (wait_timeouts) {
    *wait_timeouts = 0;
    if (h->P.clos_err) CK(cudaMemcpy(wait_timeouts, h->P.clos_err, sizeof(int), cudaMemcpyDeviceToHost));
  }
  return FVG_OK;
}

int fvg_closure_sample(fvg_handle* h, float* dev_buf, int64_t cap) {
  if (!h) return FVG_ERR_ARG;
  const int64_t need = (int64_t)CLOS_PLANES * h->P.M * (h->P.KBM1 - 1);
  if (dev_buf && cap < need) { h->err = "closure sample buffer too small"; return FVG_ERR_ARG; }
  CK(cudaStreamSynchronize(h->stream));
  if (dev_buf != h->P.clos_samp) {
    h->P.clos_samp = dev_buf;
    if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  }
  return FVG_OK;
}

int fvg_set_tuning(fvg_handle* h, const char* key, int32_t value) {
  if (!h || !key) return FVG_ERR_ARG;
  std::string k(key);
  if (k == "col_threads") {
    if (value < 32 || value > 256 || value % 32 != 0) { h->err = "col_threads must be 32..256, a multiple of 32"; return FVG_ERR_ARG; }
    h->P.col_bc = value;
  } else if (k == "col_layers") {
    if (value < 1 || value > h->P.KB) { h->err = "col_layers must be 1..KB"; return FVG_ERR_ARG; }
    h->P.col_lc = value;
  } else if (k == "staged") {
    if (value < 0 || value > 2) { h->err = "staged must be 0, 1 or 2"; return FVG_ERR_ARG; }
    h->P.staged = value;
  } else if (k == "compact") {
    h->compact_allowed = value != 0;
    h->P.f.compact = (h->P.prec == FVG_PREC_FP32_FLUX && h->compact_ok) ? h->compact_allowed : 0;
  } else if (k == "stream_hints") {
    h->P.ldcs = value != 0;
  } else if (k == "ext_grid") {
    if (value < 0 || value > 8) { h->err = "ext_grid must be 0..8 blocks per SM"; return FVG_ERR_ARG; }
    h->P.ext_grid = value;
  } else {
    h->err = "unknown tuning key " + k;
    return FVG_ERR_ARG;
  }
  // The captured step holds the old launch shapes: capture again on the next step.
  CK(cudaStreamSynchronize(h->stream));
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  return FVG_OK;
}

int fvg_get_tuning(const fvg_handle* h, const char* key, int32_t* value) {
  if (!h || !key || !value) return FVG_ERR_ARG;
  std::string k(key);
  if (k == "col_threads") *value = h->P.col_bc;
  else if (k == "col_layers") *value = h->P.col_lc;
  else if (k == "compact") *value = h->P.f.compact;
  else if (k == "staged") *value = h->P.staged;
  else if (k == "stream_hints") *value = h->P.ldcs;
  else if (k == "ext_grid") *value = h->P.ext_grid;
  else return FVG_ERR_ARG;
  return FVG_OK;
}

int fvg_run_routine(fvg_handle* h, int32_t r, int32_t arg) {
  if (!h) return FVG_ERR_ARG;
  if (r == FVG_R_INTERNAL_STEP) return fvg_run(h, 1);
  const Dev& P = h->P;
  const fvg_params& p = h->prm;
  cudaStream_t s = h->stream;
  const int len = P.sl.len;
  const int R = h->sched_cap;
  int iext = 1;
  if (r == FVG_R_EXTERNAL_STEP) {
    iext = arg;
    h->ext_time = h->ext_time + p.dte;
    if (p.iramp != 0) {
      double tmp = (double)(h->iint - 1) + (double)arg / (double)p.isplit;
      h->ramp = std::tanh(tmp / (double)p.iramp);
    } else {
      h->ramp = 1.0;
    }
  } else if (r == FVG_R_INT_FORCING) {
    h->ramp = p.iramp != 0 ? std::tanh((double)h->iint / (double)p.iramp) : 1.0;
  }
  CK(cudaStreamSynchronize(s));
  double* row = h->h_sched + (size_t)R * len;
  fill_routine_row(h, row);
  CK(cudaMemcpyAsync(h->d_sched + (size_t)R * len, row, len * sizeof(double), cudaMemcpyHostToDevice, s));
  h->h_ctl[0] = R;
  CK(cudaMemcpyAsync(P.ctl, h->h_ctl, sizeof(int), cudaMemcpyHostToDevice, s));
  const int spc = 0;
  switch (r) {
    case FVG_R_EXTEL_EDGE:
      launch_ext_prep(P, s);
      launch_ext_node(P, s, 1, arg, EN_EXTEL);
      break;
    case FVG_R_BCOND_ELF: launch_ext_node(P, s, 1, arg, EN_BC); break;
    case FVG_R_N2E2D_ELF: launch_ext_cell(P, s, 1, 1, EC_N2E); break;
    case FVG_R_WET_JUDGE: launch_wet_judge(P, s); break;
    case FVG_R_FLUX_OBN: launch_ext_cell(P, s, 1, arg, EC_FLUXOBN); break;
    case FVG_R_ADVAVE:
      launch_ext_prep(P, s);
      if (P.limiter) launch_alfa2(P, s);
      launch_ext_cell(P, s, 1, 1, EC_ADVAVE);
      break;
    case FVG_R_EXTUV_EDGE: launch_ext_cell(P, s, 1, arg, EC_EXTUV); break;
    case FVG_R_BCOND_UV2D: launch_ext_cell(P, s, 1, 1, EC_BC2); break;
    case FVG_R_EXT_UPDATE: launch_ext_update(P, s, arg); break;
    case FVG_R_EXTERNAL_STEP:
      launch_ext_prep(P, s);
      for (int K = 1; K <= 4; ++K) {
        launch_ext_node(P, s, iext, K, EN_EXTEL | EN_BC | EN_GRAD | (K == 1 ? EN_COPY_ELRK : 0));
        if (p.wetting_drying_on) launch_wet_judge(P, s);
        if (P.limiter) launch_alfa2(P, s);
        launch_ext_cell(P, s, iext, K,
                        (p.wetting_drying_on ? 0 : EC_N2E) | EC_FLUXOBN | EC_ADVAVE | EC_EXTUV | EC_BC2 |
                            (K == 1 ? EC_COPY_RK : 0));
        launch_ext_update(P, s, K);
      }
      break;
    case FVG_R_ADJUST2D3D:
      if (arg == 1) launch_cell_pre(P, s, CP_ADJUST1);
      else launch_adjust2(P, s, AJ_ADJUST);
      break;
    case FVG_R_BCOND_UV3D_SOLID: launch_cell_pre(P, s, CP_BC5); break;
    case FVG_R_BROUGH:
      launch_cell_pre(P, s, CP_BROUGH);
      launch_vertvl_col(P, s, VC_BOT_NODE);
      break;
    case FVG_R_ADVECTION3D:
      launch_grad3(P, s);
      launch_advection3d(P, s);
      break;
    case FVG_R_BAROPG:
      if (P.baropg_z) {
        launch_phy_baropg(P, s);
      } else {
        launch_baropg(P, s, 1, 0);
        launch_vertvl_col(P, s, VC_RHO_ROUNDTRIP);
      }
      break;
    case FVG_R_INT_PRE_EXT:
      launch_baropg(P, s, 0, 1);
      launch_ext_prep(P, s);
      if (P.limiter) launch_alfa2(P, s);
      launch_ext_cell(P, s, 1, 1, EC_INT_ADVAVE);
      launch_int_reset(P, s);
      break;
    case FVG_R_VERTVL:
      launch_adjust2(P, s, AJ_HE_FLUX);
      launch_vertvl_flux(P, s);
      launch_vertvl_col(P, s, VC_WTS);
      launch_w_viscofh(P, s, 1, 0);
      break;
    case FVG_R_VISCOFH: launch_w_viscofh(P, s, 0, 1); break;
    case FVG_R_ADV_UV:
      launch_grad3(P, s);
      launch_adv_uv(P, s);
      break;
    case FVG_R_VDIF_UV: launch_vdif_uv(P, s, VU_VDIF); break;
    case FVG_R_BCOND_UV3D: launch_vdif_uv(P, s, VU_BC3); break;
    case FVG_R_WREAL: launch_vdif_uv(P, s, VU_WREAL); break;
    case FVG_R_ADV_Q:
      launch_grad(P, s, 0);
      launch_adv_q(P, s, (arg == 0 ? AD_Q2 : AD_Q2L) | spc);
      break;
    case FVG_R_FCT_Q: launch_fct_q(P, s, arg == 0 ? AD_Q2 : AD_Q2L); break;
    case FVG_R_VDIF_Q:
      launch_vdif_q(P, s, 0);
      if (P.closure) launch_closure(P, s, P.clos_err, h->clos_grid);
      break;
    case FVG_R_TURB_UPDATE: launch_turb_update(P, s); break;
    case FVG_R_ADV_TS:
      launch_grad(P, s, 1);
      launch_adv_ts(P, s, arg == 1 ? AD_T : AD_S);
      break;
    case FVG_R_FCT_TS: launch_fct_ts(P, s, arg == 1 ? AD_T : AD_S); break;
    case FVG_R_VDIF_TS: launch_vdif_ts(P, s, arg == 1 ? AD_T : AD_S); break;
    case FVG_R_BCOND_TS: launch_bcond_ts(P, s, arg == 1 ? AD_T : AD_S); break;
    case FVG_R_TS_UPDATE: launch_final(P, s, arg == 1 ? FI_T : FI_S); break;
    case FVG_R_DENS2: launch_final(P, s, FI_DENS); break;
    case FVG_R_INT_FINAL: launch_final(P, s, FI_SHIFT); break;
    case FVG_R_INT_FORCING:
      launch_set_qdis(P, s);
      launch_cell_pre(P, s, CP_BCOND8);
      break;
    default: h->err = "unknown routine"; return FVG_ERR_ARG;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  return FVG_OK;
}

int fvg_shutdown_check(fvg_handle* h) {
  if (!h) return FVG_ERR_ARG;
  std::vector<double> d1(h->P.N + 1);
  int rc = fvg_get_field(h, "d1", d1.data(), (int64_t)d1.size());
  if (rc) return rc;
  double s = 0.0;
  for (int i = 1; i <= h->P.N; ++i) s = s + d1[i];
  if (!std::isfinite(s)) { h->err = "non-finite depth (SHUTDOWN_CHECK)"; return FVG_ERR_NAN; }
  return FVG_OK;
}

// ---------------------------------------------------------------------------------------
// Groups: several models stepped by one CUDA graph per internal step.
// ---------------------------------------------------------------------------------------
}  // extern "C"

struct fvg_group {
  std::vector<fvg_handle*> hs;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::vector<cudaEvent_t> ev;  // fork event + one join event per model
  std::string err;
};

static void group_free(fvg_group* g) {
  if (!g) return;
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->gexec) cudaGraphExecDestroy(g->gexec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (auto e : g->ev) cudaEventDestroy(e);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

#define GK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      g->err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
      return FVG_ERR_CUDA;                                                             \
    }                                                                                  \
  } while (0)

static int group_capture(fvg_group* g) {
  GK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
  GK(cudaEventRecord(g->ev[0], g->stream));
  for (size_t q = 0; q < g->hs.size(); ++q) {
    fvg_handle* h = g->hs[q];
    GK(cudaStreamWaitEvent(h->stream, g->ev[0], 0));
    enqueue_internal_step(h, h->stream);
    GK(cudaEventRecord(g->ev[q + 1], h->stream));
    GK(cudaStreamWaitEvent(g->stream, g->ev[q + 1], 0));
  }
  cudaError_t e = cudaStreamEndCapture(g->stream, &g->graph);
  if (e != cudaSuccess) { g->err = std::string("group capture: ") + cudaGetErrorString(e); return FVG_ERR_CUDA; }
  GK(cudaGraphInstantiate(&g->gexec, g->graph, 0));
  return FVG_OK;
}

static int group_steps(fvg_group* g, int32_t nsteps, double* ms) {
  if (nsteps < 0) return FVG_ERR_ARG;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (ms) {
    GK(cudaEventCreate(&t0));
    GK(cudaEventCreate(&t1));
  }
  double total = 0.0;
  int cap = g->hs[0]->sched_cap;
  for (fvg_handle* h : g->hs) cap = std::min(cap, h->sched_cap);
  int done = 0;
  while (done < nsteps) {
    const int c = std::min(cap, nsteps - done);
    GK(cudaStreamSynchronize(g->stream));
    for (fvg_handle* h : g->hs) {
      GK(cudaStreamSynchronize(h->stream));
      int rc = prep_chunk(h, c);
      if (rc) { g->err = h->err; return rc; }
      GK(cudaStreamSynchronize(h->stream));
    }
    if (!g->gexec) {
      int rc = group_capture(g);
      if (rc) return rc;
    }
    if (ms) GK(cudaEventRecord(t0, g->stream));
    for (int s = 0; s < c; ++s) GK(cudaGraphLaunch(g->gexec, g->stream));
    if (ms) {
      GK(cudaEventRecord(t1, g->stream));
      GK(cudaEventSynchronize(t1));
      float f = 0.f;
      GK(cudaEventElapsedTime(&f, t0, t1));
      total += f;
    }
    GK(cudaStreamSynchronize(g->stream));
    for (fvg_handle* h : g->hs) finish_chunk(h, c);
    done += c;
  }
  if (ms) {
    *ms = total;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
  }
  return FVG_OK;
}

extern "C" {

int fvg_group_create(fvg_handle* const* hs, int32_t n, fvg_group** out) {
  if (!hs || !out || n < 1) return FVG_ERR_ARG;
  *out = nullptr;
  for (int32_t q = 0; q < n; ++q) {
    if (!hs[q]) return FVG_ERR_ARG;
    for (int32_t r = 0; r < q; ++r)
      if (hs[r] == hs[q]) return FVG_ERR_ARG;
  }
  fvg_group* g = new fvg_group();
  g->hs.assign(hs, hs + n);
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) { group_free(g); return FVG_ERR_CUDA; }
  g->ev.resize((size_t)n + 1, nullptr);
  for (auto& e : g->ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) { group_free(g); return FVG_ERR_CUDA; }
  *out = g;
  return FVG_OK;
}

void fvg_group_destroy(fvg_group* g) { group_free(g); }

const char* fvg_group_last_error(const fvg_group* g) { return g ? g->err.c_str() : "null group"; }

int fvg_group_run(fvg_group* g, int32_t nsteps) {
  if (!g) return FVG_ERR_ARG;
  return group_steps(g, nsteps, nullptr);
}

int fvg_group_time_steps(fvg_group* g, int32_t nsteps, double* ms) {
  if (!g || !ms) return FVG_ERR_ARG;
  return group_steps(g, nsteps, ms);
}

int fvg_budget(fvg_handle* h, double out[3]) {
  if (!h || !out) return FVG_ERR_ARG;
  launch_budget(h->P, h->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, h->P.budget, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return FVG_OK;
}

}  // extern "C"
