/*
 * fvg.h - C ABI of the B200 mode-split time step for FVCOM.
 *
 * The library replaces FVCOM's two argument-less time-step subroutines,
 *   SUBROUTINE EXTERNAL_STEP   (FVCOM_source/external_step.F:30)
 *   SUBROUTINE INTERNAL_STEP   (FVCOM_source/internal_step.F:29)
 * which read and write FVCOM's module globals (ALL_VARS, MOD_WD, BCS, MOD_OBCS,
 * CONTROL).  Here the same state lives in device memory owned by an fvg_handle; the
 * host hands over the mesh arrays once (fvg_create), copies state in and out by FVCOM
 * variable name (fvg_set_field / fvg_get_field) and calls fvg_internal_step once per
 * internal step, as fvcom.F:848-852 calls INTERNAL_STEP.
 *
 * Array convention: every per-node, per-cell, per-edge and per-half-edge array uses
 * FVCOM's 1-based numbering with the ghost row 0 kept, and 2-D arrays are
 * column-major (Fortran order): element (i, j) of an array with rows 0..len sits at
 * a[(j-1)*(len+1) + i], j 1-based.  Arrays that FVCOM allocates without a ghost row
 * (NBSN, NBVE, NBVT, DLTXTRIE..., IEC, IENODE, NIEC, NTRG, DLTXE, DLTYE, DLTXNCVE,
 * DLTYNCVE) are passed with an unused row 0 as well.  3-D fields are (0:len, 1:KB).
 *
 * Every entry point returns an int status (FVG_OK on success) and never aborts the
 * process, in place of FVCOM's FATAL_ERROR/PSTOP (FVCOM_source/mod_utils.F:270).
 * One host thread per handle; calls on one handle are not re-entrant; separate handles
 * are independent and each owns one CUDA stream.
 */
#ifndef FVG_H
#define FVG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FVG_OK 0
#define FVG_ERR_ARG 1          /* bad argument, size or unknown field name */
#define FVG_ERR_CUDA 2         /* a CUDA runtime call failed */
#define FVG_ERR_NAN 3          /* SHUTDOWN_CHECK: non-finite depth (mod_utils.F:320-376) */
#define FVG_ERR_BOUNDS 4       /* an index in the mesh arrays is out of range */
#define FVG_ERR_TIMEOUT 5      /* a bounded device wait ran out */
#define FVG_ERR_UNSUPPORTED 6  /* option outside the supported physics set */
#define FVG_ERR_NOMEM 7        /* device allocation failed */
#define FVG_ERR_CAPACITY 8     /* input larger than a fixed-size device buffer */

/* Mesh arrays as GRID_METRICS builds them (FVCOM_source/grid_metrics.F:29-136). */
typedef struct fvg_mesh {
  int32_t m, n, kb;          /* nodes M, cells N, sigma levels KB (KBM1 = KB-1 layers) */
  int32_t ne, ncv, ncv_i;    /* element edges NE, CV half-edges NCV, interior NCV_I */
  int32_t nbsn_cols;         /* columns of NBSN (>= max NTSN) */
  int32_t nbve_cols;         /* columns of NBVE/NBVT (>= max NTVE + 1) */
  int32_t trie_cols;         /* columns of DLTXTRIE.. DLTYNEC (FVCOM: 12) */

  /* nodes (0:M) */
  const double *vx, *vy, *h, *art1, *art2, *grav_n, *nn_hvc, *sita_gd, *phpn;
  const int32_t *isonb, *ntsn, *ntve;
  const int32_t *nbsn;                 /* NBSN(0:M, nbsn_cols) */
  const int32_t *nbve, *nbvt;          /* NBVE/NBVT(0:M, nbve_cols) */
  const double *dltxtrie, *dltytrie;   /* (0:M, trie_cols) */
  const double *dltxecec, *dltyecec;   /* (0:M, trie_cols) */
  const double *dltxnec, *dltynec;     /* (0:M, trie_cols) */
  const double *z, *zz, *dz, *dzz;     /* (0:M, KB) */

  /* cells (0:N) */
  const double *xc, *yc, *art, *h1, *cor, *grav_e, *cc_hvc, *cc_sponge, *cc_z0b;
  const double *epor, *iucp, *alpha;
  const int32_t *nv;                   /* NV(0:N, 3), clockwise */
  const int32_t *nbe;                  /* NBE(0:N, 3) */
  const int32_t *isbce;
  const double *a1u, *a2u;             /* (0:N, 4) */
  const double *awx, *awy;             /* (0:N, 3) */
  const double *z1, *zz1, *dz1, *dzz1; /* (0:N, KB) */

  /* element edges (0:NE) */
  const int32_t *iec, *ienode;         /* (0:NE, 2) */
  const int32_t *isbc;
  const double *xijc, *yijc, *dltxc, *dltyc;

  /* control-volume half-edges (0:NCV) */
  const int32_t *niec;                 /* (0:NCV, 2) */
  const int32_t *ntrg;
  const double *dltxe, *dltye;
  const double *dltxncve, *dltyncve;   /* (0:NCV_I, 2) */

  /* open boundary (1:IOBCN, ghost row 0) - SETUP_OBC (mod_obcs.F:868-1173) */
  int32_t iobcn;
  const int32_t *i_obc_n, *type_obc, *next_obc, *nadjc_obc;
  const int32_t *adjc_obc;             /* (0:IOBCN, 2) */
  const double *fluxf_obc;             /* (0:IOBCN, 2) */
  const double *dltn_obc;

  /* rivers (1:NUMQBC, ghost row 0) - SET_RIVER_BNDRY_METRICS (mod_force.F:3447-3581) */
  int32_t numqbc;
  const int32_t *inodeq, *icellq;
  const int32_t *n_icellq;             /* (0:NUMQBC, 2) */
  const double *rdisq;                 /* (0:NUMQBC, 2) */
  const double *qarea, *angleq;
  const double *vqdist;                /* (0:NUMQBC, KBM1) */
} fvg_mesh;

/* Run-time switches and constants (NML_INTEGRATION, NML_PHYSICS, NML_OPEN_BOUNDARY_CONTROL,
 * NML_RIVER_TYPE; FVCOM_source/mod_main.F:121-942). */
typedef struct fvg_params {
  double dte;                 /* EXTSTEP_SECONDS */
  int32_t isplit;             /* ISPLIT */
  int32_t iramp;              /* IRAMP (0: no ramp) */
  double min_depth;           /* MIN_DEPTH */
  double static_ssh_adj;      /* STATIC_SSH_ADJ */
  int32_t horizontal_mixing;  /* 0 'closure', 1 'constant' */
  double hprnu;               /* HORIZONTAL_PRANDTL_NUMBER */
  double umol;                /* VERTICAL_MIXING_COEFFICIENT */
  double vprnu;               /* VERTICAL_PRANDTL_NUMBER */
  double cbcmin;              /* BOTTOM_ROUGHNESS_MINIMUM */
  int32_t vertical_mixing;    /* 0 'closure' (MY2.5), 1 'constant' */
  int32_t wetting_drying_on;
  int32_t scalar_positivity_control;
  int32_t barotropic;
  int32_t temperature_active, salinity_active;
  int32_t obc_elevation_forcing_on;
  int32_t obc_ts_type;        /* OBC_TS_TYPE 1..3 */
  int32_t river_ts_setting;   /* 0 'specified' */
  int32_t river_location;     /* 0 'node', 1 'edge' */
  double tide_ref_time;       /* SpecTime: the zero of the tidal phase, seconds */
  /* HEATING_ON with HEATING_TYPE 'flux' (vdif_ts.F:118-150, cntrl_prmtrs.F:144-160):
     the surface net heat flux and the short-wave radiation absorbed over depth as
     RHEAT*exp(z/ZETA1) + (1-RHEAT)*exp(z/ZETA2).  0 for no surface heating. */
  int32_t heating_on;
  double rheat;               /* HEATING_LONGWAVE_PERCTAGE */
  double zeta1;               /* HEATING_LONGWAVE_LENGTHSCALE, m */
  double zeta2;               /* HEATING_SHORTWAVE_LENGTHSCALE, m */
  /* Face-value limiter of the momentum advection (ADVAVE, ADVECTION, ADV_UV), FVCOM's
     compile-time choice: 0 LIMITED_NO; 1 LIMITED_1 (the slope limiter UALFA/VALFA and the
     clamp of both face values into the range of the two cells); 2 the slope limiter alone
     (advave_edge_gcn.F:128-330, advection_edge_gcn.F:107-335, adv_uv_edge_gcn.F:138-400). */
  int32_t limiter;
  /* BAROCLINIC_PRESSURE_GRADIENT: 0 'sigma levels' (BAROPG), 1 'z coordinates'
     (PHY_BAROPG, phy_baropg.F:37-151: 600 z levels of HMAX/600) */
  int32_t baropg_z;
  /* Solid-boundary treatment of the momentum advection: 0 GCN (no ghost cell); 1 GCY,
     ghost cells (ghostuv.F, advave_edge_gcy.F, advection_edge_gcy.F, adv_uv_edge_gcy.F,
     bcond_gcy.F).  The GCY1/GCY2 choice of ghost point lives in the mesh's A1U/A2U
     (SHAPE_COEF_GCY). */
  int32_t ghost_cells;
} fvg_params;

/* Boundary forcing that is constant in time for the supported cases. */
typedef struct fvg_forcing {
  /* spectral tide on the open boundary (BCOND_ASL, mod_obcs.F:554-583) */
  int32_t ntide;
  const double *period;       /* (ntide) seconds */
  const double *apt;          /* (0:IOBCN, ntide) amplitude m */
  const double *phai;         /* (0:IOBCN, ntide) phase, degrees */
  const double *emean;        /* (0:IOBCN) mean level m */
  /* river discharge and its temperature/salinity (UPDATE_RIVERS, mod_force.F:11229) */
  const double *qdis;         /* (0:NUMQBC) m^3/s before the ramp */
  const double *tdis, *sdis;  /* (0:NUMQBC) */
  /* surface wind stress before RAMP*0.001 scaling (UPDATE_WIND / ASIMPLE_DRAG);
     NULL for no wind.  (0:N) */
  const double *wstress_x, *wstress_y;
  /* surface heating in W/m^2 before RAMP (UPDATE_HEAT, mod_force.F:12427; positive warms
     the ocean): short-wave radiation and net heat flux per node (0:M).  Read only when
     heating_on; NULL is taken as zero. */
  const double *swrad, *wtsurf;
} fvg_forcing;

typedef struct fvg_handle fvg_handle;

/* Routine identifiers for fvg_run_routine: one FVCOM subroutine on the current state. */
enum fvg_routine {
  FVG_R_EXTEL_EDGE = 1,        /* EXTEL_EDGE(K)           extel_edge.F:32       arg: K */
  FVG_R_BCOND_ELF = 2,         /* BCOND_GCN(1,K)+RK blend external_step.F:253-266 arg: K */
  FVG_R_N2E2D_ELF = 3,         /* N2E2D(ELF,ELF1)         external_step.F:287 */
  FVG_R_WET_JUDGE = 4,         /* WET_JUDGE               mod_wd.F:193 */
  FVG_R_FLUX_OBN = 5,          /* FLUX_OBN(K)             mod_obcs.F:1181       arg: K */
  FVG_R_ADVAVE = 6,            /* ADVAVE_EDGE_GCN(ADVUA,ADVVA) advave_edge_gcn.F:32 */
  FVG_R_EXTUV_EDGE = 7,        /* EXTUV_EDGE(K)           extuv_edge.F:33       arg: K */
  FVG_R_BCOND_UV2D = 8,        /* BCOND_GCN(2,K)          bcond_gcn.F:325 */
  FVG_R_EXT_UPDATE = 9,        /* external_step.F:333-436 (state shift, K==3/4 sums) arg: K */
  FVG_R_EXTERNAL_STEP = 10,    /* EXTERNAL_STEP (all 4 stages) arg: IEXT */
  FVG_R_ADJUST2D3D = 11,       /* ADJUST2D3D(arg)         adjust2d3d.F:29 */
  FVG_R_BCOND_UV3D_SOLID = 12, /* BCOND_GCN(5,0)          bcond_gcn.F:537 */
  FVG_R_BROUGH = 13,           /* BOTTOM_ROUGHNESS        brough.F:41 */
  FVG_R_ADVECTION3D = 14,      /* ADVECTION_EDGE_GCN      advection_edge_gcn.F:30 */
  FVG_R_BAROPG = 15,           /* BAROPG                  baropg.F:33 */
  FVG_R_INT_PRE_EXT = 16,      /* internal_step.F:374-416 (2-D sums, ADVAVE, GX/GY) */
  FVG_R_VERTVL = 17,           /* VERTVL_EDGE             vertvl_edge.F:37 */
  FVG_R_VISCOFH = 18,          /* VISCOF_H                viscofh.F:33 */
  FVG_R_ADV_UV = 19,           /* ADV_UV_EDGE_GCN         adv_uv_edge_gcn.F:31 */
  FVG_R_VDIF_UV = 20,          /* VDIF_UV                 vdif_uv.F:34 */
  FVG_R_BCOND_UV3D = 21,       /* static-SSH fix + BCOND_GCN(3,0) internal_step.F:660-672 */
  FVG_R_WREAL = 22,            /* WREAL                   wreal.F:32 */
  FVG_R_ADV_Q = 23,            /* ADV_Q(Q2,Q2F) arg 0, ADV_Q(Q2L,Q2LF) arg 1  adv_q.F:35 */
  FVG_R_FCT_Q = 24,            /* FCT_Q2 arg 0, FCT_Q2L arg 1 */
  FVG_R_VDIF_Q = 25,           /* VDIF_Q                  vdif_q.F:34 */
  FVG_R_TURB_UPDATE = 26,      /* Q2=Q2F, Q2L=Q2LF, N2E3D(KM,KM1) internal_step.F:1034-1053 */
  FVG_R_ADV_TS = 27,           /* ADV_T arg 1, ADV_S arg 2 adv_t.F:34 / adv_s.F:34 */
  FVG_R_FCT_TS = 28,           /* FCT_T arg 1, FCT_S arg 2 */
  FVG_R_VDIF_TS = 29,          /* VDIF_TS(arg)            vdif_ts.F:42 */
  FVG_R_BCOND_TS = 30,         /* BCOND_TS(arg)           bcond_ts.F:35 */
  FVG_R_TS_UPDATE = 31,        /* T1=TF1 + N2E3D arg 1; S1=SF1 + N2E3D arg 2 */
  FVG_R_DENS2 = 32,            /* DENS2                   eqs_of_state.F:381 */
  FVG_R_INT_FINAL = 33,        /* U=UF ... WD_UPDATE(3)   internal_step.F:1541-1590 */
  FVG_R_INTERNAL_STEP = 34,    /* INTERNAL_STEP           internal_step.F:29 */
  FVG_R_INT_FORCING = 35       /* RAMP, BCOND_GCN(8,0)    internal_step.F:115-265 */
};

/* Lifecycle.  fvg_create copies the mesh to the device and builds the gather lists;
   the host arrays may be freed afterwards. */
int fvg_create(const fvg_mesh* mesh, const fvg_params* params, const fvg_forcing* forcing,
               fvg_handle** out);
void fvg_destroy(fvg_handle* h);
const char* fvg_last_error(const fvg_handle* h);

/* State exchange by FVCOM variable name (lower case, e.g. "el", "ua", "t1", "q2l",
   "iswetn").  count must equal the field's element count ((len+1) or (len+1)*KB). */
int fvg_set_field(fvg_handle* h, const char* name, const double* src, int64_t count);
int fvg_get_field(fvg_handle* h, const char* name, double* dst, int64_t count);
int fvg_set_ifield(fvg_handle* h, const char* name, const int32_t* src, int64_t count);
int fvg_get_ifield(fvg_handle* h, const char* name, int32_t* dst, int64_t count);
/* Element count of a field, or -1 for an unknown name. */
int64_t fvg_field_size(const fvg_handle* h, const char* name);

/* Model clock: IINT of the last completed internal step and ExtTime in seconds. */
int fvg_set_clock(fvg_handle* h, int32_t iint, double ext_time);
int fvg_get_clock(const fvg_handle* h, int32_t* iint, double* ext_time);

/* One INTERNAL_STEP for IINT+1 (fvcom.F:848-852), ISPLIT external steps included. */
int fvg_internal_step(fvg_handle* h);
/* One EXTERNAL_STEP (external_step.F:29) of external step IEXT (1..ISPLIT) of the current
   internal step: the 4 Runge-Kutta stages with their boundary conditions, as
   INTERNAL_STEP calls it at internal_step.F:499 (fvg_internal_step runs all ISPLIT). */
int fvg_external_step(fvg_handle* h, int32_t iext);
/* New forcing for the following steps (UPDATE_TIDE/UPDATE_RIVERS/UPDATE_WIND,
   mod_force.F:14341, :11229, :13415): tidal constituents (same NTIDE as at creation),
   river discharge/T/S and surface stress; NULL members are left unchanged. */
int fvg_set_forcing(fvg_handle* h, const fvg_forcing* f);
/* n consecutive internal steps; replayed from a captured CUDA graph after the first. */
int fvg_run(fvg_handle* h, int32_t nsteps);
/* One reference routine (enum fvg_routine) on the current state, for parity checks. */
int fvg_run_routine(fvg_handle* h, int32_t routine, int32_t arg);
/* Wait for all device work of the handle. */
int fvg_sync(fvg_handle* h);
/* Override the RAMP factor that fvg_run_routine uses (fvg_run sets it from IINT). */
int fvg_set_ramp(fvg_handle* h, double ramp);
/* 1 (default): replay a captured CUDA graph per internal step; 0: plain launches. */
int fvg_use_graph(fvg_handle* h, int32_t on);
/* Precision form.  FVG_PREC_FP64 (default): FP64 everywhere, bitwise equal to the
   oracle.  FVG_PREC_FP32_FLUX: the edge fluxes and advection -- ADVAVE's edge loop, the
   3-D momentum edge fluxes of ADVECTION_EDGE_GCN/ADV_UV_EDGE_GCN, ADV_Q and ADV_T/ADV_S
   with FCT and their node-ring and cell gradients -- in FP32 arithmetic over FP32 scratch
   and FP32 copies of their mesh metrics; the free-surface update (EXTEL_EDGE), the
   vertical continuity, the tridiagonal solves, the state and the budgets stay FP64.
   The first switch to FP32 allocates its scratch. */
#define FVG_PREC_FP64 0
#define FVG_PREC_FP32_FLUX 1
int fvg_set_precision(fvg_handle* h, int32_t mode);
int32_t fvg_get_precision(const fvg_handle* h);
/* Closure samples for training a learned vertical closure.  While dev_buf (device
   memory, at least 12*M*(KBM1-1) floats) is set, every VDIF_Q writes for each node I and
   interior level K=2..KBM1, at index (K-2)*M + (I-1) of 12 planes of M*(KBM1-1) floats:
   BOYGR (N^2), shear S^2, D, sigma Z, u*_surf, u*_bot, Q2, Q2L -- the closure's inputs
   after VDIF_Q's positivity fixes (vdif_q.F:250-262) -- then its outputs before the
   time averaging, KN*KAPPA*SM, KN*SM, KN*SH*VPRNU (vdif_q.F:479-491), and 1 for a wet
   node (0: the node's planes are not meaningful).  dev_buf NULL stops sampling. */
int fvg_closure_sample(fvg_handle* h, float* dev_buf, int64_t cap);
/* The learned closure's network: an MLP 8 -> 64 -> 64 -> 3, GELU on the hidden layers,
   FP32 parameters (W1 64x8, b1, W2 64x64, b2, W3 3x64, b3; fvg_mlp_num_params() floats)
   trained on the device by the library's own forward/backward kernels (mean-squared
   error, Adam, deterministic gradient sums).  x, y and out are device pointers to
   row-major [n][8] inputs, [n][3] targets and [n][3] outputs. */
typedef struct fvg_mlp fvg_mlp;
int fvg_mlp_create(uint64_t seed, fvg_mlp** out);
void fvg_mlp_destroy(fvg_mlp* q);
const char* fvg_mlp_last_error(const fvg_mlp* q);
int32_t fvg_mlp_num_params(void);
int fvg_mlp_get_params(fvg_mlp* q, float* host, int32_t n);
int fvg_mlp_set_params(fvg_mlp* q, const float* host, int32_t n);
/* Mean-squared error over the n samples and its gradient (host outputs). */
int fvg_mlp_loss_grad(fvg_mlp* q, const float* x, const float* y, int32_t n, float* loss, float* grad);
/* epochs of Adam over shuffled batches; epoch_loss[e] (host, may be NULL) = mean error. */
int fvg_mlp_train(fvg_mlp* q, const float* x, const float* y, int32_t n, int32_t epochs, int32_t batch,
                  float lr, uint64_t seed, float* epoch_loss);
/* FP32 forward pass (the reference of the tensor-core inference). */
int fvg_mlp_forward(fvg_mlp* q, const float* x, int32_t n, float* out);
const float* fvg_mlp_device_params(const fvg_mlp* q);
/* The same network in BF16 on the tensor cores (tcgen05.mma, FP32 accumulate), the
   kernel the learned closure runs; x standardised inputs [n][8], out [n][3]. */
int fvg_mlp_forward_bf16(fvg_mlp* q, const float* x, int32_t n, float* out);
/* Learned vertical closure.  mode 1: VDIF_Q's stability functions and KN of the
   interior levels are replaced by the network (params: fvg_mlp_num_params() floats, the
   layout of fvg_mlp_get_params) run in BF16 on the tensor cores, for every column whose
   inputs all lie inside the training envelope; other columns keep MY2.5.  norm
   (FVG_CLOSURE_NORM_FLOATS floats): input transform kind[8] (0 identity, 1 log, 2
   asinh(x/scale)), scale[8], mean[8], std[8], envelope lo[8], hi[8]; output tmean[3],
   tstd[3], teps (new part = exp(y*tstd + tmean) - teps).  mode 0: MY2.5 everywhere. */
#define FVG_CLOSURE_NORM_FLOATS 55
int fvg_set_closure(fvg_handle* h, int32_t mode, const float* params, int32_t nparams, const float* norm,
                    int32_t nnorm);
/* Columns that used the network in the last step, and the closure's error word: 0, or
   nonzero once a bounded tensor-core wait ran out (1; 2 if the wait for the outstanding
   MMAs before freeing tensor memory ran out as well).  Network rows of a block whose
   wait ran out keep their previous coefficients (columns outside the envelope have MY2.5's
   as always), and fvg_run / fvg_internal_step return FVG_ERR_TIMEOUT while the word is
   set; fvg_set_closure clears it. */
int fvg_closure_status(fvg_handle* h, int32_t* columns_on_network, int32_t* wait_timeouts);
/* Launch shape of the 3-D gather kernels (results do not depend on it):
   "col_threads" = entities (threads) per block, 32..256 in steps of 32 (default 128);
   "col_layers"  = consecutive layers each thread walks, 1..KB (default 8);
   "compact"     = 1 (default) lets the precision form's Runge-Kutta stages use the
                   compact cell kernel where fvg_set_precision found the mesh's edge metrics
                   to be the ones its coordinates define; 0 keeps the general kernel.
                   fvg_get_tuning("compact") reports whether the compact kernel is in use;
   "staged"      = 2 runs ADVECTION_EDGE_GCN and ADV_UV_EDGE_GCN (LIMITED_NO, GCN) as the
                   tile-staged kernels (neighbour cells in shared memory, each edge
                   evaluated once per tile); 1 (default) only the FP64 ADV_UV, where the
                   staged kernel measured faster; 0 keeps one thread per cell everywhere.
                   Results do not depend on it (bit for bit in FP64);
   "stream_hints" = 1 (default): the external loop's stage kernels load the arrays a
                   stage reads once (gather lists, slot records, EXTUV's fixed terms, the
                   Runge-Kutta start values) evict-first in L2, so that the arrays they
                   gather from neighbours stay in L2 from one stage to the next; 0 plain
                   loads.  A cache hint only: results do not depend on it (bit for bit);
   "ext_grid"     = blocks per SM (1..8, default 8) of the external loop's compact cell
                   kernel, launched as one wave whose threads walk the cells so that no
                   partly filled last wave is left; 0 launches one thread per cell.
                   Results do not depend on it. */
int fvg_set_tuning(fvg_handle* h, const char* key, int32_t value);
int fvg_get_tuning(const fvg_handle* h, const char* key, int32_t* value);

/* Groups (batched ensembles).  Several models -- for example union models of ensemble
   members on meshes of different size or layer count -- stepped together: one CUDA
   graph per internal step holds one INTERNAL_STEP of every model, each on its own branch,
   so the models run concurrently from a single launch.  The handles stay usable on their
   own; a handle may belong to several groups but must not be stepped by two host threads
   at once.  fvg_group_time_steps returns the device time of nsteps steps of all models. */
typedef struct fvg_group fvg_group;
int fvg_group_create(fvg_handle* const* handles, int32_t n, fvg_group** out);
int fvg_group_run(fvg_group* g, int32_t nsteps);
int fvg_group_time_steps(fvg_group* g, int32_t nsteps, double* ms);
const char* fvg_group_last_error(const fvg_group* g);
void fvg_group_destroy(fvg_group* g);

/* Measurement.  fvg_time_steps runs nsteps internal steps and returns their device time
   (CUDA events on the handle's stream).  fvg_profile runs nsteps with plain launches and
   events between kernel groups, adding each group's device time to group_ms (length
   fvg_profile_groups()) and the whole steps' time to *total_ms (may be NULL). */
int fvg_time_steps(fvg_handle* h, int32_t nsteps, double* ms);
int32_t fvg_profile_groups(void);
const char* fvg_profile_group_name(int32_t g);
int fvg_profile(fvg_handle* h, int32_t nsteps, double* group_ms, double* total_ms);
/* Number of kernel launches one internal step issues. */
int32_t fvg_kernels_per_step(const fvg_handle* h);

/* SHUTDOWN_CHECK (mod_utils.F:320-376): FVG_ERR_NAN when the sum of D1 is not finite. */
int fvg_shutdown_check(fvg_handle* h);
/* FP64 budgets: out[0] volume (m^3), out[1] heat content (T*volume), out[2] salt
   content (S*volume) over the node control volumes. */
int fvg_budget(fvg_handle* h, double out[3]);

/* The budgets of fvg_budget computed from caller-owned device arrays, with no handle and
   no memory allocation (no counterpart in the reference, which sums its host arrays).
   For callers that keep their own FVCOM state on the device and cannot allocate when
   they check it: cudaMalloc/cudaFree would synchronise the device on every call, and a
   run that fills HBM may have nothing left to allocate.  d and art1 are (0:M); t1, s1
   and dz are (0:M, >=KBM1) column-major with leading dimension M+1 (FVCOM's layout, ghost
   row 0), all in device memory of the current device.  The scratch is a fixed 393,240-
   byte device array: M above 4,194,304 returns FVG_ERR_CAPACITY; KBM1 must be 1..63.
   Runs on `stream` (a cudaStream_t; NULL for the default stream), waits for it and
   copies the three sums into `out` before it returns.  The first call on a device sets
   up the scratch address; make it before any stream capture.  That first call also loads
   the library's device code on the device (CUDA loads modules lazily), which reserves
   device memory for the code and the scratch array: make it early in the run, before
   HBM fills up.  Calls that overlap on one device share the scratch and race. */
int fvg_budget_fields(const double* d, const double* art1, const double* t1, const double* s1,
                      const double* dz, int32_t m, int32_t kbm1, void* stream, double out[3]);

/* Library identity for checks that the compiled CUDA path is the one loaded. */
const char* fvg_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* FVG_H */
