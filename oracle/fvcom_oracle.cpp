// fvcom_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement, in FP64, of FVCOM's mode-split time step (EXTERNAL_STEP /
// INTERNAL_STEP and every routine they call) for the flag set DOUBLE_PRECISION, GCN,
// LIMITED_NO, WET_DRY (run-time WETTING_DRYING_ON), serial (no MULTIPROCESSOR).  It is the
// checker for the CUDA library (include/fvg.h): tests, the smoke check and the timed CPU
// baseline call it; the product path never does.
//
// It follows the reference's loop order and expression order statement by statement so
// that, compiled without floating-point contraction (-ffp-contract=off), each scatter
// accumulates in the same order as the Fortran.  Default-kind (single precision) Fortran
// literals are reproduced as F4(x) = (double)(float)x.  Fortran SIGN(1.0,x) is taken as
// +1 for x == -0.0 (a processor that does not distinguish negative zero, ifort's default).
//
// Parity is unpinned at the reference boundary: no Fortran compiler exists on this machine
// to run FVCOM itself, and the reference ships no golden outputs.  Each routine cites the
// reference file:line it restates.
//
// OpenMP: loops are parallelised only where iterations touch disjoint targets (per layer
// or per column), so results are bitwise independent of the thread count.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include <algorithm>

#include "../include/fvg.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

static inline double F4(double x) { return (double)(float)x; }
static inline double fsign1(double x) { return x >= 0.0 ? 1.0 : -1.0; }
static inline double fsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }
static inline int nxt(int j) { return j + 1 - ((j + 1) / 4) * 3; }
static inline int nxt2(int j) { return j + 2 - ((j + 2) / 4) * 3; }

const double ALPHA_RK[5] = {0.0, 0.25, 1.0 / 3.0, 0.5, 1.0};  // mod_main.F:1005
const double ONE_THIRD = 1.0 / 3.0;                            // mod_main.F:1013
const double PI2 = 2.0 * 3.141592653589793238;                 // mod_main.F:1011
const double ROFVROS = 0.9775171065;                           // mod_main.F:1017

struct Field {
  double* d = nullptr;
  int32_t* i = nullptr;
  int64_t size = 0;
};

struct Oracle {
  // ---------------- dimensions ----------------
  int M, N, KB, KBM1, KBM2, NE, NCV, NCV_I, M1, N1;
  int NBSNC, NBVEC, TRIEC;
  fvg_params P;
  int IOBCN, NUMQBC, NTIDE;
  int IINT = 0;
  double ExtTime = 0.0;
  double RAMP = 0.0;
  double DTI;

  // ---------------- mesh ----------------
  std::vector<double> vx, vy, h, art1, art2, grav_n, nn_hvc, sita_gd, phpn;
  std::vector<int32_t> isonb, ntsn, ntve, nbsn, nbve, nbvt;
  std::vector<double> dltxtrie, dltytrie, dltxecec, dltyecec, dltxnec, dltynec;
  std::vector<double> z, zz, dz, dzz;
  std::vector<double> xc, yc, art, h1, cor, grav_e, cc_hvc, cc_sponge, cc_z0b, epor, iucp, alpha;
  std::vector<int32_t> nv, nbe, isbce;
  std::vector<double> a1u, a2u, awx, awy, z1, zz1, dz1, dzz1;
  std::vector<int32_t> iec, ienode, isbc;
  std::vector<double> xijc, yijc, dltxc, dltyc;
  std::vector<int32_t> niec, ntrg;
  std::vector<double> dltxe, dltye, dltxncve, dltyncve;
  std::vector<int32_t> i_obc_n, type_obc, next_obc, nadjc_obc, adjc_obc;
  std::vector<double> fluxf_obc, dltn_obc;
  std::vector<int32_t> inodeq, icellq, n_icellq;
  std::vector<double> rdisq, qarea, angleq, vqdist;
  std::vector<int32_t> obc_lst1, obc_lst2;
  // forcing
  std::vector<double> t_period, t_apt, t_phai, t_emean, qdis0, tdis, sdis, wsx, wsy;
  std::vector<double> swrad_w, wtsurf_w, swrad, wtsurf;  // surface heating (0:M)
  bool have_wind = false;

  // ---------------- state ----------------
  // node 2-D
  std::vector<double> el, elf, elrk, et, d, dt, dtfa, egf, wubot_n, wvbot_n, taubm_n;
  std::vector<double> pfpxb, pfpyb, ah_bottom;
  // node 3-D
  std::vector<double> t1, s1, tf1, sf1, rho1, tmean1, smean1, rmean1;
  std::vector<double> q2, q2l, q2f, q2lf, l, km, kh, kq, wts, viscofh;
  // cell 2-D
  std::vector<double> el1, elf1, elrk1, et1, d1, dt1, ua, va, uaf, vaf, uark, vark;
  std::vector<double> uard, vard, adx2d, ady2d, drx2d, dry2d, advua, advva, pstx, psty;
  std::vector<double> wubot, wvbot, cbc, tps, fluxobn, taubm, wusurf, wvsurf, wusurf2, wvsurf2;
  // cell 3-D
  std::vector<double> u, v, uf, vf, w, ww, advx, advy, drhox, drhoy, rho, t, s, rmean;
  std::vector<double> km1, viscofm;
  // wet/dry
  std::vector<int32_t> iswetn, iswetnt, iswetc, iswetct, iswetce;
  // open boundary
  std::vector<double> xflux_obcn, uard_obcn, xflux_obc;
  // river discharge after the ramp
  std::vector<double> qdis;

  std::map<std::string, Field> fields;

  // ---------------- index helpers ----------------
  inline size_t n3(int i, int k) const { return (size_t)(k - 1) * M1 + i; }
  inline size_t c3(int i, int k) const { return (size_t)(k - 1) * N1 + i; }
  inline int NV(int i, int j) const { return nv[(size_t)(j - 1) * N1 + i]; }
  inline int NBE(int i, int j) const { return nbe[(size_t)(j - 1) * N1 + i]; }
  inline int NBSN(int i, int j) const { return nbsn[(size_t)(j - 1) * M1 + i]; }
  inline int NBVE(int i, int j) const { return nbve[(size_t)(j - 1) * M1 + i]; }
  inline int NBVT(int i, int j) const { return nbvt[(size_t)(j - 1) * M1 + i]; }
  inline double TRIE_X(int i, int j) const { return dltxtrie[(size_t)(j - 1) * M1 + i]; }
  inline double TRIE_Y(int i, int j) const { return dltytrie[(size_t)(j - 1) * M1 + i]; }
  inline double ECEC_X(int i, int j) const { return dltxecec[(size_t)(j - 1) * M1 + i]; }
  inline double ECEC_Y(int i, int j) const { return dltyecec[(size_t)(j - 1) * M1 + i]; }
  inline double NEC_X(int i, int j) const { return dltxnec[(size_t)(j - 1) * M1 + i]; }
  inline double NEC_Y(int i, int j) const { return dltynec[(size_t)(j - 1) * M1 + i]; }
  inline double A1U(int i, int j) const { return a1u[(size_t)(j - 1) * N1 + i]; }
  inline double A2U(int i, int j) const { return a2u[(size_t)(j - 1) * N1 + i]; }
  inline double AWX(int i, int j) const { return awx[(size_t)(j - 1) * N1 + i]; }
  inline double AWY(int i, int j) const { return awy[(size_t)(j - 1) * N1 + i]; }
  inline int IEC(int i, int j) const { return iec[(size_t)(j - 1) * (NE + 1) + i]; }
  inline int IENODE(int i, int j) const { return ienode[(size_t)(j - 1) * (NE + 1) + i]; }
  inline int NIEC(int i, int j) const { return niec[(size_t)(j - 1) * (NCV + 1) + i]; }
  inline double DLTXNCVE(int i, int j) const { return dltxncve[(size_t)(j - 1) * (NCV_I + 1) + i]; }
  inline double DLTYNCVE(int i, int j) const { return dltyncve[(size_t)(j - 1) * (NCV_I + 1) + i]; }
  inline int ADJC(int i, int j) const { return adjc_obc[(size_t)(j - 1) * (IOBCN + 1) + i]; }
  inline double FLUXF(int i, int j) const { return fluxf_obc[(size_t)(j - 1) * (IOBCN + 1) + i]; }
  inline int N_ICELLQ(int i, int j) const { return n_icellq[(size_t)(j - 1) * (NUMQBC + 1) + i]; }
  inline double RDISQ(int i, int j) const { return rdisq[(size_t)(j - 1) * (NUMQBC + 1) + i]; }
  inline double VQDIST(int i, int k) const { return vqdist[(size_t)(k - 1) * (NUMQBC + 1) + i]; }
  inline double APT(int i, int j) const { return t_apt[(size_t)(j - 1) * (IOBCN + 1) + i]; }
  inline double PHAI(int i, int j) const { return t_phai[(size_t)(j - 1) * (IOBCN + 1) + i]; }

  bool is_river_node(int i) const {
    // FCT_* skip list (fct_t.F:60-69)
    for (int j = 1; j <= NUMQBC; ++j) {
      if (P.river_location == 0) {
        if (i == inodeq[j]) return true;
      } else {
        if (i == N_ICELLQ(j, 1) || i == N_ICELLQ(j, 2)) return true;
      }
    }
    return false;
  }
  bool is_obc_node(int i) const {
    for (int j = 1; j <= IOBCN; ++j)
      if (i == i_obc_n[j]) return true;
    return false;
  }

  // =====================================================================================
  // N2E2D / N2E3D / E2N2D (mod_main.F:1633-1683)
  // =====================================================================================
  void n2e2d(const std::vector<double>& nvar, std::vector<double>& evar) {
    for (int i = 1; i <= N; ++i)
      evar[i] = ONE_THIRD * (nvar[NV(i, 1)] + nvar[NV(i, 2)] + nvar[NV(i, 3)]);
  }
  void n2e3d(const std::vector<double>& nvar, std::vector<double>& evar) {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= KB; ++k)
      for (int i = 1; i <= N; ++i)
        evar[c3(i, k)] = ONE_THIRD * (nvar[n3(NV(i, 1), k)] + nvar[n3(NV(i, 2), k)] + nvar[n3(NV(i, 3), k)]);
  }
  void e2n2d(const std::vector<double>& evar, std::vector<double>& nvar) {
    for (int i = 1; i <= M; ++i) {
      double s = 0.0;
      for (int j = 1; j <= ntve[i]; ++j) s = s + evar[NBVE(i, j)];
      nvar[i] = s / (double)(float)ntve[i];
    }
  }

  // =====================================================================================
  // EXTEL_EDGE(K) (extel_edge.F:32-229)
  // =====================================================================================
  void extel_edge(int K) {
    std::vector<double> xflux(M1, 0.0);
    for (int i = 1; i <= NCV; ++i) {
      int i1 = ntrg[i];
      int ia = NIEC(i, 1);
      int ib = NIEC(i, 2);
      double dij = d1[i1];
      double uij = ua[i1];
      double vij = va[i1];
      double exflux = dij * (-uij * dltye[i] + vij * dltxe[i]);
      xflux[ia] = xflux[ia] - exflux;
      xflux[ib] = xflux[ib] + exflux;
    }
    for (int i = 1; i <= IOBCN; ++i) {
      xflux_obcn[i] = xflux[i_obc_n[i]];
      xflux[i_obc_n[i]] = 0.0;
    }
    if (NUMQBC >= 1) {
      if (P.river_location == 0) {
        for (int j = 1; j <= NUMQBC; ++j) {
          int jj = inodeq[j];
          xflux[jj] = xflux[jj] - qdis[j];
        }
      } else {
        for (int j = 1; j <= NUMQBC; ++j) {
          int j1 = N_ICELLQ(j, 1), j2 = N_ICELLQ(j, 2);
          xflux[j1] = xflux[j1] - qdis[j] * RDISQ(j, 1);
          xflux[j2] = xflux[j2] - qdis[j] * RDISQ(j, 2);
        }
      }
    }
    double dtk = ALPHA_RK[K] * P.dte;
    for (int i = 0; i <= M; ++i) elf[i] = elrk[i] - dtk * xflux[i] / art1[i];
  }

  // =====================================================================================
  // BCOND_GCN(1,K) -> BCOND_ASL, BCOND_ASL_CLP (mod_obcs.F:509-617) and the RK blend on
  // the specified-elevation nodes (external_step.F:262-266).
  // =====================================================================================
  void bcond_elf(int K) {
    double rktime = ExtTime + P.dte * (ALPHA_RK[K] - 1.0);
    if (P.obc_elevation_forcing_on) {
      double te = rktime - P.tide_ref_time;
      for (size_t ii = 0; ii < obc_lst1.size(); ++ii) {
        int I = (int)ii + 1;
        int jn = obc_lst1[ii];
        int node = i_obc_n[jn];
        double force = 0.0;
        for (int j = 1; j <= NTIDE; ++j) {
          double phai_ij = PHAI(jn, j) * PI2 / 360.0;
          double time_flt = te * PI2 / t_period[j - 1];
          force = APT(jn, j) * std::cos(time_flt - phai_ij) + force;
        }
        force = force + t_emean[jn];
        elf[node] = force * RAMP;
        (void)I;
      }
    }
    for (size_t ii = 0; ii < obc_lst2.size(); ++ii) elf[i_obc_n[obc_lst2[ii]]] = 0.0;
    for (size_t ii = 0; ii < obc_lst1.size(); ++ii) {
      int j = i_obc_n[obc_lst1[ii]];
      elf[j] = elrk[j] + ALPHA_RK[K] * (elf[j] - elrk[j]);
    }
  }

  // =====================================================================================
  // WET_JUDGE (mod_wd.F:193-284)
  // =====================================================================================
  void wet_judge() {
    for (int i = 0; i <= M; ++i) iswetn[i] = 1;
    for (int i = 1; i <= M; ++i) {
      double dtmp = h[i] + elf[i];
      if ((dtmp - P.min_depth) < 1.0e-5) iswetn[i] = 0;
    }
    for (int i = 0; i <= N; ++i) iswetc[i] = 1;
    for (int i = 1; i <= N; ++i) {
      double dtmp = std::max(std::max(elf[NV(i, 1)], elf[NV(i, 2)]), elf[NV(i, 3)]) +
                    std::min(std::min(h[NV(i, 1)], h[NV(i, 2)]), h[NV(i, 3)]);
      if ((dtmp - P.min_depth) < 1.0e-5) iswetc[i] = 0;
    }
    for (int i = 1; i <= M; ++i) {
      int s = 0;
      for (int j = 1; j <= ntve[i]; ++j) s += iswetc[NBVE(i, j)];
      if (s == 0) iswetn[i] = 0;
    }
    for (int i = 0; i <= M; ++i) elf[i] = std::max(elf[i], -h[i] + P.min_depth);
    for (int i = 1; i <= N; ++i) elf1[i] = ONE_THIRD * (elf[NV(i, 1)] + elf[NV(i, 2)] + elf[NV(i, 3)]);
  }

  // =====================================================================================
  // FLUX_OBN(K) (mod_obcs.F:1181-1215)
  // =====================================================================================
  void flux_obn(int K) {
    for (int i = 1; i <= N; ++i) fluxobn[i] = 0.0;
    for (int i = 1; i <= IOBCN; ++i) {
      int j = i_obc_n[i];
      double flux = -(elf[j] - elrk[j]) * art1[j] / (ALPHA_RK[K] * P.dte) - xflux_obcn[i];
      if (nadjc_obc[i] > 0) {
        int c1 = ADJC(i, 1);
        fluxobn[c1] = fluxobn[c1] + FLUXF(i, 1) * flux;
      }
      if (nadjc_obc[i] > 1) {
        int c2 = ADJC(i, 2);
        fluxobn[c2] = fluxobn[c2] + FLUXF(i, 2) * flux;
      }
    }
  }

  // =====================================================================================
  // ADVAVE_EDGE_GCN(XFLUX,YFLUX), LIMITED_NO branch (advave_edge_gcn.F:32-1145)
  // =====================================================================================
  // Velocity of neighbour j (1..3) of cell c for the least-squares gradient.  GCN: the
  // neighbour's value (the ghost cell 0 holds zero).  GCY where the neighbour is missing:
  // GHOSTUV2/GHOSTUV3 (ghostuv.F:32-223), the cell's velocity projected on the boundary
  // edge opposite node j, or, on an open-boundary cell, the cell's own velocity.
  inline void nbr_uv(const double* U, const double* V, int c, int j, double& uk, double& vk) const {
    const int k = NBE(c, j);
    if (!P.ghost_cells || k != 0) {
      uk = U[k];
      vk = V[k];
      return;
    }
    if (isbce[c] != 2) {
      const int J1 = nxt(j), J2 = nxt2(j);
      const double deltx = vx[NV(c, J1)] - vx[NV(c, J2)];
      const double delty = vy[NV(c, J1)] - vy[NV(c, J2)];
      const double a = std::atan2(delty, deltx);
      const double ca = std::cos(a), sa = std::sin(a);
      const double utmp = U[c] * ca + V[c] * sa;
      const double vtmp = 0.0;
      uk = utmp * ca - vtmp * sa;
      vk = utmp * sa + vtmp * ca;
    } else {
      uk = U[c];
      vk = V[c];
    }
  }
  // COFA1, COFA2 (U) and COFA5, COFA6 (V) of cell c (advave_edge_gcn.F:634-637).
  inline void cofa(const double* U, const double* V, int c, double& c1, double& c2, double& c5, double& c6) const {
    double u1, v1, u2, v2, u3, v3;
    nbr_uv(U, V, c, 1, u1, v1);
    nbr_uv(U, V, c, 2, u2, v2);
    nbr_uv(U, V, c, 3, u3, v3);
    c1 = A1U(c, 1) * U[c] + A1U(c, 2) * u1 + A1U(c, 3) * u2 + A1U(c, 4) * u3;
    c2 = A2U(c, 1) * U[c] + A2U(c, 2) * u1 + A2U(c, 3) * u2 + A2U(c, 4) * u3;
    c5 = A1U(c, 1) * V[c] + A1U(c, 2) * v1 + A1U(c, 3) * v2 + A1U(c, 4) * v3;
    c6 = A2U(c, 1) * V[c] + A2U(c, 2) * v1 + A2U(c, 3) * v2 + A2U(c, 4) * v3;
  }

  // Phase one of the limited schemes (advave_edge_gcn.F:141-318, advection_edge_gcn.F:
  // 118-259, adv_uv_edge_gcn.F:152-330): per cell the smallest, over its wet edges, of
  // |U(IA)-U(IB)| / |U'+EPSILON|, at most 1, where U' = COFA1*XIJ + COFA2*YIJ is the
  // cell's gradient extrapolation to the edge.  wet(c) is the routine's wet flag product.
  template <class Wet>
  void limiter_alfa(const double* U, const double* V, Wet wet, std::vector<double>& ualfa,
                    std::vector<double>& valfa) const {
    const double eps = 2.220446049250313e-16;  // EPSILON of the reference's REAL(SP) = REAL(DP)
    ualfa.assign(N1, 1.0);
    valfa.assign(N1, 1.0);
    auto lim = [&](double num, double ext, double& a) {
      double t = num / std::fabs(ext + eps);
      if (t > 1) t = 1.0;
      a = t < a ? t : a;
    };
    for (int i = 1; i <= NE; ++i) {
      int ia = IEC(i, 1), ib = IEC(i, 2);
      if (!(wet(ia) || wet(ib))) continue;
      for (int side = 0; side < 2; ++side) {
        int c = side == 0 ? ia : ib;
        int k1 = NBE(c, 1), k2 = NBE(c, 2), k3 = NBE(c, 3);
        double cofa1, cofa2, cofa5, cofa6;
        cofa(U, V, c, cofa1, cofa2, cofa5, cofa6);
        double xij = xijc[i] - xc[c], yij = yijc[i] - yc[c];
        lim(std::fabs(U[ia] - U[ib]), cofa1 * xij + cofa2 * yij, ualfa[c]);
        lim(std::fabs(V[ia] - V[ib]), cofa5 * xij + cofa6 * yij, valfa[c]);
      }
    }
  }
  // Face values of one edge: unlimited, U + COFA1*XIJ + COFA2*YIJ; limited, U + ALFA*(COFA1*
  // XIJ + COFA2*YIJ), and under LIMITED_1 both faces reset to the cell values when either
  // leaves their range.
  void face_values(double ua_, double ub_, double ca1, double ca2, double xa, double ya, double cb1,
                   double cb2, double xb, double yb, double alfa_a, double alfa_b, double& f1,
                   double& f2) const {
    if (P.limiter == 0) {
      f1 = ua_ + ca1 * xa + ca2 * ya;
      f2 = ub_ + cb1 * xb + cb2 * yb;
      return;
    }
    f1 = ua_ + alfa_a * (ca1 * xa + ca2 * ya);
    f2 = ub_ + alfa_b * (cb1 * xb + cb2 * yb);
    if (P.limiter == 1) {
      double hi = std::max(ua_, ub_), lo = std::min(ua_, ub_);
      if (f1 > hi || f1 < lo || f2 > hi || f2 < lo) {
        f1 = ua_;
        f2 = ub_;
      }
    }
  }

  void advave(std::vector<double>& xflux, std::vector<double>& yflux) {
    double fact = P.horizontal_mixing == 0 ? 1.0 : 0.0;
    double fm1 = P.horizontal_mixing == 0 ? 0.0 : 1.0;
    for (int i = 0; i <= N; ++i) { xflux[i] = 0.0; yflux[i] = 0.0; pstx[i] = 0.0; psty[i] = 0.0; }
    std::vector<double> ualfa, valfa;
    if (P.limiter) limiter_alfa(ua.data(), va.data(), [&](int c) { return iswetce[c] * iswetc[c] == 1; }, ualfa, valfa);
    for (int i = 1; i <= NE; ++i) {
      int ia = IEC(i, 1), ib = IEC(i, 2);
      int j1 = IENODE(i, 1), j2 = IENODE(i, 2);
      double dij = 0.5 * (d[j1] + d[j2]);
      double elij = 0.5 * (el[j1] + el[j2]);
      if (iswetce[ia] * iswetc[ia] == 1 || iswetce[ib] * iswetc[ib] == 1) {
        double cofa1, cofa2, cofa5, cofa6;
        cofa(ua.data(), va.data(), ia, cofa1, cofa2, cofa5, cofa6);
        double xija = xijc[i] - xc[ia];
        double yija = yijc[i] - yc[ia];
        double cofa3, cofa4, cofa7, cofa8;
        cofa(ua.data(), va.data(), ib, cofa3, cofa4, cofa7, cofa8);
        double xijb = xijc[i] - xc[ib];
        double yijb = yijc[i] - yc[ib];
        const bool L = P.limiter != 0;
        double uij1, uij2, vij1, vij2;
        face_values(ua[ia], ua[ib], cofa1, cofa2, xija, yija, cofa3, cofa4, xijb, yijb, L ? ualfa[ia] : 1.0,
                    L ? ualfa[ib] : 1.0, uij1, uij2);
        face_values(va[ia], va[ib], cofa5, cofa6, xija, yija, cofa7, cofa8, xijb, yijb, L ? valfa[ia] : 1.0,
                    L ? valfa[ib] : 1.0, vij1, vij2);
        double uij = 0.5 * (uij1 + uij2);
        double vij = 0.5 * (vij1 + vij2);
        double un = -uij * dltyc[i] + vij * dltxc[i];
        double viscof1 = art[ia] * std::sqrt(cofa1 * cofa1 + cofa6 * cofa6 + 0.5 * ((cofa2 + cofa5) * (cofa2 + cofa5)));
        double viscof2 = art[ib] * std::sqrt(cofa3 * cofa3 + cofa8 * cofa8 + 0.5 * ((cofa4 + cofa7) * (cofa4 + cofa7)));
        double viscof = (fact * 0.5 * (viscof1 * cc_hvc[ia] + viscof2 * cc_hvc[ib]) +
                         fm1 * 0.5 * (cc_hvc[ia] + cc_hvc[ib])) / P.hprnu;
        double txx = (cofa1 + cofa3) * viscof;
        double tyy = (cofa6 + cofa8) * viscof;
        double txy = 0.5 * (cofa2 + cofa4 + cofa5 + cofa7) * viscof;
        double fxx = dij * (txx * dltyc[i] - txy * dltxc[i]);
        double fyy = dij * (txy * dltyc[i] - tyy * dltxc[i]);
        double sg = fsign1(un);
        double xadv = dij * un * ((1.0 - sg) * uij2 + (1.0 + sg) * uij1) * 0.5;
        double yadv = dij * un * ((1.0 - sg) * vij2 + (1.0 + sg) * vij1) * 0.5;
        double nb = 1.0 - (double)isbc[i];
        xflux[ia] = xflux[ia] + (xadv + fxx * epor[ia]) * nb * iucp[ia];
        yflux[ia] = yflux[ia] + (yadv + fyy * epor[ia]) * nb * iucp[ia];
        xflux[ib] = xflux[ib] - (xadv + fxx * epor[ib]) * nb * iucp[ib];
        yflux[ib] = yflux[ib] - (yadv + fyy * epor[ib]) * nb * iucp[ib];
      }
      pstx[ia] = pstx[ia] - grav_e[ia] * d1[ia] * elij * dltyc[i];
      psty[ia] = psty[ia] + grav_e[ia] * d1[ia] * elij * dltxc[i];
      pstx[ib] = pstx[ib] + grav_e[ib] * d1[ib] * elij * dltyc[i];
      psty[ib] = psty[ib] - grav_e[ib] * d1[ib] * elij * dltxc[i];
    }
    for (int i = 1; i <= N; ++i) {
      double w_ = (double)(iswetce[i] * iswetc[i]);
      xflux[i] = xflux[i] * w_;
      yflux[i] = yflux[i] * w_;
    }
    for (int i = 1; i <= N; ++i) {
      if (isbce[i] == 2) {
        if (P.ghost_cells) {  // advave_edge_gcy.F
          xflux[i] = xflux[i] + fluxobn[i] * ua[i] * iucp[i];
          yflux[i] = yflux[i] + fluxobn[i] * va[i] * iucp[i];
        } else {
          xflux[i] = (xflux[i] + fluxobn[i] * ua[i]) * iucp[i];
          yflux[i] = (yflux[i] + fluxobn[i] * va[i]) * iucp[i];
        }
      }
    }
    if (NUMQBC > 0) {
      if (P.river_location == 0) {
        for (int k = 1; k <= NUMQBC; ++k) {
          int j = inodeq[k];
          int i1 = NBVE(j, 1), i2 = NBVE(j, ntve[j]);
          double vlctyq = qdis[k] / qarea[k];
          double ca = std::cos(angleq[k]), sa = std::sin(angleq[k]);
          xflux[i1] = xflux[i1] - 0.5 * qdis[k] * vlctyq * ca;
          yflux[i1] = yflux[i1] - 0.5 * qdis[k] * vlctyq * sa;
          xflux[i2] = xflux[i2] - 0.5 * qdis[k] * vlctyq * ca;
          yflux[i2] = yflux[i2] - 0.5 * qdis[k] * vlctyq * sa;
        }
      } else {
        for (int k = 1; k <= NUMQBC; ++k) {
          int i1 = icellq[k];
          double vlctyq = qdis[k] / qarea[k];
          double temp = qdis[k] * vlctyq;
          xflux[i1] = xflux[i1] - temp * std::cos(angleq[k]);
          yflux[i1] = yflux[i1] - temp * std::sin(angleq[k]);
        }
      }
    }
  }

  // =====================================================================================
  // EXTUV_EDGE(K) (extuv_edge.F:33-196)
  // =====================================================================================
  void extuv_edge(int K) {
    double uaft = uaf[0], vaft = vaf[0];
    h1[0] = h1[1];
    for (int i = 1; i <= N; ++i) {
      if (iswetce[i] * iswetc[i] == 1) {
        double resx = adx2d[i] + advua[i] + drx2d[i] + pstx[i] - cor[i] * va[i] * d1[i] * art[i] -
                      (wusurf2[i] + wubot[i]) * art[i];
        double resy = ady2d[i] + advva[i] + dry2d[i] + psty[i] + cor[i] * ua[i] * d1[i] * art[i] -
                      (wvsurf2[i] + wvbot[i]) * art[i];
        uaf[i] = (uark[i] * (h1[i] + elrk1[i]) - ALPHA_RK[K] * P.dte * resx / art[i]) / (h1[i] + elf1[i]);
        vaf[i] = (vark[i] * (h1[i] + elrk1[i]) - ALPHA_RK[K] * P.dte * resy / art[i]) / (h1[i] + elf1[i]);
      } else {
        uaf[i] = 0.0;
        vaf[i] = 0.0;
      }
    }
    vaf[0] = vaft;
    uaf[0] = uaft;
    for (int i = 0; i <= N; ++i) {
      uaf[i] = uaf[i] / (1.0 + cc_sponge[i] * (uaf[i] * uaf[i]));
      vaf[i] = vaf[i] / (1.0 + cc_sponge[i] * (vaf[i] * vaf[i]));
    }
  }

  // River clamp shared by BCOND_GCN cases 2, 3 and 5: returns true when cell i is a river
  // cell and its velocity was clamped (bcond_gcn.F:347-376).
  bool river_clamp(int i, double& uu, double& vv) {
    if (NUMQBC <= 0) return false;
    for (int j = 1; j <= NUMQBC; ++j) {
      bool hit;
      if (P.river_location == 0) {
        int i1 = inodeq[j];
        int j1 = NBVE(i1, 1), j2 = NBVE(i1, ntve[i1]);
        hit = (i == j1) || (i == j2);
      } else {
        hit = (i == icellq[j]);
      }
      if (hit) {
        double ca = std::cos(angleq[j]), sa = std::sin(angleq[j]);
        double untmp = uu * ca + vv * sa;
        double vntmp = -uu * sa + vv * ca;
        untmp = std::max(untmp, 0.0);
        uu = untmp * ca - vntmp * sa;
        vv = untmp * sa + vntmp * ca;
        return true;
      }
    }
    return false;
  }
  inline void tangential(int i, double& uu, double& vv) {
    double sa = std::sin(alpha[i]), ca = std::cos(alpha[i]);
    double ui = uu * (sa * sa) - vv * sa * ca;
    double vi = -uu * sa * ca + vv * (ca * ca);
    uu = ui;
    vv = vi;
  }

  // BCOND_GCN(2,K) (bcond_gcn.F:325-406)
  void bcond_uv2d() {
    for (int i = 1; i <= N; ++i) {
      // GCY (bcond_gcy.F): river clamp only, no tangential projection, no corner zero
      if (isbce[i] == 3 && !P.ghost_cells) { uaf[i] = 0.0; vaf[i] = 0.0; }
      if (isbce[i] == 1) {
        if (!river_clamp(i, uaf[i], vaf[i]) && !P.ghost_cells) tangential(i, uaf[i], vaf[i]);
      }
    }
  }

  // external_step.F:333-436 after BCOND_GCN(2,K)
  void ext_update(int K) {
    for (int i = 0; i <= M; ++i) el[i] = elf[i];
    for (int i = 0; i <= N; ++i) el1[i] = elf1[i];
    n2e2d(el, el1);
    for (int i = 0; i <= M; ++i) d[i] = h[i] + el[i];
    for (int i = 0; i <= N; ++i) { d1[i] = h1[i] + el1[i]; ua[i] = uaf[i]; va[i] = vaf[i]; }
    for (int i = 0; i <= M; ++i) dtfa[i] = d[i];
    if (K == 3) {
      for (int i = 0; i <= N; ++i) { uard[i] = uard[i] + ua[i] * d1[i]; vard[i] = vard[i] + va[i] * d1[i]; }
      for (int i = 0; i <= M; ++i) egf[i] = egf[i] + el[i] / (double)P.isplit;
    }
    if (K == 4 && IOBCN > 0) {
      for (int i = 1; i <= IOBCN; ++i) {
        int j = i_obc_n[i];
        double tmp = -(elf[j] - elrk[j]) * art1[j] / P.dte - xflux_obcn[i];
        uard_obcn[i] = uard_obcn[i] + tmp / (double)(float)P.isplit;
      }
    }
    if (P.wetting_drying_on)
      for (int i = 0; i <= N; ++i) iswetce[i] = iswetc[i];
  }

  // BCOND_GCN(9,0): external-mode wind (bcond_gcn.F:877-897)
  void bcond9() {
    if (!have_wind) return;
    for (int i = 0; i <= N; ++i) {
      wusurf2[i] = wsx[i] * RAMP * 0.001;
      wvsurf2[i] = wsy[i] * RAMP * 0.001;
    }
  }

  // =====================================================================================
  // EXTERNAL_STEP (external_step.F:30-443)
  // =====================================================================================
  void ext_stage(int K) {
    extel_edge(K);
    bcond_elf(K);
    n2e2d(elf, elf1);
    if (P.wetting_drying_on) wet_judge();
    flux_obn(K);
    advave(advua, advva);
    extuv_edge(K);
    bcond_uv2d();
    ext_update(K);
  }
  void external_step(int iext) {
    if (P.iramp != 0) {
      double tmp = (double)(IINT - 1) + (double)iext / (double)P.isplit;
      RAMP = std::tanh(tmp / (double)P.iramp);
    } else {
      RAMP = 1.0;
    }
    bcond9();
    elrk1 = el1;
    elrk = el;
    uark = ua;
    vark = va;
    for (int K = 1; K <= 4; ++K) ext_stage(K);
  }

  // =====================================================================================
  // ADJUST2D3D (adjust2d3d.F:29-115)
  // =====================================================================================
  void adjust2d3d(int type) {
    if (type == 1) {
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= N; ++i) {
        double uac = 0.0, vac = 0.0;
        for (int k = 1; k <= KBM1; ++k) uac = uac + u[c3(i, k)] * dz1[c3(i, k)];
        for (int k = 1; k <= KBM1; ++k) vac = vac + v[c3(i, k)] * dz1[c3(i, k)];
        for (int k = 1; k <= KBM1; ++k) u[c3(i, k)] = u[c3(i, k)] + 1.0 * (ua[i] - uac);
        for (int k = 1; k <= KBM1; ++k) v[c3(i, k)] = v[c3(i, k)] + 1.0 * (va[i] - vac);
      }
    } else {
      for (int i = 0; i <= N; ++i) {
        uard[i] = uard[i] / (double)(float)P.isplit;
        vard[i] = vard[i] / (double)(float)P.isplit;
      }
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= N; ++i) {
        if (iswetct[i] * iswetc[i] == 1) {
          double utmp = 0.0, vtmp = 0.0;
          for (int k = 1; k <= KBM1; ++k) {
            utmp = utmp + u[c3(i, k)] * dz1[c3(i, k)];
            vtmp = vtmp + v[c3(i, k)] * dz1[c3(i, k)];
          }
          utmp = utmp * dt1[i];
          vtmp = vtmp * dt1[i];
          for (int k = 1; k <= KBM1; ++k) {
            u[c3(i, k)] = u[c3(i, k)] - (utmp - uard[i]) / dt1[i];
            v[c3(i, k)] = v[c3(i, k)] - (vtmp - vard[i]) / dt1[i];
          }
        }
      }
    }
  }

  // BCOND_GCN(5,0) on U/V and BCOND_GCN(3,0) on UF/VF (bcond_gcn.F:424-611)
  void bcond_uv3d(std::vector<double>& uu, std::vector<double>& vv) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = c3(i, k);
        if (isbce[i] == 3 && !P.ghost_cells) { uu[q] = 0.0; vv[q] = 0.0; }
        if (isbce[i] == 1) {
          if (!river_clamp(i, uu[q], vv[q]) && !P.ghost_cells) tangential(i, uu[q], vv[q]);
        }
      }
    }
  }

  // BCOND_GCN(8,0): internal-mode river ramp and wind (bcond_gcn.F:624-683)
  void bcond8() {
    for (int j = 1; j <= NUMQBC; ++j) qdis[j] = qdis0[j] * RAMP;
    if (have_wind) {
      for (int i = 0; i <= N; ++i) {
        wusurf[i] = -wsx[i] * RAMP * 0.001;
        wvsurf[i] = -wsy[i] * RAMP * 0.001;
      }
    }
    // HEATING_ON (bcond_gcn.F:683-694): W/m^2 times RAMP over -SPCP*ROSEA
    if (P.heating_on) {
      const double SPCP = 4.2174E3, ROSEA = 1.023E3, SPRO = SPCP * ROSEA;
      for (int i = 0; i <= M; ++i) {
        wtsurf[i] = -(wtsurf_w[i] * RAMP) / SPRO;
        swrad[i] = -(swrad_w[i] * RAMP) / SPRO;
      }
    }
  }

  // =====================================================================================
  // BOTTOM_ROUGHNESS, BR_ORIG (brough.F:41-214)
  // =====================================================================================
  void bottom_roughness() {
    const double VK2 = 0.160;
    for (int i = 1; i <= N; ++i) {
      double zb = zz1[c3(i, KBM1)] - z1[c3(i, KB)];
      if (dt1[i] > 3.0) {
        double lg = std::log(zb * dt1[i] / cc_z0b[i]);
        cbc[i] = VK2 / (lg * lg);
      } else {
        double lg = std::log(zb * 3.0 / cc_z0b[i]);
        cbc[i] = VK2 / (lg * lg);
      }
    }
    for (int i = 0; i <= N; ++i)
      if (cbc[i] < P.cbcmin) cbc[i] = P.cbcmin;
    for (int i = 1; i <= N; ++i) {
      double ub = u[c3(i, KBM1)], vb = v[c3(i, KBM1)];
      double btps = cbc[i] * std::sqrt(ub * ub + vb * vb);
      wubot[i] = -btps * ub;
      wvbot[i] = -btps * vb;
      double cff = 0.75 * dz1[c3(i, KBM1)] * d1[i];
      wubot[i] = fsign(1.0, wubot[i]) * std::min(std::fabs(wubot[i]), std::fabs(ub * cff / DTI));
      wvbot[i] = fsign(1.0, wvbot[i]) * std::min(std::fabs(wvbot[i]), std::fabs(vb * cff / DTI));
    }
    for (int i = 0; i <= N; ++i) taubm[i] = std::sqrt(wubot[i] * wubot[i] + wvbot[i] * wvbot[i]);
    e2n2d(wubot, wubot_n);
    e2n2d(wvbot, wvbot_n);
    for (int i = 0; i <= M; ++i) taubm_n[i] = std::sqrt(wubot_n[i] * wubot_n[i] + wvbot_n[i] * wvbot_n[i]);
  }

  // =====================================================================================
  // ADVECTION_EDGE_GCN (advection_edge_gcn.F:30-733).  The reference loops edges outer,
  // layers inner; each (target, layer) still sums its edges in ascending order when the
  // layer loop is outermost, so the layer loop is hoisted for OpenMP.
  // =====================================================================================
  void advection3d() {
    double fact = P.horizontal_mixing == 0 ? 1.0 : 0.0;
    double fm1 = P.horizontal_mixing == 0 ? 0.0 : 1.0;
    std::fill(advx.begin(), advx.end(), 0.0);
    std::fill(advy.begin(), advy.end(), 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 1; k <= KBM1; ++k) {
      std::vector<double> ualfa, valfa;
      if (P.limiter)
        limiter_alfa(&u[c3(0, k)], &v[c3(0, k)], [&](int c) { return iswetct[c] * iswetc[c] == 1; }, ualfa, valfa);
      const bool L = P.limiter != 0;
      for (int i = 1; i <= NE; ++i) {
        int ia = IEC(i, 1), ib = IEC(i, 2);
        if (!(iswetct[ia] * iswetc[ia] == 1 || iswetct[ib] * iswetc[ib] == 1)) continue;
        int j1 = IENODE(i, 1), j2 = IENODE(i, 2);
        int k1 = NBE(ia, 1), k2 = NBE(ia, 2), k3 = NBE(ia, 3);
        int k4 = NBE(ib, 1), k5 = NBE(ib, 2), k6 = NBE(ib, 3);
        double xija = xijc[i] - xc[ia], yija = yijc[i] - yc[ia];
        double xijb = xijc[i] - xc[ib], yijb = yijc[i] - yc[ib];
        double dij = 0.5 * (dt[j1] * dz[n3(j1, k)] + dt[j2] * dz[n3(j2, k)]);
        const double *U_ = &u[c3(0, k)], *V_ = &v[c3(0, k)];
        double cofa1, cofa2, cofa5, cofa6;
        cofa(U_, V_, ia, cofa1, cofa2, cofa5, cofa6);
        double cofa3, cofa4, cofa7, cofa8;
        cofa(U_, V_, ib, cofa3, cofa4, cofa7, cofa8);
        double uij1, uij2, vij1, vij2;
        face_values(U_[ia], U_[ib], cofa1, cofa2, xija, yija, cofa3, cofa4, xijb, yijb, L ? ualfa[ia] : 1.0,
                    L ? ualfa[ib] : 1.0, uij1, uij2);
        face_values(V_[ia], V_[ib], cofa5, cofa6, xija, yija, cofa7, cofa8, xijb, yijb, L ? valfa[ia] : 1.0,
                    L ? valfa[ib] : 1.0, vij1, vij2);
        double uij = 0.5 * (uij1 + uij2);
        double vij = 0.5 * (vij1 + vij2);
        double un = vij * dltxc[i] - uij * dltyc[i];
        double viscof1 = art[ia] * std::sqrt(cofa1 * cofa1 + cofa6 * cofa6 + 0.5 * ((cofa2 + cofa5) * (cofa2 + cofa5)));
        double viscof2 = art[ib] * std::sqrt(cofa3 * cofa3 + cofa8 * cofa8 + 0.5 * ((cofa4 + cofa7) * (cofa4 + cofa7)));
        double viscof = (fact * 0.5 * (viscof1 * cc_hvc[ia] + viscof2 * cc_hvc[ib]) +
                         fm1 * 0.5 * (cc_hvc[ia] + cc_hvc[ib])) / P.hprnu;
        double txx = (cofa1 + cofa3) * viscof;
        double tyy = (cofa6 + cofa8) * viscof;
        double txy = 0.5 * (cofa2 + cofa4 + cofa5 + cofa7) * viscof;
        double fxx = dij * (txx * dltyc[i] - txy * dltxc[i]);
        double fyy = dij * (txy * dltyc[i] - tyy * dltxc[i]);
        double sg = fsign1(un);
        double xadv = dij * un * ((1.0 - sg) * uij2 + (1.0 + sg) * uij1) * 0.5;
        double yadv = dij * un * ((1.0 - sg) * vij2 + (1.0 + sg) * vij1) * 0.5;
        double isb = (double)isbc[i];
        double tpa = (double)(float)(1 - isbc[i]) * epor[ia];
        double tpb = (double)(float)(1 - isbc[i]) * epor[ib];
        double *X = &advx[c3(0, k)], *Y = &advy[c3(0, k)];
        if (P.ghost_cells) {  // advection_edge_gcy.F: the viscous flux masked like the advective
          X[ia] = X[ia] + xadv * tpa + fxx * tpa;
          Y[ia] = Y[ia] + yadv * tpa + fyy * tpa;
          X[ib] = X[ib] - xadv * tpb - fxx * tpb;
          Y[ib] = Y[ib] - yadv * tpb - fyy * tpb;
        } else {
          X[ia] = X[ia] + xadv * tpa + (fxx + 3.0 * fxx * isb) * epor[ia];
          Y[ia] = Y[ia] + yadv * tpa + (fyy + 3.0 * fyy * isb) * epor[ia];
          X[ib] = X[ib] - xadv * tpb - (fxx + 3.0 * fxx * isb) * epor[ib];
          Y[ib] = Y[ib] - yadv * tpb - (fyy + 3.0 * fyy * isb) * epor[ib];
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      double w_ = (double)(iswetct[i] * iswetc[i]);
      for (int k = 1; k <= KBM1; ++k) {
        advx[c3(i, k)] = advx[c3(i, k)] * w_;
        advy[c3(i, k)] = advy[c3(i, k)] * w_;
      }
      if (isbce[i] == 2)
        for (int k = 1; k <= KBM1; ++k) { advx[c3(i, k)] = 0.0; advy[c3(i, k)] = 0.0; }
    }
    river_momentum3d(advx, advy);
  }

  // River momentum source on the 3-D fluxes (advection_edge_gcn.F:674-708,
  // adv_uv_edge_gcn.F:1037-1074).
  void river_momentum3d(std::vector<double>& X, std::vector<double>& Y) {
    if (NUMQBC <= 0) return;
    if (P.river_location == 0) {
      for (int ii = 1; ii <= NUMQBC; ++ii) {
        int j = inodeq[ii];
        int i1 = NBVE(j, 1), i2 = NBVE(j, ntve[j]);
        for (int k = 1; k <= KBM1; ++k) {
          double vlctyq = qdis[ii] / qarea[ii];
          double temp = 0.5 * qdis[ii] * VQDIST(ii, k) * VQDIST(ii, k) * vlctyq / dz[n3(j, k)];
          double ca = std::cos(angleq[ii]), sa = std::sin(angleq[ii]);
          X[c3(i1, k)] = X[c3(i1, k)] - temp * ca;
          X[c3(i2, k)] = X[c3(i2, k)] - temp * ca;
          Y[c3(i1, k)] = Y[c3(i1, k)] - temp * sa;
          Y[c3(i2, k)] = Y[c3(i2, k)] - temp * sa;
        }
      }
    } else {
      for (int ii = 1; ii <= NUMQBC; ++ii) {
        int i1 = icellq[ii];
        for (int k = 1; k <= KBM1; ++k) {
          double vlctyq = qdis[ii] / qarea[ii];
          double temp = qdis[ii] * VQDIST(ii, k) * VQDIST(ii, k) * vlctyq / dz1[c3(i1, k)];
          X[c3(i1, k)] = X[c3(i1, k)] - temp * std::cos(angleq[ii]);
          Y[c3(i1, k)] = Y[c3(i1, k)] - temp * std::sin(angleq[ii]);
        }
      }
    }
  }

  // =====================================================================================
  // BAROPG, sigma levels (baropg.F:33-166)
  // =====================================================================================
  // SINTER_EXTRP_DOWN (sinter.F): B(I) from A over the descending abscissae X(1..M1): A(1)
  // above X(1), linear extrapolation of the last two below X(M1), else linear
  // interpolation in the last interval J (of all J = 1..M1-1) with X(J+1) <= Y <= X(J).
  static void sinter_extrp_down(const double* X, const double* A, const double* Y, double* B, int M1, int N1) {
    for (int i = 0; i < N1; ++i) {
      if (Y[i] > X[0]) B[i] = A[0];
      if (Y[i] < X[M1 - 1]) B[i] = A[M1 - 1] + (A[M1 - 2] - A[M1 - 1]) * (Y[i] - X[M1 - 1]) / (X[M1 - 2] - X[M1 - 1]);
    }
    for (int i = 0; i < N1; ++i)
      for (int j = 0; j < M1 - 1; ++j)
        if (Y[i] <= X[j] && Y[i] >= X[j + 1]) B[i] = A[j] - (A[j] - A[j + 1]) * (X[j] - Y[i]) / (X[j] - X[j + 1]);
  }

  // PHY_BAROPG (phy_baropg.F:37-151): the baroclinic pressure gradient on 600 z levels of
  // HMAX/600, with RHO1 interpolated down each node column, integrated per cell edge and
  // interpolated back to the cell's sigma depths.
  void phy_baropg() {
    const int KBBM1 = 600;
    double hmax = h[1];
    for (int i = 2; i <= M; ++i) hmax = std::max(hmax, h[i]);
    const double deltz = hmax / (double)(float)KBBM1;
    std::vector<double> phy_z(KBBM1), rhoz((size_t)(M + 1) * KBBM1), sig_z((size_t)(M + 1) * KBM1);
    for (int k = 1; k <= KBBM1; ++k) phy_z[k - 1] = (0.5 - (double)(float)k) * deltz;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= M; ++i) {
      std::vector<double> sz(KBM1), rs(KBM1);
      for (int k = 1; k <= KBM1; ++k) {
        sig_z[(size_t)i * KBM1 + k - 1] = zz[n3(i, k)] * dt[i] + et[i];
        sz[k - 1] = sig_z[(size_t)i * KBM1 + k - 1];
        rs[k - 1] = rho1[n3(i, k)];
      }
      sinter_extrp_down(sz.data(), rs.data(), phy_z.data(), &rhoz[(size_t)i * KBBM1], KBM1, KBBM1);
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      int j1 = NV(i, 1), j2 = NV(i, 2), j3 = NV(i, 3);
      std::vector<double> pb1(KBBM1 + 1), pb2(KBBM1 + 1), pb3(KBBM1 + 1), pbxz(KBBM1), pbyz(KBBM1);
      std::vector<double> sz(KBM1), pbxs(KBM1), pbys(KBM1);
      int ntmp = 0;
      pb1[0] = pb2[0] = pb3[0] = 0.0;
      const double* r1 = &rhoz[(size_t)j1 * KBBM1];
      const double* r2 = &rhoz[(size_t)j2 * KBBM1];
      const double* r3 = &rhoz[(size_t)j3 * KBBM1];
      for (int k = 1; k <= KBBM1; ++k) {
        double tmp = (double)(float)k * deltz;
        if (h[j1] < tmp || h[j2] < tmp || h[j3] < tmp) {
          pb1[k] = pb2[k] = pb3[k] = 0.0;
        } else {
          double rz1 = 0.5 * (r2[k - 1] + r3[k - 1]);
          double rz2 = 0.5 * (r3[k - 1] + r1[k - 1]);
          double rz3 = 0.5 * (r1[k - 1] + r2[k - 1]);
          double g1 = 0.5 * (grav_n[j2] + grav_n[j3]);
          double g2 = 0.5 * (grav_n[j3] + grav_n[j1]);
          double g3 = 0.5 * (grav_n[j1] + grav_n[j2]);
          pb1[k] = pb1[k - 1] + g1 * rz1 * deltz;
          pb2[k] = pb2[k - 1] + g2 * rz2 * deltz;
          pb3[k] = pb3[k - 1] + g3 * rz3 * deltz;
          ntmp = ntmp + 1;
        }
      }
      double ax1 = (vy[j3] - vy[j2]) * deltz, ay1 = (vx[j2] - vx[j3]) * deltz;
      double ax2 = (vy[j1] - vy[j3]) * deltz, ay2 = (vx[j3] - vx[j1]) * deltz;
      double ax3 = (vy[j2] - vy[j1]) * deltz, ay3 = (vx[j1] - vx[j2]) * deltz;
      for (int k = 1; k <= KBBM1; ++k) {
        double px = ax1 * pb1[k] + ax2 * pb2[k] + ax3 * pb3[k];
        double py = ay1 * pb1[k] + ay2 * pb2[k] + ay3 * pb3[k];
        pbxz[k - 1] = px / art[i] / deltz;
        pbyz[k - 1] = py / art[i] / deltz;
      }
      for (int k = 1; k <= KBM1; ++k)
        sz[k - 1] = (sig_z[(size_t)j1 * KBM1 + k - 1] + sig_z[(size_t)j2 * KBM1 + k - 1] + sig_z[(size_t)j3 * KBM1 + k - 1]) / 3.;
      if (ntmp == 0) {
        for (int k = 0; k < KBM1; ++k) pbxs[k] = pbys[k] = 0.0;
      } else if (ntmp == 1) {
        for (int k = 0; k < KBM1; ++k) { pbxs[k] = pbxz[0]; pbys[k] = pbyz[0]; }
      } else {
        sinter_extrp_down(phy_z.data(), pbxz.data(), sz.data(), pbxs.data(), ntmp, KBM1);
        sinter_extrp_down(phy_z.data(), pbyz.data(), sz.data(), pbys.data(), ntmp, KBM1);
      }
      for (int k = 1; k <= KBM1; ++k) {
        drhox[c3(i, k)] = -pbxs[k - 1] * dt1[i] * dz1[c3(i, k)] * art[i] * RAMP;
        drhoy[c3(i, k)] = -pbys[k - 1] * dt1[i] * dz1[c3(i, k)] * art[i] * RAMP;
      }
    }
  }

  void baropg() {
    for (int k = 1; k <= KBM1; ++k)
      for (int i = 0; i <= M; ++i) rho1[n3(i, k)] = rho1[n3(i, k)] - rmean1[n3(i, k)];
    for (int k = 1; k <= KB; ++k)
      for (int i = 0; i <= N; ++i) rho[c3(i, k)] = rho[c3(i, k)] - rmean[c3(i, k)];
    std::fill(drhox.begin(), drhox.end(), 0.0);
    std::fill(drhoy.begin(), drhoy.end(), 0.0);
    for (int k = 1; k <= KB; ++k) { rmean[c3(0, k)] = 0.0; rho[c3(0, k)] = 0.0; }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      std::vector<double> rijk(3 * (KBM1 + 1)), drijk1(3 * (KBM1 + 1)), drijk2(KBM1 + 1);
      for (int k = 1; k <= KBM1; ++k)
        for (int j = 1; j <= 3; ++j) {
          int J1 = nxt(j), J2 = nxt2(j);
          rijk[3 * k + j - 1] = 0.5 * (rho1[n3(NV(i, J1), k)] + rho1[n3(NV(i, J2), k)]);
        }
      for (int j = 1; j <= 3; ++j) {
        drijk1[3 * 1 + j - 1] = rijk[3 * 1 + j - 1] * (-zz1[c3(i, 1)]);
        for (int k = 2; k <= KBM1; ++k) {
          double x = 0.5 * (rijk[3 * (k - 1) + j - 1] + rijk[3 * k + j - 1]) * (zz1[c3(i, k - 1)] - zz1[c3(i, k)]);
          drijk1[3 * k + j - 1] = x + drijk1[3 * (k - 1) + j - 1];
        }
      }
      drijk2[1] = 0.0;
      for (int k = 2; k <= KBM1; ++k) {
        double x = 0.5 * (zz1[c3(i, k - 1)] + zz1[c3(i, k)]) * (rho[c3(i, k)] - rho[c3(i, k - 1)]);
        drijk2[k] = drijk2[k - 1] + x;
      }
      if (iswetct[i] * iswetc[i] == 1 &&
          (h[NV(i, 1)] > P.static_ssh_adj || h[NV(i, 2)] > P.static_ssh_adj || h[NV(i, 3)] > P.static_ssh_adj)) {
        for (int k = 1; k <= KBM1; ++k) {
          for (int j = 1; j <= 3; ++j) {
            int J1 = nxt(j), J2 = nxt2(j);
            double dij = 0.5 * (dt[NV(i, J1)] + dt[NV(i, J2)]);
            double drho1 = (vy[NV(i, J1)] - vy[NV(i, J2)]) * drijk1[3 * k + j - 1] * dt1[i];
            double drho2 = (vy[NV(i, J1)] - vy[NV(i, J2)]) * dij * drijk2[k];
            drhox[c3(i, k)] = drhox[c3(i, k)] + drho1 + drho2;
            drho1 = (vx[NV(i, J2)] - vx[NV(i, J1)]) * drijk1[3 * k + j - 1] * dt1[i];
            drho2 = (vx[NV(i, J2)] - vx[NV(i, J1)]) * dij * drijk2[k];
            drhoy[c3(i, k)] = drhoy[c3(i, k)] + drho1 + drho2;
          }
        }
      }
    }
    for (int k = 1; k <= KBM1; ++k)
      for (int i = 0; i <= N; ++i) {
        drhox[c3(i, k)] = drhox[c3(i, k)] * dt1[i] * dz1[c3(i, k)] * grav_e[i] * RAMP;
        drhoy[c3(i, k)] = drhoy[c3(i, k)] * dt1[i] * dz1[c3(i, k)] * grav_e[i] * RAMP;
      }
    for (int k = 1; k <= KBM1; ++k)
      for (int i = 0; i <= M; ++i) rho1[n3(i, k)] = rho1[n3(i, k)] + rmean1[n3(i, k)];
    for (int k = 1; k <= KB; ++k)
      for (int i = 0; i <= N; ++i) rho[c3(i, k)] = rho[c3(i, k)] + rmean[c3(i, k)];
  }

  // internal_step.F:374-416: vertical sums into the 2-D forcing, ADVAVE, GX/GY, resets
  void int_pre_ext() {
    for (int i = 0; i <= N; ++i) { adx2d[i] = 0.0; ady2d[i] = 0.0; drx2d[i] = 0.0; dry2d[i] = 0.0; }
    for (int k = 1; k <= KBM1; ++k)
      for (int i = 1; i <= N; ++i) {
        adx2d[i] = adx2d[i] + advx[c3(i, k)];
        ady2d[i] = ady2d[i] + advy[c3(i, k)];
        drx2d[i] = drx2d[i] + drhox[c3(i, k)];
        dry2d[i] = dry2d[i] + drhoy[c3(i, k)];
      }
    advave(advua, advva);
    for (int i = 0; i <= N; ++i) { adx2d[i] = adx2d[i] - advua[i]; ady2d[i] = ady2d[i] - advva[i]; }
    for (int i = 0; i <= N; ++i) { uard[i] = 0.0; vard[i] = 0.0; }
    for (int i = 0; i <= M; ++i) egf[i] = 0.0;
    for (int i = 1; i <= IOBCN; ++i) uard_obcn[i] = 0.0;
  }

  // =====================================================================================
  // VERTVL_EDGE (vertvl_edge.F:37-569)
  // =====================================================================================
  void vertvl() {
    std::vector<double> xflux((size_t)M1 * KBM1, 0.0);
    auto XF = [&](int i, int k) -> double& { return xflux[(size_t)(k - 1) * M1 + i]; };
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 1; k <= KBM1; ++k)
      for (int i = 1; i <= NCV; ++i) {
        int i1 = ntrg[i], ia = NIEC(i, 1), ib = NIEC(i, 2);
        double dij = dt1[i1] * dz1[c3(i1, k)];
        double uij = u[c3(i1, k)], vij = v[c3(i1, k)];
        double exflux = dij * (-uij * dltye[i] + vij * dltxe[i]);
        XF(ia, k) = XF(ia, k) - exflux;
        XF(ib, k) = XF(ib, k) + exflux;
      }
    for (int i = 1; i <= M; ++i)
      for (int k = 1; k <= KBM1; ++k)
        if (isonb[i] == 2) XF(i, k) = 0.0;
    if (NUMQBC >= 1) {
      if (P.river_location == 0) {
        for (int j = 1; j <= NUMQBC; ++j) {
          int jj = inodeq[j];
          for (int k = 1; k <= KBM1; ++k) XF(jj, k) = XF(jj, k) - qdis[j] * VQDIST(j, k);
        }
      } else {
        for (int j = 1; j <= NUMQBC; ++j) {
          int j1 = N_ICELLQ(j, 1), j2 = N_ICELLQ(j, 2);
          for (int k = 1; k <= KBM1; ++k) {
            XF(j1, k) = XF(j1, k) - qdis[j] * RDISQ(j, 1) * VQDIST(j, k);
            XF(j2, k) = XF(j2, k) - qdis[j] * RDISQ(j, 2) * VQDIST(j, k);
          }
        }
      }
    }
    std::fill(wts.begin(), wts.end(), 0.0);
    for (int i = 0; i <= M; ++i) wts[n3(i, 1)] = -(0.0 + 0.0) * ROFVROS;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= M; ++i) {
      double wbottom = 0.0 / art1[i];
      if (iswetnt[i] * iswetn[i] == 1) {
        for (int k = 1; k <= KBM1; ++k)
          wts[n3(i, k + 1)] = wts[n3(i, k)] + XF(i, k) / art1[i] + dz[n3(i, k)] * (d[i] - dt[i]) / DTI;
      } else {
        for (int k = 1; k <= KBM1; ++k) wts[n3(i, k + 1)] = 0.0;
      }
      if (std::fabs(wts[n3(i, KB)] - wbottom) > 1.0e-8) {
        if (isonb[i] != 2) {
          double tmp1 = elf[i] * (double)(float)KBM1 - (wts[n3(i, KB)] - wbottom) * DTI / dz[n3(i, 1)];
          tmp1 = tmp1 / (double)(float)KBM1;
          dtfa[i] = tmp1 + h[i];
          for (int k = 2; k <= KB; ++k)
            wts[n3(i, k)] = wts[n3(i, k)] - (double)((float)(k - 1) / (float)KBM1) * (wts[n3(i, KB)] - wbottom);
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= KB; ++k)
      for (int i = 1; i <= N; ++i) {
        w[c3(i, k)] = ONE_THIRD * (wts[n3(NV(i, 1), k)] + wts[n3(NV(i, 2), k)] + wts[n3(NV(i, 3), k)]);
        w[c3(i, k)] = (double)(float)iswetc[i] * w[c3(i, k)];
      }
  }

  // WD_UPDATE (mod_wd.F:289-337)
  void wd_update(int c) {
    if (c == 1) {
      for (int i = 0; i <= N; ++i) iswetce[i] = iswetc[i];
    } else if (c == 2) {
      for (int i = 1; i <= M; ++i)
        if (dtfa[i] - P.min_depth <= 1.0e-5) iswetn[i] = 0;
    } else {
      for (int i = 0; i <= N; ++i) iswetct[i] = iswetc[i];
      for (int i = 0; i <= M; ++i) iswetnt[i] = iswetn[i];
    }
  }

  // =====================================================================================
  // VISCOF_H (viscofh.F:33-127)
  // =====================================================================================
  void viscof_h() {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= KBM1; ++k) {
      const double *U_ = &u[c3(0, k)], *V_ = &v[c3(0, k)];
      for (int i = 1; i <= M; ++i) {
        double pupx = 0.0, pupy = 0.0, pvpx = 0.0, pvpy = 0.0;
        int j = 1;
        int i1 = NBVE(i, j);
        pupx = pupx + U_[i1] * ECEC_Y(i, j);
        pupy = pupy + U_[i1] * ECEC_X(i, j);
        pvpx = pvpx + V_[i1] * ECEC_Y(i, j);
        pvpy = pvpy + V_[i1] * ECEC_X(i, j);
        if (isonb[i] != 0) {
          pupx = pupx + U_[i1] * NEC_Y(i, j);
          pupy = pupy + U_[i1] * NEC_X(i, j);
          pvpx = pvpx + V_[i1] * NEC_Y(i, j);
          pvpy = pvpy + V_[i1] * NEC_X(i, j);
        }
        for (j = 2; j <= ntve[i] - 1; ++j) {
          i1 = NBVE(i, j);
          pupx = pupx + U_[i1] * ECEC_Y(i, j);
          pupy = pupy + U_[i1] * ECEC_X(i, j);
          pvpx = pvpx + V_[i1] * ECEC_Y(i, j);
          pvpy = pvpy + V_[i1] * ECEC_X(i, j);
        }
        j = ntve[i];
        i1 = NBVE(i, j);
        pupx = pupx + U_[i1] * ECEC_Y(i, j);
        pupy = pupy + U_[i1] * ECEC_X(i, j);
        pvpx = pvpx + V_[i1] * ECEC_Y(i, j);
        pvpy = pvpy + V_[i1] * ECEC_X(i, j);
        if (isonb[i] != 0) {
          pupx = pupx + U_[i1] * (-NEC_Y(i, j));
          pupy = pupy + U_[i1] * (-NEC_X(i, j));
          pvpx = pvpx + V_[i1] * (-NEC_Y(i, j));
          pvpy = pvpy + V_[i1] * (-NEC_X(i, j));
        }
        pupx = pupx / art1[i];
        pupy = pupy / art1[i];
        pvpx = pvpx / art1[i];
        pvpy = pvpy / art1[i];
        double tmp1 = pupx * pupx + pvpy * pvpy;
        double tmp2 = 0.5 * ((pupy + pvpx) * (pupy + pvpx));
        viscofh[n3(i, k)] = std::sqrt(tmp1 + tmp2) * art1[i];
      }
    }
  }

  // =====================================================================================
  // ADV_UV_EDGE_GCN (adv_uv_edge_gcn.F:31-1198), layer loop hoisted (see ADVECTION).
  // =====================================================================================
  void adv_uv() {
    double fact = P.horizontal_mixing == 0 ? 1.0 : 0.0;
    double fm1 = P.horizontal_mixing == 0 ? 0.0 : 1.0;
    std::vector<double> xflux((size_t)N1 * KB, 0.0), yflux((size_t)N1 * KB, 0.0);
    std::vector<double> pstx_tm((size_t)N1 * KB, 0.0), psty_tm((size_t)N1 * KB, 0.0);
    std::fill(viscofm.begin(), viscofm.end(), 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 1; k <= KBM1; ++k) {
      const double *U_ = &u[c3(0, k)], *V_ = &v[c3(0, k)];
      double *X = &xflux[c3(0, k)], *Y = &yflux[c3(0, k)];
      double *PX = &pstx_tm[c3(0, k)], *PY = &psty_tm[c3(0, k)], *VM = &viscofm[c3(0, k)];
      std::vector<double> ualfa, valfa;
      if (P.limiter) limiter_alfa(U_, V_, [&](int c) { return iswetct[c] * iswetc[c] == 1; }, ualfa, valfa);
      const bool L = P.limiter != 0;
      for (int i = 1; i <= NE; ++i) {
        int ia = IEC(i, 1), ib = IEC(i, 2);
        int j1 = IENODE(i, 1), j2 = IENODE(i, 2);
        double elij = 0.5 * (egf[j1] + egf[j2]);
        int k1 = NBE(ia, 1), k2 = NBE(ia, 2), k3 = NBE(ia, 3);
        int k4 = NBE(ib, 1), k5 = NBE(ib, 2), k6 = NBE(ib, 3);
        double dij = 0.5 * (dt[j1] * dz[n3(j1, k)] + dt[j2] * dz[n3(j2, k)]);
        if (iswetct[ia] * iswetc[ia] == 1 || iswetct[ib] * iswetc[ib] == 1) {
          double xija = xijc[i] - xc[ia], yija = yijc[i] - yc[ia];
          double xijb = xijc[i] - xc[ib], yijb = yijc[i] - yc[ib];
          double cofa1, cofa2, cofa5, cofa6;
          cofa(U_, V_, ia, cofa1, cofa2, cofa5, cofa6);
          double cofa3, cofa4, cofa7, cofa8;
          cofa(U_, V_, ib, cofa3, cofa4, cofa7, cofa8);
          double uij1, uij2, vij1, vij2;
          face_values(U_[ia], U_[ib], cofa1, cofa2, xija, yija, cofa3, cofa4, xijb, yijb, L ? ualfa[ia] : 1.0,
                      L ? ualfa[ib] : 1.0, uij1, uij2);
          face_values(V_[ia], V_[ib], cofa5, cofa6, xija, yija, cofa7, cofa8, xijb, yijb, L ? valfa[ia] : 1.0,
                      L ? valfa[ib] : 1.0, vij1, vij2);
          double uij = 0.5 * (uij1 + uij2);
          double vij = 0.5 * (vij1 + vij2);
          double exflux = dij * (-uij * dltyc[i] + vij * dltxc[i]);
          double viscof1 = art[ia] * std::sqrt(cofa1 * cofa1 + cofa6 * cofa6 + 0.5 * ((cofa2 + cofa5) * (cofa2 + cofa5)));
          double viscof2 = art[ib] * std::sqrt(cofa3 * cofa3 + cofa8 * cofa8 + 0.5 * ((cofa4 + cofa7) * (cofa4 + cofa7)));
          double viscof = (fact * 0.5 * (viscof1 * cc_hvc[ia] + viscof2 * cc_hvc[ib]) +
                           fm1 * 0.5 * (cc_hvc[ia] + cc_hvc[ib])) / P.hprnu;
          VM[ia] = VM[ia] + viscof;
          VM[ib] = VM[ib] + viscof;
          double txx = (cofa1 + cofa3) * viscof;
          double tyy = (cofa6 + cofa8) * viscof;
          double txy = 0.5 * (cofa2 + cofa4 + cofa5 + cofa7) * viscof;
          double fxx = dij * (txx * dltyc[i] - txy * dltxc[i]);
          double fyy = dij * (txy * dltyc[i] - tyy * dltxc[i]);
          double sg = fsign1(exflux);
          double xadv = exflux * ((1.0 - sg) * uij2 + (1.0 + sg) * uij1) * 0.5;
          double yadv = exflux * ((1.0 - sg) * vij2 + (1.0 + sg) * vij1) * 0.5;
          double isb = (double)isbc[i];
          double tpa = (double)(float)(1 - isbc[i]) * epor[ia];
          double tpb = (double)(float)(1 - isbc[i]) * epor[ib];
          if (P.ghost_cells) {  // adv_uv_edge_gcy.F
            X[ia] = X[ia] + xadv * tpa + fxx * tpa;
            Y[ia] = Y[ia] + yadv * tpa + fyy * tpa;
            X[ib] = X[ib] - xadv * tpb - fxx * tpb;
            Y[ib] = Y[ib] - yadv * tpb - fyy * tpb;
          } else {
            X[ia] = X[ia] + xadv * tpa + (fxx + 3.0 * fxx * isb) * epor[ia];
            Y[ia] = Y[ia] + yadv * tpa + (fyy + 3.0 * fyy * isb) * epor[ia];
            X[ib] = X[ib] - xadv * tpb - (fxx + 3.0 * fxx * isb) * epor[ib];
            Y[ib] = Y[ib] - yadv * tpb - (fyy + 3.0 * fyy * isb) * epor[ib];
          }
        }
        PX[ia] = PX[ia] - grav_e[ia] * dt1[ia] * dz1[c3(ia, k)] * elij * dltyc[i];
        PY[ia] = PY[ia] + grav_e[ia] * dt1[ia] * dz1[c3(ia, k)] * elij * dltxc[i];
        PX[ib] = PX[ib] + grav_e[ib] * dt1[ib] * dz1[c3(ib, k)] * elij * dltyc[i];
        PY[ib] = PY[ib] - grav_e[ib] * dt1[ib] * dz1[c3(ib, k)] * elij * dltxc[i];
      }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      double w_ = (double)(iswetct[i] * iswetc[i]);
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = c3(i, k);
        xflux[q] = xflux[q] * w_;
        yflux[q] = yflux[q] * w_;
        pstx_tm[q] = pstx_tm[q] * w_;
        psty_tm[q] = psty_tm[q] * w_;
      }
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = c3(i, k);
        xflux[q] = xflux[q] + pstx_tm[q];
        yflux[q] = yflux[q] + psty_tm[q];
      }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      if (iswetct[i] * iswetc[i] != 1) continue;
      for (int k = 1; k <= KBM1; ++k) {
        double xfv, yfv;
        if (k == 1) {
          xfv = -w[c3(i, k + 1)] * (u[c3(i, k)] * dz1[c3(i, k + 1)] + u[c3(i, k + 1)] * dz1[c3(i, k)]) /
                (dz1[c3(i, k)] + dz1[c3(i, k + 1)]);
          yfv = -w[c3(i, k + 1)] * (v[c3(i, k)] * dz1[c3(i, k + 1)] + v[c3(i, k + 1)] * dz1[c3(i, k)]) /
                (dz1[c3(i, k)] + dz1[c3(i, k + 1)]);
        } else if (k == KBM1) {
          xfv = w[c3(i, k)] * (u[c3(i, k)] * dz1[c3(i, k - 1)] + u[c3(i, k - 1)] * dz1[c3(i, k)]) /
                (dz1[c3(i, k)] + dz1[c3(i, k - 1)]);
          yfv = w[c3(i, k)] * (v[c3(i, k)] * dz1[c3(i, k - 1)] + v[c3(i, k - 1)] * dz1[c3(i, k)]) /
                (dz1[c3(i, k)] + dz1[c3(i, k - 1)]);
        } else {
          xfv = w[c3(i, k)] * (u[c3(i, k)] * dz1[c3(i, k - 1)] + u[c3(i, k - 1)] * dz1[c3(i, k)]) /
                    (dz1[c3(i, k)] + dz1[c3(i, k - 1)]) -
                w[c3(i, k + 1)] * (u[c3(i, k)] * dz1[c3(i, k + 1)] + u[c3(i, k + 1)] * dz1[c3(i, k)]) /
                    (dz1[c3(i, k)] + dz1[c3(i, k + 1)]);
          yfv = w[c3(i, k)] * (v[c3(i, k)] * dz1[c3(i, k - 1)] + v[c3(i, k - 1)] * dz1[c3(i, k)]) /
                    (dz1[c3(i, k)] + dz1[c3(i, k - 1)]) -
                w[c3(i, k + 1)] * (v[c3(i, k)] * dz1[c3(i, k + 1)] + v[c3(i, k + 1)] * dz1[c3(i, k)]) /
                    (dz1[c3(i, k)] + dz1[c3(i, k + 1)]);
        }
        size_t q = c3(i, k);
        xflux[q] = xflux[q] + xfv * art[i] + drhox[q] - cor[i] * v[q] * dt1[i] * dz1[q] * art[i];
        yflux[q] = yflux[q] + yfv * art[i] + drhoy[q] + cor[i] * u[q] * dt1[i] * dz1[q] * art[i];
      }
    }
    for (int i = 1; i <= N; ++i)
      if (isbce[i] == 2)
        for (int k = 1; k <= KBM1; ++k) { xflux[c3(i, k)] = 0.0; yflux[c3(i, k)] = 0.0; }
    river_momentum3d(xflux, yflux);
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = c3(i, k);
        uf[q] = u[q] * dt1[i] / d1[i] - DTI * xflux[q] / art[i] / (d1[i] * dz1[q]);
        vf[q] = v[q] * dt1[i] / d1[i] - DTI * yflux[q] / art[i] / (d1[i] * dz1[q]);
      }
      if (iswetct[i] * iswetc[i] != 1)
        for (int k = 1; k <= KBM1; ++k) { uf[c3(i, k)] = 0.0; vf[c3(i, k)] = 0.0; }
    }
    for (int k = 1; k <= KB; ++k)
      for (int i = 0; i <= N; ++i) viscofm[c3(i, k)] = viscofm[c3(i, k)] / art[i];
  }

  // =====================================================================================
  // VDIF_UV (vdif_uv.F:34-189)
  // =====================================================================================
  void vdif_uv() {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      if (iswetc[i] != 1) {
        for (int k = 2; k <= KBM1; ++k) {
          int ki = KB - k;
          uf[c3(i, ki)] = 0.0;
          vf[c3(i, ki)] = 0.0;
        }
        wubot[i] = 0.0;
        wvbot[i] = 0.0;
        continue;
      }
      std::vector<double> a(KB + 1), c(KB + 1), vhu(KB + 1), vhpu(KB + 1), vhv(KB + 1), vhpv(KB + 1);
      for (int k = 1; k <= KB; ++k) c[k] = km1[c3(i, k)];
      double d1i = d1[i];
      for (int k = 2; k <= KBM1; ++k) {
        a[k - 1] = -DTI * (c[k] + P.umol) / (dz1[c3(i, k - 1)] * dzz1[c3(i, k - 1)] * d1i * d1i);
        c[k] = -DTI * (c[k] + P.umol) / (dz1[c3(i, k)] * dzz1[c3(i, k - 1)] * d1i * d1i);
      }
      int itmp1 = isonb[NV(i, 1)], itmp2 = isonb[NV(i, 2)], itmp3 = isonb[NV(i, 3)];
      double tmp = (itmp1 == 2 || itmp2 == 2 || itmp3 == 2) ? 0.0 : 1.0;
      vhu[1] = a[1] / (a[1] - 1.0);
      vhv[1] = a[1] / (a[1] - 1.0);
      vhpu[1] = (-DTI * wusurf[i] * tmp / (-dz1[c3(i, 1)] * d1i) - uf[c3(i, 1)]) / (a[1] - 1.0);
      vhpv[1] = (-DTI * wvsurf[i] * tmp / (-dz1[c3(i, 1)] * d1i) - vf[c3(i, 1)]) / (a[1] - 1.0);
      for (int k = 2; k <= KBM2; ++k) {
        vhpu[k] = 1.0 / (a[k] + c[k] * (1.0 - vhu[k - 1]) - 1.0);
        vhpv[k] = 1.0 / (a[k] + c[k] * (1.0 - vhv[k - 1]) - 1.0);
        vhu[k] = a[k] * vhpu[k];
        vhv[k] = a[k] * vhpv[k];
        vhpu[k] = (c[k] * vhpu[k - 1] - uf[c3(i, k)]) * vhpu[k];
        vhpv[k] = (c[k] * vhpv[k - 1] - vf[c3(i, k)]) * vhpv[k];
      }
      double ub = u[c3(i, KBM1)], vb = v[c3(i, KBM1)];
      tps[i] = cbc[i] * std::sqrt(ub * ub + vb * vb);
      uf[c3(i, KBM1)] = (c[KBM1] * vhpu[KBM2] - uf[c3(i, KBM1)]) /
                        (tps[i] * DTI / (-dz1[c3(i, KBM1)] * d1i) - 1.0 - (vhu[KBM2] - 1.0) * c[KBM1]);
      vf[c3(i, KBM1)] = (c[KBM1] * vhpv[KBM2] - vf[c3(i, KBM1)]) /
                        (tps[i] * DTI / (-dz1[c3(i, KBM1)] * d1i) - 1.0 - (vhv[KBM2] - 1.0) * c[KBM1]);
      for (int k = 2; k <= KBM1; ++k) {
        int ki = KB - k;
        uf[c3(i, ki)] = (vhu[ki] * uf[c3(i, ki + 1)] + vhpu[ki]);
        vf[c3(i, ki)] = (vhv[ki] * vf[c3(i, ki + 1)] + vhpv[ki]);
      }
      wubot[i] = -tps[i] * u[c3(i, KBM1)];
      wvbot[i] = -tps[i] * v[c3(i, KBM1)];
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i)
      for (int k = 1; k <= KBM1; ++k) {
        size_t q = c3(i, k);
        uf[q] = uf[q] / (1.0 + cc_sponge[i] * (uf[q] * uf[q]));
        vf[q] = vf[q] / (1.0 + cc_sponge[i] * (vf[q] * vf[q]));
      }
  }

  // static-SSH fix (internal_step.F:660-667) and BCOND_GCN(3,0)
  void bcond_uv3d_final() {
    for (int i = 1; i <= N; ++i)
      if (h1[i] <= P.static_ssh_adj)
        for (int k = 1; k <= KBM1; ++k) { uf[c3(i, k)] = ua[i]; vf[c3(i, k)] = va[i]; }
    bcond_uv3d(uf, vf);
  }

  // =====================================================================================
  // WREAL (wreal.F:32-140)
  // =====================================================================================
  void wreal() {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; ++i) {
      if (iswetc[i] == 1) {
        int j1 = NV(i, 1), j2 = NV(i, 2), j3 = NV(i, 3);
        double dddx = AWX(i, 1) * d[j1] + AWX(i, 2) * d[j2] + AWX(i, 3) * d[j3];
        double dddy = AWY(i, 1) * d[j1] + AWY(i, 2) * d[j2] + AWY(i, 3) * d[j3];
        double dedx = AWX(i, 1) * elf[j1] + AWX(i, 2) * elf[j2] + AWX(i, 3) * elf[j3];
        double dedy = AWY(i, 1) * elf[j1] + AWY(i, 2) * elf[j2] + AWY(i, 3) * elf[j3];
        double etf1aa = ONE_THIRD * (el[j1] + el[j2] + el[j3]);
        for (int k = 1; k <= KBM1; ++k) {
          size_t q = c3(i, k);
          double ww1 = 0.5 * (w[q] + w[c3(i, k + 1)]) + u[q] * (zz1[q] * dddx + dedx) + v[q] * (zz1[q] * dddy + dedy);
          double ww2 = (zz1[q] + 1.0) * (etf1aa - et1[i]) / DTI;
          ww[q] = ww1 + ww2;
        }
      } else {
        for (int k = 1; k <= KBM1; ++k) ww[c3(i, k)] = 0.0;
      }
    }
  }

  // Node-ring gradient of a node field over NBSN (adv_t.F:214-376 / adv_q.F:161-235)
  // =====================================================================================
  // ADV_Q(Q,QF) (adv_q.F:35-417)
  // =====================================================================================
  void adv_q(std::vector<double>& Q, std::vector<double>& QF) {
    double fact = P.horizontal_mixing == 0 ? 1.0 : 0.0;
    double fm1 = P.horizontal_mixing == 0 ? 0.0 : 1.0;
    const double QMEAN1 = F4(1.e-8);
    std::fill(QF.begin(), QF.end(), 0.0);
    std::vector<double> xflux((size_t)M1 * KB, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 2; k <= KBM1; ++k) {
      std::vector<double> pqpx(M1, 0.0), pqpy(M1, 0.0), pqpxd(M1, 0.0), pqpyd(M1, 0.0), viscoff(M1, 0.0);
      for (int i = 1; i <= M; ++i) {
        for (int j = 1; j <= ntsn[i] - 1; ++j) {
          int i1 = NBSN(i, j), i2 = NBSN(i, j + 1);
          double ffd = 0.5 * (Q[n3(i1, k)] + Q[n3(i2, k)] - QMEAN1 - QMEAN1);
          double ff1 = 0.5 * (Q[n3(i1, k)] + Q[n3(i2, k)]);
          pqpx[i] = pqpx[i] + ff1 * TRIE_Y(i, j);
          pqpy[i] = pqpy[i] + ff1 * TRIE_X(i, j);
          pqpxd[i] = pqpxd[i] + ffd * TRIE_Y(i, j);
          pqpyd[i] = pqpyd[i] + ffd * TRIE_X(i, j);
        }
        pqpx[i] = pqpx[i] / art2[i];
        pqpy[i] = pqpy[i] / art2[i];
        pqpxd[i] = pqpxd[i] / art2[i];
        pqpyd[i] = pqpyd[i] / art2[i];
      }
      for (int i = 1; i <= M; ++i)
        viscoff[i] = (viscofh[n3(i, k)] * dz[n3(i, k - 1)] + viscofh[n3(i, k - 1)] * dz[n3(i, k)]) /
                     (dz[n3(i, k)] + dz[n3(i, k - 1)]);
      double* XF = &xflux[n3(0, k)];
      for (int i = 1; i <= NCV_I; ++i) {
        int ia = NIEC(i, 1), ib = NIEC(i, 2);
        int i1 = ntrg[i];
        double uq = (u[c3(i1, k)] * dz1[c3(i1, k - 1)] + u[c3(i1, k - 1)] * dz1[c3(i1, k)]) /
                    (dz1[c3(i1, k)] + dz1[c3(i1, k - 1)]);
        double vq = (v[c3(i1, k)] * dz1[c3(i1, k - 1)] + v[c3(i1, k - 1)] * dz1[c3(i1, k)]) /
                    (dz1[c3(i1, k)] + dz1[c3(i1, k - 1)]);
        double dtij = dt1[i1] * dzz1[c3(i1, k - 1)];
        double un = vq * dltxe[i] - uq * dltye[i];
        double fij1 = Q[n3(ia, k)] + DLTXNCVE(i, 1) * pqpx[ia] + DLTYNCVE(i, 1) * pqpy[ia];
        double fij2 = Q[n3(ib, k)] + DLTXNCVE(i, 2) * pqpx[ib] + DLTYNCVE(i, 2) * pqpy[ib];
        double q1min = Q[n3(NBSN(ia, 1), k)], q1max = q1min;
        for (int j = 2; j <= ntsn[ia] - 1; ++j) {
          q1min = std::min(q1min, Q[n3(NBSN(ia, j), k)]);
          q1max = std::max(q1max, Q[n3(NBSN(ia, j), k)]);
        }
        q1min = std::min(q1min, Q[n3(ia, k)]);
        q1max = std::max(q1max, Q[n3(ia, k)]);
        double q2min = Q[n3(NBSN(ib, 1), k)], q2max = q2min;
        for (int j = 2; j <= ntsn[ib] - 1; ++j) {
          q2min = std::min(q2min, Q[n3(NBSN(ib, j), k)]);
          q2max = std::max(q2max, Q[n3(NBSN(ib, j), k)]);
        }
        q2min = std::min(q2min, Q[n3(ib, k)]);
        q2max = std::max(q2max, Q[n3(ib, k)]);
        if (fij1 < q1min) fij1 = q1min;
        if (fij1 > q1max) fij1 = q1max;
        if (fij2 < q2min) fij2 = q2min;
        if (fij2 > q2max) fij2 = q2max;
        double viscof = (fact * 0.5 * (viscoff[ia] * nn_hvc[ia] + viscoff[ib] * nn_hvc[ib]) +
                         fm1 * 0.5 * (nn_hvc[ia] + nn_hvc[ib])) / P.hprnu;
        double txx = 0.5 * (pqpxd[ia] + pqpxd[ib]) * viscof;
        double tyy = 0.5 * (pqpyd[ia] + pqpyd[ib]) * viscof;
        double fxx = -dtij * txx * dltye[i];
        double fyy = dtij * tyy * dltxe[i];
        double sg = fsign1(un);
        double exflux = -un * dtij * ((1.0 + sg) * fij2 + (1.0 - sg) * fij1) * 0.5 + fxx + fyy;
        XF[ia] = XF[ia] + exflux;
        XF[ib] = XF[ib] - exflux;
      }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= M; ++i) {
      if (iswetn[i] * iswetnt[i] == 1) {
        for (int k = 2; k <= KBM1; ++k) {
          double temp = wts[n3(i, k - 1)] * Q[n3(i, k - 1)] - wts[n3(i, k + 1)] * Q[n3(i, k + 1)];
          xflux[n3(i, k)] = xflux[n3(i, k)] + temp * art1[i] * dzz[n3(i, k - 1)] / (dz[n3(i, k - 1)] + dz[n3(i, k)]);
        }
        for (int k = 2; k <= KBM1; ++k)
          QF[n3(i, k)] = (Q[n3(i, k)] - xflux[n3(i, k)] / art1[i] * (DTI / (dt[i] * dzz[n3(i, k - 1)]))) * (dt[i] / d[i]);
      } else {
        for (int k = 2; k <= KBM1; ++k) QF[n3(i, k)] = Q[n3(i, k)];
      }
    }
  }

  // FCT_Q2 / FCT_Q2L (fct_q2.F:33-103, fct_q2l.F:33-101)
  void fct_q(const std::vector<double>& Q, std::vector<double>& QF) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= M; ++i) {
      if (is_obc_node(i) || is_river_node(i)) continue;
      for (int k = 2; k <= KBM1; ++k) {
        double qmax = Q[n3(NBSN(i, 1), k)], qmin = qmax;
        for (int j = 2; j <= ntsn[i]; ++j) {
          qmax = std::max(qmax, Q[n3(NBSN(i, j), k)]);
          qmin = std::min(qmin, Q[n3(NBSN(i, j), k)]);
        }
        if (k == 2) {
          double a = (Q[n3(i, k)] * dzz[n3(i, k)] + Q[n3(i, k + 1)] * dzz[n3(i, k - 1)]) / (dzz[n3(i, k)] + dzz[n3(i, k - 1)]);
          qmax = std::max(qmax, a);
          qmin = std::min(qmin, a);
        } else if (k == KBM1) {
          double a = (Q[n3(i, k)] * dzz[n3(i, k - 2)] + Q[n3(i, k - 1)] * dzz[n3(i, k - 1)]) / (dzz[n3(i, k - 1)] + dzz[n3(i, k - 2)]);
          qmax = std::max(qmax, a);
          qmin = std::min(qmin, a);
        } else {
          double a = (Q[n3(i, k)] * dzz[n3(i, k - 2)] + Q[n3(i, k - 1)] * dzz[n3(i, k - 1)]) / (dzz[n3(i, k - 1)] + dzz[n3(i, k - 2)]);
          double b = (Q[n3(i, k)] * dzz[n3(i, k)] + Q[n3(i, k + 1)] * dzz[n3(i, k - 1)]) / (dzz[n3(i, k)] + dzz[n3(i, k - 1)]);
          qmax = std::max(std::max(qmax, a), b);
          qmin = std::min(std::min(qmin, a), b);
        }
        if (qmin - QF[n3(i, k)] > 0.0) QF[n3(i, k)] = qmin;
        if (QF[n3(i, k)] - qmax > 0.0) QF[n3(i, k)] = qmax;
      }
    }
  }

  // =====================================================================================
  // VDIF_Q, MY2.5 (vdif_q.F:34-551)
  // =====================================================================================
  void vdif_q() {
    const double A1 = 0.92, B1 = 16.6, A2 = 0.74, B2 = 10.1, C1 = 0.08;
    const double E1 = 1.80, E2 = 1.33, SEF = 1.00, KAPPA = 0.40;
    const double SMALL = 1.e-8, GH_MAX = .0233, GH_MIN = -.281;
    const double CBCNST = 100.0, SURFL = 2.e+5, GHC = -6.0;
    const double CONST1 = std::pow(16.6, .6666667) * SEF;
    const double VHP1C = std::pow(15.8 * CBCNST, 0.6666667);
    const double COEF4 = 18.0 * A1 * A1 + 9.0 * A1 * A2;
    const double COEF5 = 9.0 * A1 * A2;
#pragma omp parallel for schedule(static)
    for (int i = 0; i <= M; ++i) {
      std::vector<double> gh(KB + 1, 0.0), sm(KB + 1, 0.0), sh(KB + 1, 0.0), prod(KB + 1, 0.0),
          dtef(KB + 1, 0.0), boygr(KB + 1, 0.0), a(KB + 1, 0.0), c(KB + 1, 0.0), vhp(KB + 1, 0.0),
          vh(KB + 1, 0.0), stf(KB + 1, 0.0);
      double l0 = 0.0;
      auto Q2 = [&](int k) -> double& { return q2[n3(i, k)]; };
      auto Q2L = [&](int k) -> double& { return q2l[n3(i, k)]; };
      auto Q2F = [&](int k) -> double& { return q2f[n3(i, k)]; };
      auto Q2LF = [&](int k) -> double& { return q2lf[n3(i, k)]; };
      auto L = [&](int k) -> double& { return l[n3(i, k)]; };
      bool real = i >= 1;
      if (real) {
        for (int k = 2; k <= KBM1; ++k)
          if (Q2F(k) <= SMALL || Q2LF(k) <= SMALL) { Q2F(k) = SMALL; Q2LF(k) = SMALL; }
        if (iswetn[i] == 1)
          for (int k = 2; k <= KBM1; ++k) {
            a[k] = -0.5 * DTI * (kq[n3(i, k + 1)] + kq[n3(i, k)] + 2.0 * P.umol) /
                   (dzz[n3(i, k - 1)] * dz[n3(i, k)] * d[i] * d[i]);
            c[k] = -0.5 * DTI * (kq[n3(i, k - 1)] + kq[n3(i, k)] + 2.0 * P.umol) /
                   (dzz[n3(i, k - 1)] * dz[n3(i, k - 1)] * d[i] * d[i]);
          }
        double wus = 0.0, wvs = 0.0;
        for (int j = 1; j <= ntve[i]; ++j) { wus = wus + wusurf[NBVE(i, j)]; wvs = wvs + wvsurf[NBVE(i, j)]; }
        wus = wus / (double)(float)ntve[i];
        wvs = wvs / (double)(float)ntve[i];
        double utau2 = std::sqrt(wus * wus + wvs * wvs);
        vhp[1] = VHP1C * utau2;
        vh[1] = 0.0;
        l0 = SURFL * utau2 / grav_n[i];
        double wub = 0.0, wvb = 0.0;
        for (int j = 1; j <= ntve[i]; ++j) { wub = wub + wubot[NBVE(i, j)]; wvb = wvb + wvbot[NBVE(i, j)]; }
        wub = wub / (double)(float)ntve[i];
        wvb = wvb / (double)(float)ntve[i];
        Q2F(KB) = std::sqrt(wub * wub + wvb * wvb) * CONST1;
      }
      for (int k = 1; k <= KB; ++k) { Q2(k) = std::fabs(Q2(k) + SMALL); Q2L(k) = std::fabs(Q2L(k)); }
      if (real) {
        if (iswetn[i] == 1)
          for (int k = 2; k <= KBM1; ++k) {
            boygr[k] = grav_n[i] * (rho1[n3(i, k - 1)] - rho1[n3(i, k)]) / (dzz[n3(i, k - 1)] * d[i]);
            prod[k] = km[n3(i, k)] * 0.0 * std::pow(.5 * (-boygr[k] + std::fabs(boygr[k])), 1.5);
          }
        if (iswetn[i] == 1)
          for (int k = 2; k <= KBM1; ++k) {
            double uk = 0.0, vk = 0.0, ukm1 = 0.0, vkm1 = 0.0;
            for (int j = 1; j <= ntve[i]; ++j) {
              int e = NBVE(i, j);
              uk = uk + u[c3(e, k)];
              vk = vk + v[c3(e, k)];
              ukm1 = ukm1 + u[c3(e, k - 1)];
              vkm1 = vkm1 + v[c3(e, k - 1)];
            }
            double fn = (double)(float)ntve[i];
            uk = uk / fn; vk = vk / fn; ukm1 = ukm1 / fn; vkm1 = vkm1 / fn;
            double den = dzz[n3(i, k - 1)] * d[i];
            prod[k] = prod[k] + km[n3(i, k)] * SEF * ((uk - ukm1) * (uk - ukm1) + (vk - vkm1) * (vk - vkm1)) / (den * den);
            prod[k] = prod[k] + kh[n3(i, k)] * boygr[k];
          }
        for (int k = 2; k <= KBM1; ++k) L(k) = Q2L(k) / Q2(k);
        for (int k = 2; k <= KBM1; ++k) {
          if (z[n3(i, k)] > -0.5) L(k) = std::max(L(k), KAPPA * l0);
          if (boygr[k] < 0.0) {
            double lmax = std::sqrt(std::fabs(GH_MIN) * Q2(k) / (-boygr[k] + SMALL));
            L(k) = std::min(L(k), lmax);
            Q2L(k) = Q2(k) * L(k);
          }
        }
        for (int k = 1; k <= KBM1; ++k) gh[k] = (L(k) * L(k) / Q2(k)) * boygr[k];
      }
      for (int k = 1; k <= KB; ++k) gh[k] = std::min(gh[k], GH_MAX);
      L(1) = KAPPA * l0;
      L(KB) = 0.0;
      gh[1] = 0.0;
      gh[KB] = 0.0;
      for (int k = 1; k <= KB; ++k) stf[k] = 1.0;
      if (real)
        for (int k = 1; k <= KB; ++k) {
          if (gh[k] < 0.0) stf[k] = 1.0 - F4(0.9) * std::pow(gh[k] / GHC, 1.5);
          if (gh[k] < GHC) stf[k] = F4(0.1);
        }
      for (int k = 1; k <= KB; ++k) dtef[k] = std::sqrt(Q2(k)) / (B1 * L(k) + SMALL) * stf[k];
      if (real) {
        for (int k = 2; k <= KBM1; ++k) {
          vhp[k] = 1. / (a[k] + c[k] * (1. - vh[k - 1]) - (2. * DTI * dtef[k] + 1.));
          vh[k] = a[k] * vhp[k];
          vhp[k] = (-2. * DTI * prod[k] + c[k] * vhp[k - 1] - Q2F(k)) * vhp[k];
        }
        if (iswetn[i] == 1)
          for (int k = 1; k <= KBM1; ++k) {
            int ki = KB - k;
            Q2F(ki) = vh[ki] * Q2F(ki + 1) + vhp[ki];
          }
        vh[1] = 0.0;
        vhp[1] = 0.0;
        if (iswetn[i] == 1)
          for (int k = 2; k <= KBM1; ++k) {
            double x = (1. / std::fabs(z[n3(i, k)] - z[n3(i, 1)]) + 1. / std::fabs(z[n3(i, k)] - z[n3(i, KB)])) *
                       L(k) / (d[i] * KAPPA);
            dtef[k] = dtef[k] * (1. + E2 * (x * x));
            vhp[k] = 1. / (a[k] + c[k] * (1. - vh[k - 1]) - (DTI * dtef[k] + 1.));
            vh[k] = a[k] * vhp[k];
            vhp[k] = (DTI * (-prod[k] * L(k) * E1) + c[k] * vhp[k - 1] - Q2LF(k)) * vhp[k];
          }
        if (iswetn[i] == 1)
          for (int k = 1; k <= KBM1; ++k) {
            int ki = KB - k;
            Q2LF(ki) = vh[ki] * Q2LF(ki + 1) + vhp[ki];
          }
        for (int k = 2; k <= KBM1; ++k)
          if (Q2F(k) <= SMALL || Q2LF(k) <= SMALL) { Q2F(k) = SMALL; Q2LF(k) = SMALL; }
        for (int k = 1; k <= KB; ++k) {
          double coef1 = A2 * (1.0 - 6.0 * A1 / B1 * stf[k]);
          double coef2 = 3.0 * A2 * B2 / stf[k] + 18.0 * A1 * A2;
          double coef3 = A1 * (1.0 - 3.0 * C1 - 6.0 * A1 / B1 * stf[k]);
          sh[k] = coef1 / (1.0 - coef2 * gh[k]);
          sm[k] = (coef3 + sh[k] * COEF4 * gh[k]) / (1. - COEF5 * gh[k]);
        }
      }
      for (int k = 1; k <= KB; ++k) {
        double kn = L(k) * std::sqrt(Q2(k));
        kq[n3(i, k)] = 0.5 * (kn * KAPPA * sm[k] + kq[n3(i, k)]);
        km[n3(i, k)] = 0.5 * (kn * sm[k] + km[n3(i, k)]);
        kh[n3(i, k)] = 0.5 * (kn * sh[k] * P.vprnu + kh[n3(i, k)]);
      }
      if (real && h[i] <= P.static_ssh_adj) {
        double kqt = 0.0, kmt = 0.0, kht = 0.0;
        for (int k = 2; k <= KBM1; ++k) { kqt = kqt + kq[n3(i, k)]; kmt = kmt + km[n3(i, k)]; kht = kht + kh[n3(i, k)]; }
        kqt = kqt / (double)(KBM1 - 1);
        kmt = kmt / (double)(KBM1 - 1);
        kht = kht / (double)(KBM1 - 1);
        for (int k = 2; k <= KBM1; ++k) { kq[n3(i, k)] = kqt; km[n3(i, k)] = kmt; kh[n3(i, k)] = kht; }
      }
    }
  }

  // =====================================================================================
  // ADV_T / ADV_S (adv_t.F:34-1077, adv_s.F:34-1028); ncon 1 = T, 2 = S
  // =====================================================================================
  void adv_ts(int ncon) {
    std::vector<double>& F1 = ncon == 1 ? t1 : s1;
    std::vector<double>& FMEAN = ncon == 1 ? tmean1 : smean1;
    std::vector<double>& FF1 = ncon == 1 ? tf1 : sf1;
    double fact = P.horizontal_mixing == 0 ? 1.0 : 0.0;
    double fm1 = P.horizontal_mixing == 0 ? 0.0 : 1.0;
    std::vector<double> xflux((size_t)M1 * KB, 0.0), xflux_adv((size_t)M1 * KB, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 1; k <= KBM1; ++k) {
      std::vector<double> ptpx(M1, 0.0), ptpy(M1, 0.0), ptpxd(M1, 0.0), ptpyd(M1, 0.0), viscoff(M1, 0.0);
      for (int i = 1; i <= M; ++i) {
        for (int j = 1; j <= ntsn[i] - 1; ++j) {
          int i1 = NBSN(i, j), i2 = NBSN(i, j + 1);
          double ffd, ff1;
          if (iswetn[i1] == 0 && iswetn[i2] == 1) {
            ffd = 0.5 * (F1[n3(i, k)] + F1[n3(i2, k)] - FMEAN[n3(i, k)] - FMEAN[n3(i2, k)]);
            ff1 = 0.5 * (F1[n3(i, k)] + F1[n3(i2, k)]);
          } else if (iswetn[i1] == 1 && iswetn[i2] == 0) {
            ffd = 0.5 * (F1[n3(i1, k)] + F1[n3(i, k)] - FMEAN[n3(i1, k)] - FMEAN[n3(i, k)]);
            ff1 = 0.5 * (F1[n3(i1, k)] + F1[n3(i, k)]);
          } else if (iswetn[i1] == 0 && iswetn[i2] == 0) {
            ffd = 0.5 * (F1[n3(i, k)] + F1[n3(i, k)] - FMEAN[n3(i, k)] - FMEAN[n3(i, k)]);
            ff1 = 0.5 * (F1[n3(i, k)] + F1[n3(i, k)]);
          } else {
            ffd = 0.5 * (F1[n3(i1, k)] + F1[n3(i2, k)] - FMEAN[n3(i1, k)] - FMEAN[n3(i2, k)]);
            ff1 = 0.5 * (F1[n3(i1, k)] + F1[n3(i2, k)]);
          }
          ptpx[i] = ptpx[i] + ff1 * TRIE_Y(i, j);
          ptpy[i] = ptpy[i] + ff1 * TRIE_X(i, j);
          ptpxd[i] = ptpxd[i] + ffd * TRIE_Y(i, j);
          ptpyd[i] = ptpyd[i] + ffd * TRIE_X(i, j);
        }
        ptpx[i] = ptpx[i] / art2[i];
        ptpy[i] = ptpy[i] / art2[i];
        ptpxd[i] = ptpxd[i] / art2[i];
        ptpyd[i] = ptpyd[i] / art2[i];
      }
      if (k == KBM1)
        for (int i = 1; i <= M; ++i) { pfpxb[i] = ptpx[i]; pfpyb[i] = ptpy[i]; }
      for (int i = 1; i <= M; ++i) viscoff[i] = viscofh[n3(i, k)];
      if (k == KBM1)
        for (int i = 1; i <= M; ++i) ah_bottom[i] = (fact * viscoff[i] + fm1) * nn_hvc[i];
      double *XF = &xflux[n3(0, k)], *XA = &xflux_adv[n3(0, k)];
      for (int i = 1; i <= NCV_I; ++i) {
        int ia = NIEC(i, 1), ib = NIEC(i, 2);
        int i1 = ntrg[i];
        double dtij = dt1[i1] * dz1[c3(i1, k)];
        double un = v[c3(i1, k)] * dltxe[i] - u[c3(i1, k)] * dltye[i];
        double fij1 = F1[n3(ia, k)] + DLTXNCVE(i, 1) * ptpx[ia] + DLTYNCVE(i, 1) * ptpy[ia];
        double fij2 = F1[n3(ib, k)] + DLTXNCVE(i, 2) * ptpx[ib] + DLTYNCVE(i, 2) * ptpy[ib];
        double t1min = F1[n3(NBSN(ia, 1), k)], t1max = t1min;
        for (int j = 2; j <= ntsn[ia] - 1; ++j) {
          t1min = std::min(t1min, F1[n3(NBSN(ia, j), k)]);
          t1max = std::max(t1max, F1[n3(NBSN(ia, j), k)]);
        }
        t1min = std::min(t1min, F1[n3(ia, k)]);
        t1max = std::max(t1max, F1[n3(ia, k)]);
        double t2min = F1[n3(NBSN(ib, 1), k)], t2max = t2min;
        for (int j = 2; j <= ntsn[ib] - 1; ++j) {
          t2min = std::min(t2min, F1[n3(NBSN(ib, j), k)]);
          t2max = std::max(t2max, F1[n3(NBSN(ib, j), k)]);
        }
        t2min = std::min(t2min, F1[n3(ib, k)]);
        t2max = std::max(t2max, F1[n3(ib, k)]);
        if (fij1 < t1min) fij1 = t1min;
        if (fij1 > t1max) fij1 = t1max;
        if (fij2 < t2min) fij2 = t2min;
        if (fij2 > t2max) fij2 = t2max;
        double viscof = fact * 0.5 * (viscoff[ia] * nn_hvc[ia] + viscoff[ib] * nn_hvc[ib]) +
                        fm1 * 0.5 * (nn_hvc[ia] + nn_hvc[ib]);
        double txx = 0.5 * (ptpxd[ia] + ptpxd[ib]) * viscof;
        double tyy = 0.5 * (ptpyd[ia] + ptpyd[ib]) * viscof;
        double fxx = -dtij * txx * dltye[i];
        double fyy = dtij * tyy * dltxe[i];
        double sg = fsign1(un);
        double exflux = -un * dtij * ((1.0 + sg) * fij2 + (1.0 - sg) * fij1) * 0.5 + fxx + fyy;
        XF[ia] = XF[ia] + exflux;
        XF[ib] = XF[ib] - exflux;
        XA[ia] = XA[ia] + (exflux - fxx - fyy);
        XA[ib] = XA[ib] - (exflux - fxx - fyy);
      }
    }
    for (int k = 1; k <= KBM1; ++k)
      for (int i = 1; i <= IOBCN; ++i) xflux_obc[(size_t)(k - 1) * (IOBCN + 1) + i] = xflux_adv[n3(i_obc_n[i], k)];
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= M; ++i) {
      if (iswetn[i] * iswetnt[i] == 1) {
        for (int k = 1; k <= KBM1; ++k) {
          double temp;
          if (k == 1) {
            temp = -wts[n3(i, k + 1)] * (F1[n3(i, k)] * dz[n3(i, k + 1)] + F1[n3(i, k + 1)] * dz[n3(i, k)]) /
                   (dz[n3(i, k)] + dz[n3(i, k + 1)]);
          } else if (k == KBM1) {
            temp = wts[n3(i, k)] * (F1[n3(i, k)] * dz[n3(i, k - 1)] + F1[n3(i, k - 1)] * dz[n3(i, k)]) /
                   (dz[n3(i, k)] + dz[n3(i, k - 1)]);
          } else {
            temp = wts[n3(i, k)] * (F1[n3(i, k)] * dz[n3(i, k - 1)] + F1[n3(i, k - 1)] * dz[n3(i, k)]) /
                       (dz[n3(i, k)] + dz[n3(i, k - 1)]) -
                   wts[n3(i, k + 1)] * (F1[n3(i, k)] * dz[n3(i, k + 1)] + F1[n3(i, k + 1)] * dz[n3(i, k)]) /
                       (dz[n3(i, k)] + dz[n3(i, k + 1)]);
          }
          if (isonb[i] == 2)
            xflux[n3(i, k)] = temp * art1[i];
          else
            xflux[n3(i, k)] = xflux[n3(i, k)] + temp * art1[i];
        }
      }
      if (iswetn[i] * iswetnt[i] == 1) {
        for (int k = 1; k <= KBM1; ++k)
          FF1[n3(i, k)] = (F1[n3(i, k)] - xflux[n3(i, k)] / art1[i] * (DTI / (dt[i] * dz[n3(i, k)]))) * (dt[i] / dtfa[i]);
      } else {
        for (int k = 1; k <= KBM1; ++k) FF1[n3(i, k)] = F1[n3(i, k)];
      }
    }
  }

  // FCT_T / FCT_S (fct_t.F:33-108, fct_s.F:33-112)
  void fct_ts(int ncon) {
    std::vector<double>& F1 = ncon == 1 ? t1 : s1;
    std::vector<double>& FF1 = ncon == 1 ? tf1 : sf1;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= M; ++i) {
      if (is_obc_node(i) || is_river_node(i)) continue;
      for (int k = 1; k <= KBM1; ++k) {
        double fmax = F1[n3(NBSN(i, 1), k)], fmin = fmax;
        for (int j = 2; j <= ntsn[i]; ++j) {
          fmax = std::max(fmax, F1[n3(NBSN(i, j), k)]);
          fmin = std::min(fmin, F1[n3(NBSN(i, j), k)]);
        }
        if (k == 1) {
          double a = (F1[n3(i, k)] * dz[n3(i, k + 1)] + F1[n3(i, k + 1)] * dz[n3(i, k)]) / (dz[n3(i, k)] + dz[n3(i, k + 1)]);
          fmax = std::max(fmax, a);
          fmin = std::min(fmin, a);
        } else if (k == KBM1) {
          double a = (F1[n3(i, k)] * dz[n3(i, k - 1)] + F1[n3(i, k - 1)] * dz[n3(i, k)]) / (dz[n3(i, k)] + dz[n3(i, k - 1)]);
          fmax = std::max(fmax, a);
          fmin = std::min(fmin, a);
        } else {
          double a = (F1[n3(i, k)] * dz[n3(i, k - 1)] + F1[n3(i, k - 1)] * dz[n3(i, k)]) / (dz[n3(i, k)] + dz[n3(i, k - 1)]);
          double b = (F1[n3(i, k)] * dz[n3(i, k + 1)] + F1[n3(i, k + 1)] * dz[n3(i, k)]) / (dz[n3(i, k)] + dz[n3(i, k + 1)]);
          fmax = std::max(std::max(fmax, a), b);
          fmin = std::min(std::min(fmin, a), b);
        }
        if (fmin - FF1[n3(i, k)] > 0.0) FF1[n3(i, k)] = fmin;
        if (FF1[n3(i, k)] - fmax > 0.0) FF1[n3(i, k)] = fmax;
      }
    }
    if (ncon == 2)
      for (size_t q = 0; q < sf1.size(); ++q)
        if (sf1[q] < 0.0) sf1[q] = 0.0;
  }

  // =====================================================================================
  // VDIF_TS(NCON1,F) (vdif_ts.F:42-385).  Heating off: WFSURF, SWRADF, SASURF and RAD are 0.
  // =====================================================================================
  void vdif_ts(int ncon) {
    std::vector<double>& F = ncon == 1 ? tf1 : sf1;
    const double UMOLPR = P.umol * 1.e0;
    const double GW = 0.0;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= M; ++i) {
      if (iswetn[i] != 1) continue;
      std::vector<double> af(KB + 1, 0.0), cf(KB + 1, 0.0), vhf(KB + 1, 0.0), vhpf(KB + 1, 0.0), ff(KB + 1, 0.0);
      std::vector<double> rad(KB + 1, 0.0);
      double wfsurf = 0.0, swradf = 0.0;
      const double sasurf = 0.0;
      if (ncon == 1 && P.heating_on) {
        // HEATING_TYPE 'flux' (vdif_ts.F:118-150), no ICE: no further cooling below -2 C
        wfsurf = wtsurf[i];
        swradf = swrad[i];
        const double WFTMP1 = -2.0;
        double wftmp2 = wfsurf;
        double wftmp3 = 0.5 * (1.0 + fsign(1.0, WFTMP1 - F[n3(i, 1)]));
        wfsurf = wftmp2 - wftmp3 * 0.5 * (wftmp2 + std::fabs(wftmp2));
        for (int k = 1; k <= KB; ++k) {
          double zdep = z[n3(i, k)] * d[i];
          rad[k] = swradf * (P.rheat * std::exp(zdep / P.zeta1) + (1 - P.rheat) * std::exp(zdep / P.zeta2));
        }
      }
      double khbottom = 0.0;
      for (int k = 2; k <= KBM1; ++k) {
        double fkh = kh[n3(i, k)];
        if (k == KBM1) khbottom = fkh;
        af[k - 1] = -DTI * (fkh + UMOLPR) / (dz[n3(i, k - 1)] * dzz[n3(i, k - 1)] * d[i] * d[i]);
        cf[k] = -DTI * (fkh + UMOLPR) / (dz[n3(i, k)] * dzz[n3(i, k - 1)] * d[i] * d[i]);
      }
      vhf[1] = af[1] / (af[1] - 1.);
      vhpf[1] = -DTI * (sasurf + wfsurf - swradf + rad[1] - rad[2]) / (-dz[n3(i, 1)] * d[i]) - F[n3(i, 1)];
      vhpf[1] = vhpf[1] / (af[1] - 1.);
      for (int k = 2; k <= KBM2; ++k) {
        vhpf[k] = 1. / (af[k] + cf[k] * (1. - vhf[k - 1]) - 1.);
        vhf[k] = af[k] * vhpf[k];
        vhpf[k] = (cf[k] * vhpf[k - 1] - F[n3(i, k)] + DTI * (rad[k] - rad[k + 1]) / (d[i] * dz[n3(i, k)])) * vhpf[k];
      }
      for (int k = 1; k <= KBM1; ++k) ff[k] = F[n3(i, k)];
      if (isonb[i] != 2) {
        double tmp1 = pfpxb[i] * std::cos(sita_gd[i]) + pfpyb[i] * std::sin(sita_gd[i]);
        double tmp2 = ah_bottom[i] * phpn[i];
        double tmp3 = khbottom + UMOLPR + ah_bottom[i] * phpn[i] * phpn[i];
        double tmp = tmp1 * tmp2 / tmp3 * (khbottom + UMOLPR);
        if (ncon == 1) {
          if (tmp1 > 0.0) tmp = 0.0;
        } else {
          if (tmp1 < 0.0) tmp = 0.0;
          tmp = -tmp;
        }
        ff[KBM1] = (cf[KBM1] * vhpf[KBM2] - ff[KBM1] - GW + DTI * (rad[KBM1] - rad[KB] - tmp) / (d[i] * dz[n3(i, KBM1)])) /
                   (cf[KBM1] * (1. - vhf[KBM2]) - 1.);
        for (int k = 2; k <= KBM1; ++k) {
          int ki = KB - k;
          ff[ki] = (vhf[ki] * ff[ki + 1] + vhpf[ki]);
        }
      }
      if (iswetn[i] * iswetnt[i] == 1)
        for (int k = 1; k <= KBM1; ++k) F[n3(i, k)] = ff[k];
    }
  }

  // =====================================================================================
  // BCOND_TS(NCON2) (bcond_ts.F:35-267, mod_obcs.F:1223-1373)
  // =====================================================================================
  void bcond_ts(int ncon) {
    if (P.river_ts_setting == 0 && NUMQBC > 0) {
      if (P.river_location == 0) {
        for (int i = 1; i <= NUMQBC; ++i) {
          int j11 = inodeq[i];
          for (int k = 1; k <= KBM1; ++k) { tf1[n3(j11, k)] = tdis[i]; sf1[n3(j11, k)] = sdis[i]; }
        }
      } else {
        for (int i = 1; i <= NUMQBC; ++i) {
          int j11 = N_ICELLQ(i, 1), j22 = N_ICELLQ(i, 2);
          for (int k = 1; k <= KBM1; ++k) {
            tf1[n3(j11, k)] = tdis[i]; sf1[n3(j11, k)] = sdis[i];
            tf1[n3(j22, k)] = tdis[i]; sf1[n3(j22, k)] = sdis[i];
          }
        }
      }
    }
    if (IOBCN <= 0) return;
    std::vector<double>& F1 = ncon == 1 ? t1 : s1;
    std::vector<double>& FF1 = ncon == 1 ? tf1 : sf1;
    std::vector<double> ttmp(KB + 1, 0.0);
    for (int i = 1; i <= IOBCN; ++i) {
      int j = i_obc_n[i], j1 = next_obc[i];
      double t2d = 0.0, t2d_next = 0.0, xflux2d = 0.0;
      for (int k = 1; k <= KBM1; ++k) {
        t2d = t2d + F1[n3(j, k)] * dz[n3(j, k)];
        t2d_next = t2d_next + FF1[n3(j1, k)] * dz[n3(j1, k)];
        xflux2d = xflux2d + xflux_obc[(size_t)(k - 1) * (IOBCN + 1) + i];
      }
      if (uard_obcn[i] > 0.0) {
        double tmp = xflux2d + t2d * uard_obcn[i];
        double t2d_obc = (t2d * dt[j] - tmp * DTI / art1[j]) / d[j];
        // BCOND_T_PERTURBATION / BCOND_S_PERTURBATION
        if (P.obc_ts_type == 1) {
          for (int k = 1; k <= KBM1; ++k) ttmp[k] = FF1[n3(j1, k)] - t2d_next;
        } else if (P.obc_ts_type == 2) {
          double cc = std::sqrt(grav_n[j] * h[j]) * DTI / dltn_obc[i];
          double cp = cc + 1.0;
          for (int k = 1; k <= KBM1; ++k) {
            double pert_next = FF1[n3(j1, k)] - t2d_next;
            double pert = F1[n3(j, k)] - t2d;
            ttmp[k] = (cc * pert_next + pert) / cp;
          }
        } else {
          double cc = std::sqrt(grav_n[j] * h[j]) * DTI / dltn_obc[i];
          double cp = cc + 1.0;
          for (int k = 1; k <= KBM1; ++k) {
            double pert_next = FF1[n3(j1, k)] - t2d_next;
            double pert = F1[n3(j, k)] - t2d;
            ttmp[k] = (cc * pert_next + pert * (1.0 - DTI / 10800.0)) / cp;
          }
        }
        for (int k = 1; k <= KBM1; ++k) FF1[n3(j, k)] = t2d_obc + ttmp[k];
        for (int k = 1; k <= KBM1; ++k) {
          double fmax = F1[n3(NBSN(j, 1), k)], fmin = fmax;
          for (int jj = 2; jj <= ntsn[j]; ++jj) {
            fmax = std::max(fmax, F1[n3(NBSN(j, jj), k)]);
            fmin = std::min(fmin, F1[n3(NBSN(j, jj), k)]);
          }
          if (k == 1) {
            double a = (F1[n3(j, k)] * dz[n3(j, k + 1)] + F1[n3(j, k + 1)] * dz[n3(j, k)]) / (dz[n3(j, k)] + dz[n3(j, k + 1)]);
            fmax = std::max(fmax, a);
            fmin = std::min(fmin, a);
          } else if (k == KBM1) {
            double a = (F1[n3(j, k)] * dz[n3(j, k - 1)] + F1[n3(j, k - 1)] * dz[n3(j, k)]) / (dz[n3(j, k)] + dz[n3(j, k - 1)]);
            fmax = std::max(fmax, a);
            fmin = std::min(fmin, a);
          } else {
            double a = (F1[n3(j, k)] * dz[n3(j, k - 1)] + F1[n3(j, k - 1)] * dz[n3(j, k)]) / (dz[n3(j, k)] + dz[n3(j, k - 1)]);
            double b = (F1[n3(j, k)] * dz[n3(j, k + 1)] + F1[n3(j, k + 1)] * dz[n3(j, k)]) / (dz[n3(j, k)] + dz[n3(j, k + 1)]);
            fmax = std::max(std::max(fmax, a), b);
            fmin = std::min(std::min(fmin, a), b);
          }
          if (fmin - FF1[n3(j, k)] > 0.0) FF1[n3(j, k)] = fmin;
          if (FF1[n3(j, k)] - fmax > 0.0) FF1[n3(j, k)] = fmax;
        }
      } else {
        for (int k = 1; k <= KBM1; ++k) FF1[n3(j, k)] = F1[n3(j, k)];
      }
    }
    for (int k = 1; k <= KBM1; ++k) { t[c3(0, k)] = 0.0; s[c3(0, k)] = 0.0; }
  }

  // T1=TF1, N2E3D(T1,T) (internal_step.F:1203-1206) / S1=SF1, N2E3D(S1,S)
  void ts_update(int ncon) {
    if (ncon == 1) { t1 = tf1; n2e3d(t1, t); }
    else { s1 = sf1; n2e3d(s1, s); }
  }

  // =====================================================================================
  // DENS2 (eqs_of_state.F:254-403)
  // =====================================================================================
  void dens2() {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= KB; ++k)
      for (int i = 0; i <= M; ++i) {
        size_t q = n3(i, k);
        double S = s1[q], T = t1[q];
        double r = S * S * S * 6.76786136E-6 - S * S * 4.8249614E-4 + S * 8.14876577E-1 - 0.22584586E0;
        r = r * (T * T * T * 1.667E-8 - T * T * 8.164E-7 + T * 1.803E-5);
        r = r + 1.0 - T * T * T * 1.0843E-6 + T * T * 9.8185E-5 - T * 4.786E-3;
        r = r * (S * S * S * 6.76786136E-6 - S * S * 4.8249614E-4 + S * 8.14876577E-1 + 3.895414E-2);
        r = r - (T - 3.98) * (T - 3.98) * (T + 283.0) / (503.57 * (T + 67.26));
        rho1[q] = r * 1.e-3;
      }
    for (int i = 0; i <= M; ++i) rho1[n3(i, KB)] = 0.0;
    for (int k = 1; k <= KB; ++k) rho1[n3(0, k)] = 0.0;
    n2e3d(rho1, rho);
  }

  // internal_step.F:1541-1590
  void int_final() {
    u = uf;
    v = vf;
    et = el;
    dt = d;
    et1 = el1;
    dt1 = d1;
    if (P.wetting_drying_on) wd_update(3);
  }

  // internal_step.F:115-265: RAMP, ADJUST2D3D(1), BCOND_GCN(5,0), BCOND_GCN(8,0)
  void int_forcing() {
    if (P.iramp != 0)
      RAMP = std::tanh((double)IINT / (double)P.iramp);
    else
      RAMP = 1.0;
    bcond8();
  }

  // =====================================================================================
  // INTERNAL_STEP (internal_step.F:29-1607)
  // =====================================================================================
  void internal_step() {
    IINT = IINT + 1;
    if (P.iramp != 0)
      RAMP = std::tanh((double)IINT / (double)P.iramp);
    else
      RAMP = 1.0;
    adjust2d3d(1);
    bcond_uv3d(u, v);
    bcond8();
    bottom_roughness();
    advection3d();
    if (!P.barotropic) {
      if (P.baropg_z) phy_baropg();
      else baropg();
    }
    int_pre_ext();
    for (int iext = 1; iext <= P.isplit; ++iext) {
      ExtTime = ExtTime + P.dte;
      external_step(iext);
    }
    adjust2d3d(2);
    vertvl();
    if (P.wetting_drying_on) wd_update(2);
    viscof_h();
    adv_uv();
    vdif_uv();
    bcond_uv3d_final();
    wreal();
    if (P.vertical_mixing == 0) {
      adv_q(q2, q2f);
      adv_q(q2l, q2lf);
      if (P.scalar_positivity_control) { fct_q(q2, q2f); fct_q(q2l, q2lf); }
      vdif_q();
      q2 = q2f;
      q2l = q2lf;
    } else {
      for (size_t q = 0; q < km.size(); ++q) { km[q] = P.umol; kh[q] = P.umol * P.vprnu; }
    }
    n2e3d(km, km1);
    if (P.temperature_active) {
      adv_ts(1);
      if (P.scalar_positivity_control) fct_ts(1);
      vdif_ts(1);
      bcond_ts(1);
      ts_update(1);
    }
    if (P.salinity_active) {
      adv_ts(2);
      if (P.scalar_positivity_control) fct_ts(2);
      vdif_ts(2);
      bcond_ts(2);
      ts_update(2);
    }
    if (!P.barotropic) dens2();
    int_final();
  }

  int run_routine(int r, int arg) {
    switch (r) {
      case FVG_R_EXTEL_EDGE: extel_edge(arg); break;
      case FVG_R_BCOND_ELF: bcond_elf(arg); break;
      case FVG_R_N2E2D_ELF: n2e2d(elf, elf1); break;
      case FVG_R_WET_JUDGE: wet_judge(); break;
      case FVG_R_FLUX_OBN: flux_obn(arg); break;
      case FVG_R_ADVAVE: advave(advua, advva); break;
      case FVG_R_EXTUV_EDGE: extuv_edge(arg); break;
      case FVG_R_BCOND_UV2D: bcond_uv2d(); break;
      case FVG_R_EXT_UPDATE: ext_update(arg); break;
      case FVG_R_EXTERNAL_STEP: ExtTime = ExtTime + P.dte; external_step(arg); break;
      case FVG_R_ADJUST2D3D: adjust2d3d(arg); break;
      case FVG_R_BCOND_UV3D_SOLID: bcond_uv3d(u, v); break;
      case FVG_R_BROUGH: bottom_roughness(); break;
      case FVG_R_ADVECTION3D: advection3d(); break;
      case FVG_R_BAROPG:
        if (P.baropg_z) phy_baropg();
        else baropg();
        break;
      case FVG_R_INT_PRE_EXT: int_pre_ext(); break;
      case FVG_R_VERTVL: vertvl(); break;
      case FVG_R_VISCOFH: viscof_h(); break;
      case FVG_R_ADV_UV: adv_uv(); break;
      case FVG_R_VDIF_UV: vdif_uv(); break;
      case FVG_R_BCOND_UV3D: bcond_uv3d_final(); break;
      case FVG_R_WREAL: wreal(); break;
      case FVG_R_ADV_Q: if (arg == 0) adv_q(q2, q2f); else adv_q(q2l, q2lf); break;
      case FVG_R_FCT_Q: if (arg == 0) fct_q(q2, q2f); else fct_q(q2l, q2lf); break;
      case FVG_R_VDIF_Q: vdif_q(); break;
      case FVG_R_TURB_UPDATE: q2 = q2f; q2l = q2lf; n2e3d(km, km1); break;
      case FVG_R_ADV_TS: adv_ts(arg); break;
      case FVG_R_FCT_TS: fct_ts(arg); break;
      case FVG_R_VDIF_TS: vdif_ts(arg); break;
      case FVG_R_BCOND_TS: bcond_ts(arg); break;
      case FVG_R_TS_UPDATE: ts_update(arg); break;
      case FVG_R_DENS2: dens2(); break;
      case FVG_R_INT_FINAL: int_final(); break;
      case FVG_R_INTERNAL_STEP: internal_step(); break;
      case FVG_R_INT_FORCING: int_forcing(); break;
      default: return FVG_ERR_ARG;
    }
    return FVG_OK;
  }

  // ---------------- construction ----------------
  template <class T>
  static void cp(std::vector<T>& dst, const T* src, size_t n) {
    dst.assign(n, T(0));
    if (src) std::memcpy(dst.data(), src, n * sizeof(T));
  }
  void reg(const char* name, std::vector<double>& v) { fields[name] = Field{v.data(), nullptr, (int64_t)v.size()}; }
  void regi(const char* name, std::vector<int32_t>& v) { fields[name] = Field{nullptr, v.data(), (int64_t)v.size()}; }

  // The boundary forcing between internal steps (the caller's UPDATE_RIVERS / UPDATE_WIND
  // of BCOND_GCN(8), bcond_gcn.F:626-676, done on the host): the same rules as
  // fvg_set_forcing.  NULL river or wind arrays leave those values unchanged.
  int set_forcing(const fvg_forcing* f) {
    if (!f || f->ntide != NTIDE) return FVG_ERR_ARG;
    const bool wind = f->wstress_x && f->wstress_y;
    if (wind && !have_wind) return FVG_ERR_UNSUPPORTED;
    const size_t o1 = IOBCN + 1, q1 = NUMQBC + 1, n1 = N1;
    if (NTIDE > 0) {
      cp(t_period, f->period, (size_t)NTIDE);
      cp(t_apt, f->apt, o1 * NTIDE);
      cp(t_phai, f->phai, o1 * NTIDE);
      if (f->emean) cp(t_emean, f->emean, o1); else t_emean.assign(o1, 0.0);
    }
    if (NUMQBC > 0) {
      if (f->qdis) cp(qdis0, f->qdis, q1);
      if (f->tdis) cp(tdis, f->tdis, q1);
      if (f->sdis) cp(sdis, f->sdis, q1);
    }
    if (wind) {
      cp(wsx, f->wstress_x, n1);
      cp(wsy, f->wstress_y, n1);
    }
    if (P.heating_on) {
      if (f->swrad) cp(swrad_w, f->swrad, (size_t)M1);
      if (f->wtsurf) cp(wtsurf_w, f->wtsurf, (size_t)M1);
    }
    return FVG_OK;
  }

  int init(const fvg_mesh* m, const fvg_params* p, const fvg_forcing* f) {
    M = m->m; N = m->n; KB = m->kb; KBM1 = KB - 1; KBM2 = KB - 2;
    NE = m->ne; NCV = m->ncv; NCV_I = m->ncv_i; M1 = M + 1; N1 = N + 1;
    NBSNC = m->nbsn_cols; NBVEC = m->nbve_cols; TRIEC = m->trie_cols;
    IOBCN = m->iobcn; NUMQBC = m->numqbc;
    P = *p;
    DTI = P.dte * (double)P.isplit;
    size_t m1 = M1, n1 = N1, kb = KB;
    cp(vx, m->vx, m1); cp(vy, m->vy, m1); cp(h, m->h, m1); cp(art1, m->art1, m1); cp(art2, m->art2, m1);
    cp(grav_n, m->grav_n, m1); cp(nn_hvc, m->nn_hvc, m1); cp(sita_gd, m->sita_gd, m1); cp(phpn, m->phpn, m1);
    cp(isonb, m->isonb, m1); cp(ntsn, m->ntsn, m1); cp(ntve, m->ntve, m1);
    cp(nbsn, m->nbsn, m1 * NBSNC); cp(nbve, m->nbve, m1 * NBVEC); cp(nbvt, m->nbvt, m1 * NBVEC);
    cp(dltxtrie, m->dltxtrie, m1 * TRIEC); cp(dltytrie, m->dltytrie, m1 * TRIEC);
    cp(dltxecec, m->dltxecec, m1 * TRIEC); cp(dltyecec, m->dltyecec, m1 * TRIEC);
    cp(dltxnec, m->dltxnec, m1 * TRIEC); cp(dltynec, m->dltynec, m1 * TRIEC);
    cp(z, m->z, m1 * kb); cp(zz, m->zz, m1 * kb); cp(dz, m->dz, m1 * kb); cp(dzz, m->dzz, m1 * kb);
    cp(xc, m->xc, n1); cp(yc, m->yc, n1); cp(art, m->art, n1); cp(h1, m->h1, n1); cp(cor, m->cor, n1);
    cp(grav_e, m->grav_e, n1); cp(cc_hvc, m->cc_hvc, n1); cp(cc_sponge, m->cc_sponge, n1);
    cp(cc_z0b, m->cc_z0b, n1); cp(epor, m->epor, n1); cp(iucp, m->iucp, n1); cp(alpha, m->alpha, n1);
    cp(nv, m->nv, n1 * 3); cp(nbe, m->nbe, n1 * 3); cp(isbce, m->isbce, n1);
    cp(a1u, m->a1u, n1 * 4); cp(a2u, m->a2u, n1 * 4); cp(awx, m->awx, n1 * 3); cp(awy, m->awy, n1 * 3);
    cp(z1, m->z1, n1 * kb); cp(zz1, m->zz1, n1 * kb); cp(dz1, m->dz1, n1 * kb); cp(dzz1, m->dzz1, n1 * kb);
    size_t e1 = NE + 1, v1 = NCV + 1, vi1 = NCV_I + 1, o1 = IOBCN + 1, q1 = NUMQBC + 1;
    cp(iec, m->iec, e1 * 2); cp(ienode, m->ienode, e1 * 2); cp(isbc, m->isbc, e1);
    cp(xijc, m->xijc, e1); cp(yijc, m->yijc, e1); cp(dltxc, m->dltxc, e1); cp(dltyc, m->dltyc, e1);
    cp(niec, m->niec, v1 * 2); cp(ntrg, m->ntrg, v1); cp(dltxe, m->dltxe, v1); cp(dltye, m->dltye, v1);
    cp(dltxncve, m->dltxncve, vi1 * 2); cp(dltyncve, m->dltyncve, vi1 * 2);
    cp(i_obc_n, m->i_obc_n, o1); cp(type_obc, m->type_obc, o1); cp(next_obc, m->next_obc, o1);
    cp(nadjc_obc, m->nadjc_obc, o1); cp(adjc_obc, m->adjc_obc, o1 * 2); cp(fluxf_obc, m->fluxf_obc, o1 * 2);
    cp(dltn_obc, m->dltn_obc, o1);
    cp(inodeq, m->inodeq, q1); cp(icellq, m->icellq, q1); cp(n_icellq, m->n_icellq, q1 * 2);
    cp(rdisq, m->rdisq, q1 * 2); cp(qarea, m->qarea, q1); cp(angleq, m->angleq, q1);
    cp(vqdist, m->vqdist, q1 * (size_t)KBM1);
    for (int i = 1; i <= IOBCN; ++i) {
      int t_ = type_obc[i];
      if (t_ == 1 || t_ == 2) obc_lst1.push_back(i);
      else if (t_ == 3 || t_ == 4) obc_lst2.push_back(i);
      else return FVG_ERR_UNSUPPORTED;
    }
    NTIDE = f ? f->ntide : 0;
    if (NTIDE > 0) {
      cp(t_period, f->period, (size_t)NTIDE);
      cp(t_apt, f->apt, o1 * NTIDE);
      cp(t_phai, f->phai, o1 * NTIDE);
      cp(t_emean, f->emean, o1);
    } else {
      t_emean.assign(o1, 0.0);
    }
    cp(qdis0, f ? f->qdis : nullptr, q1);
    cp(tdis, f ? f->tdis : nullptr, q1);
    cp(sdis, f ? f->sdis : nullptr, q1);
    have_wind = f && f->wstress_x && f->wstress_y;
    cp(wsx, have_wind ? f->wstress_x : nullptr, n1);
    cp(wsy, have_wind ? f->wstress_y : nullptr, n1);
    if (P.heating_on && !(P.rheat >= 0.0 && P.zeta1 > 0.0 && P.zeta2 > 0.0)) return FVG_ERR_ARG;
    if (P.limiter < 0 || P.limiter > 2) return FVG_ERR_ARG;
    if (P.ghost_cells < 0 || P.ghost_cells > 1) return FVG_ERR_ARG;
    cp(swrad_w, P.heating_on && f ? f->swrad : nullptr, m1);
    cp(wtsurf_w, P.heating_on && f ? f->wtsurf : nullptr, m1);
    swrad.assign(m1, 0.0);
    wtsurf.assign(m1, 0.0);
    if (P.obc_ts_type < 1 || P.obc_ts_type > 3 || P.river_ts_setting != 0) return FVG_ERR_UNSUPPORTED;

    auto Z = [](std::vector<double>& a, size_t n) { a.assign(n, 0.0); };
    for (auto* a : {&el, &elf, &elrk, &et, &d, &dt, &dtfa, &egf, &wubot_n, &wvbot_n, &taubm_n, &pfpxb, &pfpyb, &ah_bottom})
      Z(*a, m1);
    for (auto* a : {&t1, &s1, &tf1, &sf1, &rho1, &tmean1, &smean1, &rmean1, &q2, &q2l, &q2f, &q2lf, &l, &km, &kh, &kq, &wts, &viscofh})
      Z(*a, m1 * kb);
    for (auto* a : {&el1, &elf1, &elrk1, &et1, &d1, &dt1, &ua, &va, &uaf, &vaf, &uark, &vark, &uard, &vard, &adx2d, &ady2d,
                    &drx2d, &dry2d, &advua, &advva, &pstx, &psty, &wubot, &wvbot, &cbc, &tps, &fluxobn, &taubm,
                    &wusurf, &wvsurf, &wusurf2, &wvsurf2})
      Z(*a, n1);
    for (auto* a : {&u, &v, &uf, &vf, &w, &ww, &advx, &advy, &drhox, &drhoy, &rho, &t, &s, &rmean, &km1, &viscofm})
      Z(*a, n1 * kb);
    iswetn.assign(m1, 1); iswetnt.assign(m1, 1);
    iswetc.assign(n1, 1); iswetct.assign(n1, 1); iswetce.assign(n1, 1);
    xflux_obcn.assign(o1, 0.0); uard_obcn.assign(o1, 0.0); xflux_obc.assign(o1 * KBM1, 0.0);
    qdis.assign(q1, 0.0);

#define R(x) reg(#x, x)
    R(el); R(elf); R(elrk); R(et); R(d); R(dt); R(dtfa); R(egf); R(wubot_n); R(wvbot_n); R(taubm_n);
    R(pfpxb); R(pfpyb); R(ah_bottom);
    R(t1); R(s1); R(tf1); R(sf1); R(rho1); R(tmean1); R(smean1); R(rmean1); R(q2); R(q2l); R(q2f); R(q2lf);
    R(l); R(km); R(kh); R(kq); R(wts); R(viscofh);
    R(el1); R(elf1); R(elrk1); R(et1); R(d1); R(dt1); R(ua); R(va); R(uaf); R(vaf); R(uark); R(vark);
    R(uard); R(vard); R(adx2d); R(ady2d); R(drx2d); R(dry2d); R(advua); R(advva); R(pstx); R(psty);
    R(wubot); R(wvbot); R(cbc); R(tps); R(fluxobn); R(taubm); R(wusurf); R(wvsurf); R(wusurf2); R(wvsurf2);
    R(u); R(v); R(uf); R(vf); R(w); R(ww); R(advx); R(advy); R(drhox); R(drhoy); R(rho); R(t); R(s);
    R(rmean); R(km1); R(viscofm); R(xflux_obcn); R(uard_obcn); R(xflux_obc); R(qdis); R(h1);
#undef R
    regi("iswetn", iswetn); regi("iswetnt", iswetnt); regi("iswetc", iswetc);
    regi("iswetct", iswetct); regi("iswetce", iswetce);
    return FVG_OK;
  }
};

}  // namespace

extern "C" {

typedef struct orc orc;

int orc_create(const fvg_mesh* m, const fvg_params* p, const fvg_forcing* f, orc** out) {
  if (!m || !p || !out) return FVG_ERR_ARG;
  Oracle* o = new Oracle();
  int rc = o->init(m, p, f);
  if (rc != FVG_OK) { delete o; return rc; }
  *out = reinterpret_cast<orc*>(o);
  return FVG_OK;
}

void orc_destroy(orc* h) { delete reinterpret_cast<Oracle*>(h); }

int64_t orc_field_size(orc* h, const char* name) {
  Oracle* o = reinterpret_cast<Oracle*>(h);
  auto it = o->fields.find(name);
  return it == o->fields.end() ? -1 : it->second.size;
}

int orc_set_field(orc* h, const char* name, const double* src, int64_t n) {
  Oracle* o = reinterpret_cast<Oracle*>(h);
  auto it = o->fields.find(name);
  if (it == o->fields.end() || !it->second.d || it->second.size != n) return FVG_ERR_ARG;
  std::memcpy(it->second.d, src, n * sizeof(double));
  return FVG_OK;
}
int orc_get_field(orc* h, const char* name, double* dst, int64_t n) {
  Oracle* o = reinterpret_cast<Oracle*>(h);
  auto it = o->fields.find(name);
  if (it == o->fields.end() || !it->second.d || it->second.size != n) return FVG_ERR_ARG;
  std::memcpy(dst, it->second.d, n * sizeof(double));
  return FVG_OK;
}
int orc_set_ifield(orc* h, const char* name, const int32_t* src, int64_t n) {
  Oracle* o = reinterpret_cast<Oracle*>(h);
  auto it = o->fields.find(name);
  if (it == o->fields.end() || !it->second.i || it->second.size != n) return FVG_ERR_ARG;
  std::memcpy(it->second.i, src, n * sizeof(int32_t));
  return FVG_OK;
}
int orc_get_ifield(orc* h, const char* name, int32_t* dst, int64_t n) {
  Oracle* o = reinterpret_cast<Oracle*>(h);
  auto it = o->fields.find(name);
  if (it == o->fields.end() || !it->second.i || it->second.size != n) return FVG_ERR_ARG;
  std::memcpy(dst, it->second.i, n * sizeof(int32_t));
  return FVG_OK;
}
int orc_set_clock(orc* h, int32_t iint, double ext_time) {
  Oracle* o = reinterpret_cast<Oracle*>(h);
  o->IINT = iint;
  o->ExtTime = ext_time;
  return FVG_OK;
}
int orc_get_clock(orc* h, int32_t* iint, double* ext_time) {
  Oracle* o = reinterpret_cast<Oracle*>(h);
  *iint = o->IINT;
  *ext_time = o->ExtTime;
  return FVG_OK;
}
int orc_set_ramp(orc* h, double ramp) {
  reinterpret_cast<Oracle*>(h)->RAMP = ramp;
  return FVG_OK;
}
double orc_get_ramp(orc* h) { return reinterpret_cast<Oracle*>(h)->RAMP; }
int orc_internal_step(orc* h) {
  reinterpret_cast<Oracle*>(h)->internal_step();
  return FVG_OK;
}
int orc_run(orc* h, int32_t n) {
  for (int i = 0; i < n; ++i) reinterpret_cast<Oracle*>(h)->internal_step();
  return FVG_OK;
}
int orc_set_forcing(orc* h, const fvg_forcing* f) { return reinterpret_cast<Oracle*>(h)->set_forcing(f); }
int orc_run_routine(orc* h, int32_t r, int32_t arg) { return reinterpret_cast<Oracle*>(h)->run_routine(r, arg); }
int orc_set_threads(int32_t n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
  return FVG_OK;
#else
  return n == 1 ? FVG_OK : FVG_ERR_UNSUPPORTED;
#endif
}
int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
