"""Cold-start state, as FVCOM's STARTUP builds it before the first internal step.

Follows FVCOM_source/mod_startup.F:75-372 for STARTUP_TYPE='coldstart':
SET_WATER_DEPTH (:1408-1495), SET_WD_DATA (mod_wd.F:83-141) when wetting and drying is
on, STARTUP_UV_TYPE='default' (zero velocity), SET_DEFAULT_TURB (:1332-1394) and
SET_CONSTANT_TS (:1136-1181) with DENS2 (eqs_of_state.F:381-403).  The stratified
start of the large coastal mesh sets T and S linearly in sigma (T1(I,K) =
T_top + (T_bot - T_top) * (-ZZ(I,K))), which is what the workload asks for; the means
TMEAN1/SMEAN1/RMEAN1 are taken from that start as SET_CONSTANT_TS does.

The result is a dict of FVCOM variable name (lower case) -> flat Fortran-order float64
or int32 array, ready for fvg_set_field / fvg_set_ifield.
"""
from __future__ import annotations

import numpy as np

from .grid import ONE_THIRD, _f4


def dens2(s, t):
    """DENS2_2D polynomial (eqs_of_state.F:254-321), same operation order."""
    S, T = s, t
    r = S * S * S * 6.76786136E-6 - S * S * 4.8249614E-4 + S * 8.14876577E-1 - 0.22584586E0
    r = r * (T * T * T * 1.667E-8 - T * T * 8.164E-7 + T * 1.803E-5)
    r = r + 1.0 - T * T * T * 1.0843E-6 + T * T * 9.8185E-5 - T * 4.786E-3
    r = r * (S * S * S * 6.76786136E-6 - S * S * 4.8249614E-4 + S * 8.14876577E-1 + 3.895414E-2)
    r = r - (T - 3.98) * (T - 3.98) * (T + 283.0) / (503.57 * (T + 67.26))
    return r * 1.e-3


def _n2e(g, a):
    nv = g["NV"]
    out = np.zeros((g["N"] + 1,) + a.shape[1:])
    out[1:] = ONE_THIRD * (a[nv[1:, 0]] + a[nv[1:, 1]] + a[nv[1:, 2]])
    return out


def _wet_judge(g, p, elf):
    """WET_JUDGE (mod_wd.F:193-284) on the start elevation."""
    M, N = g["M"], g["N"]
    h, nv = g["H"], g["NV"]
    md = p["MIN_DEPTH"]
    iswetn = np.ones(M + 1, dtype=np.int32)
    iswetn[1:][(h[1:] + elf[1:] - md) < 1.0e-5] = 0
    iswetc = np.ones(N + 1, dtype=np.int32)
    dtmp = (np.maximum(np.maximum(elf[nv[1:, 0]], elf[nv[1:, 1]]), elf[nv[1:, 2]]) +
            np.minimum(np.minimum(h[nv[1:, 0]], h[nv[1:, 1]]), h[nv[1:, 2]]))
    iswetc[1:][(dtmp - md) < 1.0e-5] = 0
    ntve, nbve = g["NTVE"], g["NBVE"]
    for i in range(1, M + 1):
        if iswetc[nbve[i, :ntve[i]]].sum() == 0:
            iswetn[i] = 0
    elf = np.maximum(elf, -h + md)
    elf1 = _n2e(g, elf)
    return iswetn, iswetc, elf, elf1


def coldstart(case):
    g, p, init = case["grid"], case["params"], case["init"]
    M, N, KB = g["M"], g["N"], g["KB"]
    KBM1 = KB - 1
    h, h1 = g["H"], g["H1"]
    st = {}
    el = np.zeros(M + 1)
    el1 = np.zeros(N + 1)
    iswetn = np.ones(M + 1, dtype=np.int32)
    iswetc = np.ones(N + 1, dtype=np.int32)
    if p["WETTING_DRYING_ON"]:
        iswetn, iswetc, el, el1 = _wet_judge(g, p, np.zeros(M + 1))
    d = h + el
    d1 = h1 + el1
    st.update(el=el, elf=el.copy(), et=el.copy(), el1=el1, elf1=el1.copy(), et1=el1.copy(),
              d=d, dt=d.copy(), dtfa=d.copy(), d1=d1, dt1=d1.copy())
    # SET_DEFAULT_TURB (mod_startup.F:1341-1390)
    umol, vprnu = p["UMOL"], p["VPRNU"]
    q2 = np.zeros((M + 1, KB))
    q2l = np.zeros((M + 1, KB))
    L = np.zeros((M + 1, KB))
    km = np.zeros((M + 1, KB))
    kq = np.zeros((M + 1, KB))
    kh = np.zeros((M + 1, KB))
    wet = d[1:] > 0.0
    for k in range(1, KBM1):
        q2[1:, k] = np.where(wet, _f4(1.e-8), 0.0)
        q2l[1:, k] = np.where(wet, _f4(1.e-8), 0.0)
        L[1:, k] = np.where(wet, 1.0, 0.0)
        km[1:, k] = np.where(wet, 2.0 * umol, 0.0)
        kq[1:, k] = np.where(wet, 2.0 * umol, 0.0)
        kh[1:, k] = np.where(wet, 2.0 * umol / vprnu, 0.0)
    st.update(q2=q2, q2l=q2l, l=L, km=km, kq=kq, kh=kh, km1=_n2e(g, km))
    # Temperature and salinity
    t1 = np.zeros((M + 1, KB))
    s1 = np.zeros((M + 1, KB))
    if init["kind"] == "constant":
        t1[:, :KBM1] = init["t"]
        s1[:, :KBM1] = init["s"]
    else:
        zz = g["ZZ"]
        tt, tb = init["t"]
        ss, sb = init["s"]
        t1[1:, :KBM1] = tt + (tb - tt) * (-zz[1:, :KBM1])
        s1[1:, :KBM1] = ss + (sb - ss) * (-zz[1:, :KBM1])
    if init.get("t_offset") is not None:
        # ensemble perturbation of the initial temperature, per node (0:M)
        t1[1:, :KBM1] += np.asarray(init["t_offset"], dtype=np.float64)[1:, None]
    rho1 = dens2(s1, t1)
    rho1[:, KB - 1] = 0.0
    rho1[0, :] = 0.0
    rho = _n2e(g, rho1)
    st.update(t1=t1, s1=s1, tf1=t1.copy(), sf1=s1.copy(), rho1=rho1, rho=rho,
              tmean1=t1.copy(), smean1=s1.copy(), rmean1=rho1.copy(), rmean=rho.copy(),
              t=_n2e(g, t1), s=_n2e(g, s1))
    st.update(iswetn=iswetn, iswetnt=np.ones(M + 1, dtype=np.int32), iswetc=iswetc,
              iswetct=np.ones(N + 1, dtype=np.int32), iswetce=np.ones(N + 1, dtype=np.int32))
    out = {}
    for k, v in st.items():
        v = np.asarray(v)
        out[k] = np.ascontiguousarray(v.reshape(-1, order="F")) if v.ndim > 1 else v
    return out
