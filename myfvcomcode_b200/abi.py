"""ctypes mirror of the structs in include/fvg.h and their construction from a Grid.

The same structs feed the CUDA library (libfvg.so) and the CPU oracle, so a model is
marshalled once and handed to either.  Arrays are converted to contiguous Fortran-order
copies with the dtype the header names; the bundle keeps them alive for the lifetime of
the structs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .cases import simple_drag

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)


class FvgMesh(C.Structure):
    _fields_ = [
        ("m", C.c_int32), ("n", C.c_int32), ("kb", C.c_int32),
        ("ne", C.c_int32), ("ncv", C.c_int32), ("ncv_i", C.c_int32),
        ("nbsn_cols", C.c_int32), ("nbve_cols", C.c_int32), ("trie_cols", C.c_int32),
        ("vx", _d), ("vy", _d), ("h", _d), ("art1", _d), ("art2", _d), ("grav_n", _d),
        ("nn_hvc", _d), ("sita_gd", _d), ("phpn", _d),
        ("isonb", _i), ("ntsn", _i), ("ntve", _i),
        ("nbsn", _i), ("nbve", _i), ("nbvt", _i),
        ("dltxtrie", _d), ("dltytrie", _d), ("dltxecec", _d), ("dltyecec", _d),
        ("dltxnec", _d), ("dltynec", _d),
        ("z", _d), ("zz", _d), ("dz", _d), ("dzz", _d),
        ("xc", _d), ("yc", _d), ("art", _d), ("h1", _d), ("cor", _d), ("grav_e", _d),
        ("cc_hvc", _d), ("cc_sponge", _d), ("cc_z0b", _d),
        ("epor", _d), ("iucp", _d), ("alpha", _d),
        ("nv", _i), ("nbe", _i), ("isbce", _i),
        ("a1u", _d), ("a2u", _d), ("awx", _d), ("awy", _d),
        ("z1", _d), ("zz1", _d), ("dz1", _d), ("dzz1", _d),
        ("iec", _i), ("ienode", _i), ("isbc", _i),
        ("xijc", _d), ("yijc", _d), ("dltxc", _d), ("dltyc", _d),
        ("niec", _i), ("ntrg", _i), ("dltxe", _d), ("dltye", _d),
        ("dltxncve", _d), ("dltyncve", _d),
        ("iobcn", C.c_int32),
        ("i_obc_n", _i), ("type_obc", _i), ("next_obc", _i), ("nadjc_obc", _i),
        ("adjc_obc", _i), ("fluxf_obc", _d), ("dltn_obc", _d),
        ("numqbc", C.c_int32),
        ("inodeq", _i), ("icellq", _i), ("n_icellq", _i), ("rdisq", _d),
        ("qarea", _d), ("angleq", _d), ("vqdist", _d),
    ]


class FvgParams(C.Structure):
    _fields_ = [
        ("dte", C.c_double), ("isplit", C.c_int32), ("iramp", C.c_int32),
        ("min_depth", C.c_double), ("static_ssh_adj", C.c_double),
        ("horizontal_mixing", C.c_int32), ("hprnu", C.c_double), ("umol", C.c_double),
        ("vprnu", C.c_double), ("cbcmin", C.c_double), ("vertical_mixing", C.c_int32),
        ("wetting_drying_on", C.c_int32), ("scalar_positivity_control", C.c_int32),
        ("barotropic", C.c_int32), ("temperature_active", C.c_int32),
        ("salinity_active", C.c_int32), ("obc_elevation_forcing_on", C.c_int32),
        ("obc_ts_type", C.c_int32), ("river_ts_setting", C.c_int32),
        ("river_location", C.c_int32), ("tide_ref_time", C.c_double),
        ("heating_on", C.c_int32), ("rheat", C.c_double), ("zeta1", C.c_double), ("zeta2", C.c_double),
        ("limiter", C.c_int32), ("baropg_z", C.c_int32), ("ghost_cells", C.c_int32),
    ]


class FvgForcing(C.Structure):
    _fields_ = [
        ("ntide", C.c_int32), ("period", _d), ("apt", _d), ("phai", _d), ("emean", _d),
        ("qdis", _d), ("tdis", _d), ("sdis", _d),
        ("wstress_x", _d), ("wstress_y", _d),
        ("swrad", _d), ("wtsurf", _d),
    ]


class Bundle:
    """Owns the Fortran-ordered copies the structs point to."""

    def __init__(self):
        self.keep = []

    def d(self, a):
        a = np.asfortranarray(np.asarray(a, dtype=np.float64))
        self.keep.append(a)
        return a.ctypes.data_as(_d)

    def i(self, a):
        a = np.asfortranarray(np.asarray(a, dtype=np.int32))
        self.keep.append(a)
        return a.ctypes.data_as(_i)


def _pad_rows(a, rows):
    """Row-0-ghosted array with at least ``rows`` rows (for empty OBC/river lists)."""
    a = np.asarray(a)
    if a.shape[0] >= rows:
        return a
    shape = (rows,) + a.shape[1:]
    out = np.zeros(shape, dtype=a.dtype)
    out[: a.shape[0]] = a
    return out


def wind_stress(case):
    """Surface stress (N/m^2, (0:N)) before FVCOM's RAMP*0.001 scaling, or None."""
    wind = case["forcing"].get("wind")
    if wind is None:
        return None
    N = case["grid"]["N"]
    if wind["kind"] == "field":
        sx = np.array(wind["sx"], dtype=np.float64)
        sy = np.array(wind["sy"], dtype=np.float64)
    elif wind["kind"] == "speed":
        sx, sy = simple_drag(np.full(N + 1, wind["u"]), np.full(N + 1, wind["v"]))
    else:
        sx, sy = np.full(N + 1, float(wind["u"])), np.full(N + 1, float(wind["v"]))
    sx[0] = 0.0
    sy[0] = 0.0
    return sx, sy


def heat_flux(case):
    """(short-wave, net heat flux) in W/m^2 per node (0:M) before RAMP, or None.
    ``case["forcing"]["heat"]`` holds ``swrad`` and ``wtsurf`` as scalars or (0:M) arrays."""
    heat = case["forcing"].get("heat")
    if heat is None:
        return None
    M = case["grid"]["M"]
    out = []
    for key in ("swrad", "wtsurf"):
        a = np.broadcast_to(np.asarray(heat[key], dtype=np.float64), (M + 1,)).copy()
        a[0] = 0.0
        out.append(a)
    return tuple(out)


def make_structs(case):
    """Build (mesh, params, forcing, bundle) ctypes structs for a case dict."""
    g = case["grid"]
    p = case["params"]
    fc = case["forcing"]
    b = Bundle()
    ms = FvgMesh()
    ms.m, ms.n, ms.kb = g["M"], g["N"], g["KB"]
    ms.ne, ms.ncv, ms.ncv_i = g["NE"], g["NCV"], g["NCV_I"]
    ms.nbsn_cols = g["NBSN"].shape[1]
    ms.nbve_cols = g["NBVE"].shape[1]
    ms.trie_cols = g["DLTXTRIE"].shape[1]
    for name in ("vx", "vy", "h", "art1", "art2", "grav_n", "nn_hvc", "sita_gd", "phpn",
                 "dltxtrie", "dltytrie", "dltxecec", "dltyecec", "dltxnec", "dltynec",
                 "z", "zz", "dz", "dzz", "xc", "yc", "art", "h1", "cor", "grav_e", "cc_hvc",
                 "cc_sponge", "cc_z0b", "epor", "iucp", "alpha", "a1u", "a2u", "awx", "awy",
                 "z1", "zz1", "dz1", "dzz1", "xijc", "yijc", "dltxc", "dltyc", "dltxe", "dltye",
                 "dltxncve", "dltyncve"):
        setattr(ms, name, b.d(g[name.upper()]))
    for name in ("isonb", "ntsn", "ntve", "nbsn", "nbve", "nbvt", "nv", "nbe", "isbce",
                 "iec", "ienode", "isbc", "niec", "ntrg"):
        setattr(ms, name, b.i(g[name.upper()]))
    nob = g["IOBCN"]
    ms.iobcn = nob
    for name in ("i_obc_n", "next_obc", "nadjc_obc", "type_obc"):
        setattr(ms, name, b.i(_pad_rows(g[name.upper()], nob + 1)))
    ms.adjc_obc = b.i(_pad_rows(g["ADJC_OBC"], nob + 1))
    ms.fluxf_obc = b.d(_pad_rows(g["FLUXF_OBC"], nob + 1))
    ms.dltn_obc = b.d(_pad_rows(g["DLTN_OBC"], nob + 1))
    nq = g["NUMQBC"]
    ms.numqbc = nq
    ms.inodeq = b.i(g["INODEQ"])
    ms.icellq = b.i(g["ICELLQ"])
    ms.n_icellq = b.i(g["N_ICELLQ"])
    ms.rdisq = b.d(g["RDISQ"])
    ms.qarea = b.d(g["QAREA"])
    ms.angleq = b.d(g["ANGLEQ"])
    ms.vqdist = b.d(g["VQDIST"])

    ps = FvgParams()
    ps.dte = p["DTE"]
    ps.isplit = p["ISPLIT"]
    ps.iramp = p["IRAMP"]
    ps.min_depth = p["MIN_DEPTH"]
    ps.static_ssh_adj = p["STATIC_SSH_ADJ"]
    ps.horizontal_mixing = {"closure": 0, "constant": 1}[p["HORIZONTAL_MIXING_TYPE"]]
    ps.hprnu = p["HPRNU"]
    ps.umol = p["UMOL"]
    ps.vprnu = p["VPRNU"]
    ps.cbcmin = p["CBCMIN"]
    ps.vertical_mixing = {"closure": 0, "constant": 1}[p["VERTICAL_MIXING_TYPE"]]
    ps.wetting_drying_on = int(bool(p["WETTING_DRYING_ON"]))
    ps.scalar_positivity_control = int(bool(p["SCALAR_POSITIVITY_CONTROL"]))
    ps.barotropic = int(bool(p["BAROTROPIC"]))
    ps.temperature_active = int(bool(p["TEMPERATURE_ACTIVE"]))
    ps.salinity_active = int(bool(p["SALINITY_ACTIVE"]))
    ps.obc_elevation_forcing_on = int(nob > 0 and fc.get("tide") is not None)
    ps.obc_ts_type = p["OBC_TS_TYPE"]
    ps.river_ts_setting = {"specified": 0, "calculated": 1}[p["RIVER_TS_SETTING"]]
    ps.river_location = {"node": 0, "edge": 1}[g["RIVER_LOC"]]
    ps.tide_ref_time = p.get("TIDE_REF_TIME", 0.0)
    ps.heating_on = int(bool(p.get("HEATING_ON", False)))
    ps.rheat = p.get("HEATING_LONGWAVE_PERCTAGE", 0.78)
    ps.zeta1 = p.get("HEATING_LONGWAVE_LENGTHSCALE", 1.4)
    ps.zeta2 = p.get("HEATING_SHORTWAVE_LENGTHSCALE", 6.3)
    ps.limiter = {"LIMITED_NO": 0, "LIMITED_1": 1, "LIMITED_2": 2}.get(p.get("LIMITER", "LIMITED_NO"), -1)
    ps.baropg_z = {"sigma levels": 0, "z coordinates": 1}.get(
        p.get("BAROCLINIC_PRESSURE_GRADIENT", "sigma levels"), -1)
    ps.ghost_cells = 0 if g.a.get("GHOST_CELLS", "GCN") == "GCN" else 1

    fs = forcing_struct(case, b)
    return ms, ps, fs, b


def forcing_struct(case, b=None):
    """An fvg_forcing struct for ``case["forcing"]``: the tide, river discharge with its
    temperature and salinity, and the wind stress (``wind_stress``).  ``b`` (a Bundle)
    keeps the arrays the struct points to alive; pass ``None`` to get a new one back as
    the struct's ``_keep`` attribute."""
    g = case["grid"]
    fc = case["forcing"]
    nob, nq = g["IOBCN"], g["NUMQBC"]
    own = b is None
    if own:
        b = Bundle()
    fs = FvgForcing()
    tide = fc.get("tide")
    if tide is not None and nob > 0:
        nt = len(tide["period"])
        fs.ntide = nt
        fs.period = b.d(tide["period"])
        apt = np.zeros((nob + 1, nt)); apt[1:] = tide["apt"]
        phai = np.zeros((nob + 1, nt)); phai[1:] = tide["phai"]
        em = np.zeros(nob + 1); em[1:] = tide["emean"]
        fs.apt, fs.phai, fs.emean = b.d(apt), b.d(phai), b.d(em)
    else:
        fs.ntide = 0
    q = np.zeros(nq + 1); q[1:] = fc["qdis"]
    td = np.zeros(nq + 1); td[1:] = fc["tdis"]
    sd = np.zeros(nq + 1); sd[1:] = fc["sdis"]
    fs.qdis, fs.tdis, fs.sdis = b.d(q), b.d(td), b.d(sd)
    ws = wind_stress(case)
    if ws is not None:
        fs.wstress_x, fs.wstress_y = b.d(ws[0]), b.d(ws[1])
    hf = heat_flux(case)
    if hf is not None:
        fs.swrad, fs.wtsurf = b.d(hf[0]), b.d(hf[1])
    if own:
        fs._keep = b
    return fs
