"""NetCDF-3 classic output and restart with FVCOM's variable names.

History files carry the mesh (x, y, xc, yc, nv, h, siglay, siglev) once and, per record,
time and the prognostic fields under the names and units FVCOM's history writer uses
(mod_ncdio.F: zeta :3019, u/v :3406/:3461, ua/va :3637/:3656, ww :3735, temp :3792,
salinity :3842, km/kh/kq :4113-4161, q2/q2l :4219/:4240), so the files read like FVCOM
output.  Dimensions: node, nele, siglay, siglev, three, time (unlimited).

Restart files hold every state array of the step (STATE_FIELDS) in the library's field
layout, plus IINT, ExtTime and RAMP; ``read_restart`` into a model of the same case
continues the run bit for bit.  scipy.io's NetCDF-3 writer is used (no NetCDF library is
installed).
"""
from __future__ import annotations

import numpy as np
from scipy.io import netcdf_file

# Every array the step carries from one internal step to the next.
NODE2 = ["el", "elf", "elrk", "et", "d", "dt", "dtfa", "egf", "wubot_n", "wvbot_n", "taubm_n"]
NODE3 = ["t1", "s1", "tf1", "sf1", "rho1", "tmean1", "smean1", "rmean1", "q2", "q2l", "q2f",
         "q2lf", "l", "km", "kh", "kq", "wts", "viscofh"]
CELL2 = ["el1", "elf1", "elrk1", "et1", "d1", "dt1", "ua", "va", "uaf", "vaf", "uark", "vark",
         "uard", "vard", "adx2d", "ady2d", "drx2d", "dry2d", "advua", "advva", "pstx", "psty",
         "wubot", "wvbot", "cbc", "tps", "fluxobn", "taubm", "wusurf", "wvsurf"]
CELL3 = ["u", "v", "uf", "vf", "w", "ww", "advx", "advy", "drhox", "drhoy", "rho", "t", "s",
         "rmean", "km1", "viscofm"]
INTS = ["iswetn", "iswetnt", "iswetc", "iswetct", "iswetce"]
OTHER = ["xflux_obcn", "uard_obcn", "qdis", "pfpxb_t", "pfpxb_s", "pfpyb_t", "pfpyb_s",
         "ah_bottom_t", "ah_bottom_s", "xflux_obc_t", "xflux_obc_s"]
STATE_FIELDS = NODE2 + NODE3 + CELL2 + CELL3 + INTS + OTHER

# name in the file -> (library field, location, long_name, units)
HISTORY = [
    ("zeta", "el", "node", "Water Surface Elevation", "meters"),
    ("ua", "ua", "nele", "Vertically Averaged x-velocity", "meters s-1"),
    ("va", "va", "nele", "Vertically Averaged y-velocity", "meters s-1"),
    ("u", "u", "siglay_nele", "East Velocity Component", "m s-1"),
    ("v", "v", "siglay_nele", "North Velocity Component", "m s-1"),
    ("ww", "ww", "siglay_nele", "Upward Water Velocity", "meters s-1"),
    ("temp", "t1", "siglay_node", "temperature", "degC"),
    ("salinity", "s1", "siglay_node", "salinity", "1e-3"),
    ("km", "km", "siglev_node", "Turbulent Eddy Viscosity For Momentum", "m 2 s-1"),
    ("kh", "kh", "siglev_node", "Turbulent Eddy Viscosity For Scalars", "m 2 s-1"),
    ("kq", "kq", "siglev_node", "Turbulent Eddy Viscosity For Q2/Q2L", "m 2 s-1"),
    ("q2", "q2", "siglev_node", "Turbulent Kinetic Energy", "m2 s-2"),
    ("q2l", "q2l", "siglev_node", "Turbulent Kinetic Energy X Turbulent Macroscale", "m3 s-2"),
]


class History:
    """An FVCOM-style history file; ``write(model)`` appends one record."""

    def __init__(self, path, case, title="fvg"):
        g = case["grid"]
        M, N, KB = g["M"], g["N"], g["KB"]
        self.M, self.N, self.KB = M, N, KB
        self.nc = netcdf_file(path, "w", version=1)
        nc = self.nc
        nc.title = title
        nc.source = "FVCOM mode-split step on the GPU (myfvcomcode_b200)"
        nc.Conventions = "CF-1.0"
        for name, n in (("time", None), ("node", M), ("nele", N), ("siglay", KB - 1), ("siglev", KB),
                        ("three", 3)):
            nc.createDimension(name, n)

        def var(name, typ, dims, data=None, **att):
            v = nc.createVariable(name, typ, dims)
            for k, a in att.items():
                setattr(v, k, a)
            if data is not None:
                v[:] = data
            return v

        var("x", "f", ("node",), g["VX"][1:] + g.a.get("VXMIN", 0.0), long_name="nodal x-coordinate", units="meters")
        var("y", "f", ("node",), g["VY"][1:] + g.a.get("VYMIN", 0.0), long_name="nodal y-coordinate", units="meters")
        var("xc", "f", ("nele",), g["XC"][1:] + g.a.get("VXMIN", 0.0), long_name="zonal x-coordinate", units="meters")
        var("yc", "f", ("nele",), g["YC"][1:] + g.a.get("VYMIN", 0.0), long_name="zonal y-coordinate", units="meters")
        var("nv", "i", ("three", "nele"), np.asarray(g["NV"][1:]).T.astype(np.int32),
            long_name="nodes surrounding element")
        var("h", "f", ("node",), g["H"][1:], long_name="Bathymetry", units="m", positive="down")
        var("siglay", "f", ("siglay", "node"), np.asarray(g["ZZ"][1:, :KB - 1]).T, long_name="Sigma Layers",
            positive="up", valid_min=-1.0, valid_max=0.0)
        var("siglev", "f", ("siglev", "node"), np.asarray(g["Z"][1:, :KB]).T, long_name="Sigma Levels",
            positive="up", valid_min=-1.0, valid_max=0.0)
        self.t = var("time", "f", ("time",), long_name="time", units="days since model start")
        self.it = var("Itime", "i", ("time",), units="days since model start")
        self.it2 = var("Itime2", "i", ("time",), units="msec since 00:00:00")
        self.iint = var("iint", "i", ("time",), long_name="internal mode iteration number")
        self.vars = {}
        for fname, field, loc, ln, un in HISTORY:
            dims = {"node": ("time", "node"), "nele": ("time", "nele"), "siglay_nele": ("time", "siglay", "nele"),
                    "siglay_node": ("time", "siglay", "node"), "siglev_node": ("time", "siglev", "node")}[loc]
            self.vars[fname] = (field, loc, var(fname, "f", dims, long_name=ln, units=un))
        self.n = 0

    def write(self, model):
        iint, ext_time = model.clock()
        rec = self.n
        days = ext_time / 86400.0
        self.t[rec] = days
        self.it[rec] = int(np.floor(days))
        self.it2[rec] = int(round((days - np.floor(days)) * 86400000.0))
        self.iint[rec] = iint
        for fname, (field, loc, v) in self.vars.items():
            a = model.get(field)
            if loc in ("node", "nele"):
                v[rec] = a[1:]
            else:
                rows = a.size // self.KB
                a2 = a.reshape((rows, self.KB), order="F")
                nl = self.KB - 1 if loc.startswith("siglay") else self.KB
                v[rec] = a2[1:, :nl].T
        self.n += 1

    def close(self):
        self.nc.close()


def write_restart(path, model):
    """Every state array of the step plus the clock and RAMP, in the library's layout."""
    nc = netcdf_file(path, "w", version=2)
    iint, ext_time = model.clock()
    nc.iint = np.int32(iint)
    nc.ext_time = np.float64(ext_time)
    nc.ramp = np.float64(model.ramp() if hasattr(model, "ramp") else np.nan)
    for name in STATE_FIELDS:
        try:
            a = model.get(name)
        except KeyError:
            continue
        dim = "n_" + name
        nc.createDimension(dim, a.size)
        v = nc.createVariable(name, "i" if a.dtype.kind == "i" else "d", (dim,))
        v[:] = a
    nc.close()


def read_restart(path, model):
    """Load a restart written by ``write_restart`` into a model of the same case."""
    nc = netcdf_file(path, "r", mmap=False)
    for name in STATE_FIELDS:
        if name in nc.variables:
            model.set(name, np.array(nc.variables[name][:]))
    model.set_clock(int(nc.iint), float(nc.ext_time))
    r = float(nc.ramp)
    if np.isfinite(r) and hasattr(model, "set_ramp"):
        model.set_ramp(r)
    nc.close()
