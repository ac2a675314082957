"""FVCOM run directories: the run namelist, the cold-start grid files and the NetCDF
forcing files, read into a case and stepped with forcing that varies in time.

Readers (each follows the FVCOM routine that reads the same file):

* ``parse_namelist`` / ``read_namelist``: Fortran namelist groups (``&NML_CASE`` ...
  ``/``), repeated groups (``&NML_RIVER``) kept in order (mod_input.F:470-840).
* ``read_grid``: ``*_grd.dat``, connectivity then coordinates, node order swapped to
  FVCOM's clockwise order (READ_COLDSTART_GRID, mod_input.F:3654-3764;
  READ_COLDSTART_COORDS :3958-4019).
* ``read_depth`` (:4022-4131), ``read_obc`` (:3767-3866), ``read_coriolis``
  (:4133-4234), ``read_sponge`` (:4238-4335), ``read_sigma`` (:4338-4577, UNIFORM and
  GEOMETRIC levels).
* ``read_river_namelist`` + ``RiverSeries``: NML_RIVER groups and the river NetCDF file
  (river_names, river_flux, river_temp, river_salt); the value at a time is the nearer
  of the two bracketing records, as UPDATE_RIVERS takes it (mod_force.F:11229-11420).
* ``WindSeries``: constant wind, or uwind_stress/vwind_stress (uwind_speed/vwind_speed
  through ASIMPLE_DRAG) per cell, interpolated linearly between the bracketing records
  (UPDATE_WIND, mod_force.F:13415-13550).
* ``read_spectral_tide``: the spectral elevation file (tide_period, tide_Eamp,
  tide_Ephase, tide_Eref, time_origin) mapped onto the open-boundary node list.

Forcing times: a file's record time is Itime (days) + Itime2 (ms) when both exist,
else ``time`` in days (UPDATE_FILE_BRACKET / GET_FILE_TIME, mod_nctools.F).  The
bracketing rule is ``prev < now <= next`` with the weight of ``next`` equal to
``(now - prev) / (next - prev)`` in FP64; a time outside the records is an error, as in
FVCOM.  The forcing of internal step IINT is evaluated at IntTime = start + IINT * DTI,
the time fvcom.F:850 sets before calling INTERNAL_STEP, and handed to the model with
``fvg_set_forcing`` (the RAMP and the 0.001 scaling stay on the device, BCOND_GCN(8)).

``FvcomRun`` ties these together: ``FvcomRun(nml_path).run(engine)`` steps a model to
END_DATE, updating the forcing every internal step and writing an FVCOM-named history
file every NC_OUT_INTERVAL (``ncio.History``).  ``write_run`` writes a case in the same
file formats, so that a case generated here can be run from files like any FVCOM case.

* ``HeatSeries``: surface heating of HEATING_TYPE 'flux', constant or from short_wave and
  net_heat_flux per node, interpolated linearly (UPDATE_HEAT, mod_force.F:12427-12539).

What the supported path does not cover raises ``ValueError`` naming the option:
body heating, calculated heat flux, precipitation, groundwater, air pressure, TANH and
GENERALIZED sigma levels,
periodic river or wind kinds, non-spectral open-boundary elevation, restarts other
than ``coldstart`` with constant or linear-in-sigma temperature and salinity.
"""
from __future__ import annotations

import datetime as _dt
import os
import re

import numpy as np
from scipy.io import netcdf_file

from .cases import default_params, simple_drag
from .grid import build_grid

MJD_EPOCH = _dt.datetime(1858, 11, 17)


# --------------------------------------------------------------------------------------
# Fortran namelists
# --------------------------------------------------------------------------------------
def _strip_comments(text):
    out = []
    for line in text.splitlines():
        q = None
        cut = len(line)
        for i, ch in enumerate(line):
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "!":
                cut = i
                break
        out.append(line[:cut])
    return "\n".join(out)


def _tokens(body):
    """Quoted strings, '=', ',' and bare words of a namelist group body."""
    i, n = 0, len(body)
    toks = []
    while i < n:
        ch = body[i]
        if ch.isspace():
            i += 1
        elif ch in "'\"":
            j = i + 1
            buf = []
            while j < n:
                if body[j] == ch:
                    if j + 1 < n and body[j + 1] == ch:
                        buf.append(ch)
                        j += 2
                        continue
                    break
                buf.append(body[j])
                j += 1
            toks.append(("s", "".join(buf)))
            i = j + 1
        elif ch in "=,":
            toks.append((ch, ch))
            i += 1
        else:
            j = i
            while j < n and not body[j].isspace() and body[j] not in "=,'\"":
                j += 1
            toks.append(("w", body[i:j]))
            i = j
    return toks


_LOGICAL = {"T": True, ".T.": True, ".TRUE.": True, "TRUE": True,
            "F": False, ".F.": False, ".FALSE.": False, "FALSE": False}


def _value(tok):
    kind, text = tok
    if kind == "s":
        return [text]
    m = re.fullmatch(r"(\d+)\*(.*)", text)
    if m:
        return _value(("w", m.group(2))) * int(m.group(1))
    up = text.upper()
    if up in _LOGICAL:
        return [_LOGICAL[up]]
    try:
        return [int(text)]
    except ValueError:
        pass
    try:
        return [float(up.replace("D", "E"))]
    except ValueError:
        return [text]


def parse_namelist(text):
    """{GROUP: [ {KEY: value, ...}, ... ]} for every ``&GROUP ... /`` in ``text``.
    Keys and group names are upper case; a key with one value maps to the value, with
    several to a list, with none to ``None``."""
    text = _strip_comments(text)
    groups = {}
    pos = 0
    while True:
        m = re.compile(r"&(\w+)").search(text, pos)
        if not m:
            break
        name = m.group(1).upper()
        if name == "END":
            pos = m.end()
            continue
        # the group ends at the first '/' (or &END) outside quotes
        i, q = m.end(), None
        while i < len(text):
            ch = text[i]
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "/" or text[i:i + 4].upper() == "&END":
                break
            i += 1
        body = text[m.end():i]
        pos = i + 1
        toks = _tokens(body)
        entry = {}
        key, vals = None, []
        k = 0
        while k < len(toks):
            t = toks[k]
            if t[0] == "w" and k + 1 < len(toks) and toks[k + 1][0] == "=":
                if key is not None:
                    entry[key] = vals
                key, vals = re.sub(r"\(.*\)$", "", t[1]).upper(), []
                k += 2
                continue
            if t[0] in ("s", "w") and key is not None:
                vals.extend(_value(t))
            k += 1
        if key is not None:
            entry[key] = vals
        for kk, v in list(entry.items()):
            entry[kk] = None if not v else (v[0] if len(v) == 1 else v)
        groups.setdefault(name, []).append(entry)
    return groups


def read_namelist(path):
    with open(path) as fh:
        return parse_namelist(fh.read())


def group(nml, name):
    """The first ``&name`` group of a parsed namelist ({} when absent)."""
    g = nml.get(name.upper())
    return g[0] if g else {}


# --------------------------------------------------------------------------------------
# Cold-start grid files
# --------------------------------------------------------------------------------------
def _header_int(lines, label, path):
    pat = re.compile(re.escape(label) + r"\s*=\s*([-+]?\d+)", re.IGNORECASE)
    for ln in lines:
        m = pat.search(ln)
        if m:
            return int(m.group(1))
    raise ValueError("%s: the header must contain '%s = <integer>'" % (path, label))


def _numeric_rows(lines, ncols):
    """Leading ``ncols`` numbers of every line that starts with that many numbers."""
    rows = []
    for ln in lines:
        parts = ln.replace(",", " ").split()
        if len(parts) < ncols:
            continue
        try:
            rows.append([float(x.replace("D", "E").replace("d", "e")) for x in parts[:ncols]])
        except ValueError:
            continue
    return rows


def _read_lines(path):
    with open(path) as fh:
        return fh.read().splitlines()


def read_grid(path):
    """(x, y, nv_cw): node coordinates and each cell's nodes (1-based) in FVCOM's
    clockwise order, from a ``*_grd.dat`` file whose cells are listed
    counter-clockwise (mod_input.F:3739-3741 stores N1, N3, N2)."""
    lines = _read_lines(path)
    mgl = _header_int(lines, "Node Number", path)
    ngl = _header_int(lines, "Cell Number", path)
    data = [ln for ln in lines if not re.search(r"number", ln, re.IGNORECASE)]
    rows = _numeric_rows(data, 3)
    if len(rows) < ngl + mgl:
        raise ValueError("%s: %d data rows, expected %d cells and %d nodes" % (path, len(rows), ngl, mgl))
    cells = np.array([[int(round(v)) for v in r] for r in _numeric_rows(data[:], 4)[:ngl]], dtype=np.int64)
    if cells.shape[0] != ngl or not np.array_equal(cells[:, 0], np.arange(1, ngl + 1)):
        raise ValueError("%s: the connectivity rows must number the cells 1..%d" % (path, ngl))
    coords = np.array(rows[ngl:ngl + mgl])
    if not np.array_equal(coords[:, 0].astype(np.int64), np.arange(1, mgl + 1)):
        raise ValueError("%s: the coordinate rows must number the nodes 1..%d" % (path, mgl))
    tri = cells[:, 1:4]
    if tri.min() < 1 or tri.max() != mgl:
        raise ValueError("%s: the connectivity must use nodes 1..%d" % (path, mgl))
    x, y = coords[:, 1].copy(), coords[:, 2].copy()
    # IS_TRI_CW on the first cell as FVCOM checks it (mod_input.F:4004-4010)
    a, b, c = tri[0] - 1
    cross = (x[b] - x[a]) * (y[c] - y[a]) - (y[b] - y[a]) * (x[c] - x[a])
    if cross <= 0.0:
        raise ValueError("%s: the nodes of each cell must be listed counter-clockwise" % path)
    nv_cw = np.stack([tri[:, 0], tri[:, 2], tri[:, 1]], axis=1)
    return x, y, nv_cw


def _xyv(path, label, m, x=None, y=None):
    lines = _read_lines(path)
    n = _header_int(lines, label, path)
    if n != m:
        raise ValueError("%s: %d nodes stated, the grid has %d" % (path, n, m))
    data = [ln for ln in lines if not re.search(r"number", ln, re.IGNORECASE)]
    rows = np.array(_numeric_rows(data, 3))
    if rows.shape[0] != m:
        raise ValueError("%s: %d data rows, expected %d" % (path, rows.shape[0], m))
    return rows[:, 2].copy()


def read_depth(path, m):
    """Depth per node from ``X Y H`` rows (mod_input.F:4022-4131)."""
    return _xyv(path, "Node Number", m)


def read_coriolis(path, m):
    """Latitude per node (degrees) from ``X Y LAT`` rows (mod_input.F:4133-4234)."""
    return _xyv(path, "Node Number", m)


def read_obc(path, m):
    """(nodes, types) of the open boundary from ``I NODE TYPE`` rows (mod_input.F:3767)."""
    lines = _read_lines(path)
    n = _header_int(lines, "OBC Node Number", path)
    if n == 0:
        return [], []
    data = [ln for ln in lines if not re.search(r"number", ln, re.IGNORECASE)]
    rows = [[int(round(v)) for v in r] for r in _numeric_rows(data, 3)]
    if len(rows) != n:
        raise ValueError("%s: %d rows, %d stated" % (path, len(rows), n))
    nodes = [r[1] for r in rows]
    types = [r[2] for r in rows]
    if min(nodes) < 1 or max(nodes) > m:
        raise ValueError("%s: open-boundary node outside 1..%d" % (path, m))
    if min(types) < 1 or max(types) > 10:
        raise ValueError("%s: open-boundary type outside 1..10" % path)
    return nodes, types


def read_sponge(path, m):
    """[(node, radius, coefficient)] from ``NODE R C`` rows (mod_input.F:4238-4335)."""
    lines = _read_lines(path)
    n = _header_int(lines, "Sponge Node Number", path)
    if n == 0:
        return []
    data = [ln for ln in lines if not re.search(r"number", ln, re.IGNORECASE)]
    rows = _numeric_rows(data, 3)
    if len(rows) != n:
        raise ValueError("%s: %d rows, %d stated" % (path, len(rows), n))
    out = [(int(round(r[0])), float(r[1]), float(r[2])) for r in rows]
    if any(not 1 <= s[0] <= m for s in out):
        raise ValueError("%s: sponge node outside 1..%d" % (path, m))
    return out


def read_sigma(path):
    """(KB, P_SIGMA) from a sigma file of type UNIFORM or GEOMETRIC (mod_input.F:4338)."""
    kb, stype, power = None, None, None
    for ln in _read_lines(path):
        s = ln.split("!")[0].strip()
        if not s or "=" not in s:
            continue
        key, val = [t.strip() for t in s.split("=", 1)]
        key = key.upper()
        if key == "NUMBER OF SIGMA LEVELS":
            kb = int(val)
        elif key == "SIGMA COORDINATE TYPE":
            stype = val.upper()
        elif key == "SIGMA POWER":
            power = float(val.replace("D", "E"))
    if kb is None or stype is None:
        raise ValueError("%s: needs NUMBER OF SIGMA LEVELS and SIGMA COORDINATE TYPE" % path)
    if stype == "UNIFORM":
        return kb, 1.0
    if stype == "GEOMETRIC":
        if power is None:
            raise ValueError("%s: GEOMETRIC sigma needs SIGMA POWER" % path)
        return kb, power
    raise ValueError("%s: sigma coordinate type %s is not on the supported path "
                     "(UNIFORM, GEOMETRIC)" % (path, stype))


# --------------------------------------------------------------------------------------
# Time
# --------------------------------------------------------------------------------------
def parse_time(spec):
    """('relative', seconds) for 'seconds=', 'days=', 'hours=', 'minutes=' and 'cycle='
    specs, ('date', MJD seconds) for 'YYYY-MM-DD[ HH:MM:SS]' dates, None for 'none'."""
    s = str(spec).strip()
    if not s or s.lower() == "none":
        return None
    m = re.fullmatch(r"(seconds|days|hours|minutes|cycle)\s*=\s*([-+.\deEdD]+)", s, re.IGNORECASE)
    if m:
        unit = m.group(1).lower()
        v = float(m.group(2).replace("D", "E").replace("d", "e"))
        if unit == "cycle":
            return ("cycle", v)
        return ("relative", v * {"seconds": 1.0, "minutes": 60.0, "hours": 3600.0, "days": 86400.0}[unit])
    for fmt in ("%Y-%m-%d %H:%M:%S", "%Y-%m-%dT%H:%M:%S", "%Y-%m-%d %H:%M", "%Y-%m-%d"):
        try:
            t = _dt.datetime.strptime(s.split(".")[0].rstrip("Z"), fmt)
            return ("date", (t - MJD_EPOCH).total_seconds())
        except ValueError:
            continue
    raise ValueError("time '%s' is neither 'unit=value' nor a YYYY-MM-DD date" % s)


def file_times(nc):
    """Record times of a forcing file in seconds (Itime + Itime2, else ``time`` days)."""
    v = nc.variables
    if "Itime" in v and "Itime2" in v:
        return np.asarray(v["Itime"][:], dtype=np.float64) * 86400.0 + \
            np.asarray(v["Itime2"][:], dtype=np.float64) / 1000.0
    if "time" in v:
        return np.asarray(v["time"][:], dtype=np.float64) * 86400.0
    raise ValueError("forcing file has no Itime/Itime2 or time variable")


def bracket(times, now):
    """(prev, next, next_weight) for ``now`` inside the record times, as
    UPDATE_FILE_BRACKET finds them (prev < now <= next; now == first record -> 0, 1)."""
    times = np.asarray(times)
    if times.size < 2:
        raise ValueError("a forcing file needs at least two records")
    if now < times[0] or now > times[-1]:
        raise ValueError("time %.3f s is outside the forcing records [%.3f, %.3f] s"
                         % (now, times[0], times[-1]))
    j = int(np.searchsorted(times, now, side="left"))
    if j == 0:
        j = 1
    numer = now - times[j - 1]
    denom = times[j] - times[j - 1]
    return j - 1, j, numer / denom


# --------------------------------------------------------------------------------------
# Forcing series
# --------------------------------------------------------------------------------------
def _chars(a):
    a = np.asarray(a)
    if a.dtype.kind == "S" and a.ndim == 2:
        return [b"".join(r).decode("latin-1").strip().strip("\x00").strip() for r in a]
    return [str(x).strip() for x in a]


def read_river_namelist(path):
    """NML_RIVER groups in order: dicts name, file, location, distribution."""
    out = []
    for g in read_namelist(path).get("NML_RIVER", []):
        dist = g.get("RIVER_VERTICAL_DISTRIBUTION")
        out.append(dict(name=str(g.get("RIVER_NAME", "")).strip(), file=str(g.get("RIVER_FILE", "")).strip(),
                        location=int(g.get("RIVER_GRID_LOCATION", -1)), distribution=dist))
    return out


class RiverSeries:
    """Discharge, temperature and salinity of the model's rivers from their files; the
    value at a time is the nearer bracketing record (UPDATE_RIVERS, mod_force.F:11330)."""

    def __init__(self, rivers, input_dir, time_offset=0.0):
        self.n = len(rivers)
        self.files = []
        by_file = {}
        for q, r in enumerate(rivers):
            by_file.setdefault(r["file"], []).append((q, r["name"]))
        for fname, members in by_file.items():
            with netcdf_file(os.path.join(input_dir, fname), "r", mmap=False) as nc:
                names = _chars(nc.variables["river_names"][:])
                t = file_times(nc) - time_offset
                flux = np.asarray(nc.variables["river_flux"][:], dtype=np.float64)
                temp = np.asarray(nc.variables["river_temp"][:], dtype=np.float64) \
                    if "river_temp" in nc.variables else None
                salt = np.asarray(nc.variables["river_salt"][:], dtype=np.float64) \
                    if "river_salt" in nc.variables else None
            cols = []
            for q, name in members:
                if name not in names:
                    raise ValueError("river '%s' is not in %s (names: %s)" % (name, fname, names))
                cols.append((q, names.index(name)))
            self.files.append(dict(t=t, flux=flux, temp=temp, salt=salt, cols=cols))

    def at(self, now):
        q = np.zeros(self.n)
        t = np.zeros(self.n)
        s = np.zeros(self.n)
        for f in self.files:
            p, n, wn = bracket(f["t"], now)
            rec = n if (1.0 - wn) <= 0.5 else p  # CURRENT = VNP unless PREV_WGHT > 0.5
            for qi, col in f["cols"]:
                q[qi] = f["flux"][rec, col]
                if f["temp"] is not None:
                    t[qi] = f["temp"][rec, col]
                if f["salt"] is not None:
                    s[qi] = f["salt"][rec, col]
        return q, t, s


class WindSeries:
    """Surface stress per cell before RAMP*0.001 (0:N), constant or from a file."""

    def __init__(self, n_cells, wind_type="stress", kind="constant", wx=0.0, wy=0.0, path=None,
                 time_offset=0.0):
        self.n = n_cells
        self.type = wind_type.lower()
        self.kind = kind.lower()
        if self.type not in ("stress", "speed"):
            raise ValueError("WIND_TYPE '%s' is not 'stress' or 'speed'" % wind_type)
        if self.kind == "constant":
            self.const = (float(wx), float(wy))
        elif self.kind == "variable":
            with netcdf_file(path, "r", mmap=False) as nc:
                self.t = file_times(nc) - time_offset
                ux, uy = ("uwind_stress", "vwind_stress") if self.type == "stress" else ("uwind_speed", "vwind_speed")
                if ux not in nc.variables:
                    raise ValueError("%s has no %s" % (path, ux))
                self.u = np.asarray(nc.variables[ux][:], dtype=np.float64)
                self.v = np.asarray(nc.variables[uy][:], dtype=np.float64)
            if self.u.shape[1] != n_cells:
                raise ValueError("%s: %d cells per record, the grid has %d" % (path, self.u.shape[1], n_cells))
        else:
            raise ValueError("WIND_KIND '%s' is not on the supported path (constant, variable)" % kind)

    def at(self, now):
        if self.kind == "constant":
            u = np.full(self.n, self.const[0])
            v = np.full(self.n, self.const[1])
        else:
            p, n, wn = bracket(self.t, now)
            u = wn * self.u[n] + (1.0 - wn) * self.u[p]
            v = wn * self.v[n] + (1.0 - wn) * self.v[p]
        if self.type == "speed":
            u, v = simple_drag(u, v)
        sx = np.zeros(self.n + 1)
        sy = np.zeros(self.n + 1)
        sx[1:], sy[1:] = u, v
        return sx, sy


class HeatSeries:
    """Short-wave radiation and net heat flux per node in W/m^2 (0:M) before RAMP,
    constant (HEATING_RADIATION, HEATING_NETFLUX) or from a file's short_wave and
    net_heat_flux records interpolated linearly (UPDATE_HEAT, mod_force.F:12427-12539)."""

    def __init__(self, n_nodes, kind="constant", radiation=0.0, netflux=0.0, path=None, time_offset=0.0):
        self.n = n_nodes
        self.kind = kind.lower()
        if self.kind == "constant":
            self.const = (float(radiation), float(netflux))
        elif self.kind == "variable":
            with netcdf_file(path, "r", mmap=False) as nc:
                self.t = file_times(nc) - time_offset
                for need in ("short_wave", "net_heat_flux"):
                    if need not in nc.variables:
                        raise ValueError("%s has no %s" % (path, need))
                self.sw = np.asarray(nc.variables["short_wave"][:], dtype=np.float64)
                self.nf = np.asarray(nc.variables["net_heat_flux"][:], dtype=np.float64)
            if self.sw.shape[1] != n_nodes:
                raise ValueError("%s: %d nodes per record, the grid has %d" % (path, self.sw.shape[1], n_nodes))
        else:
            raise ValueError("HEATING_KIND '%s' is not on the supported path (constant, variable)" % kind)

    def at(self, now):
        sw = np.zeros(self.n + 1)
        nf = np.zeros(self.n + 1)
        if self.kind == "constant":
            sw[1:], nf[1:] = self.const
        else:
            p, n, wn = bracket(self.t, now)
            sw[1:] = wn * self.sw[n] + (1.0 - wn) * self.sw[p]
            nf[1:] = wn * self.nf[n] + (1.0 - wn) * self.nf[p]
        return sw, nf


def read_spectral_tide(path, obc_nodes):
    """Tide dict (period, apt, phai, emean) for the open-boundary list, and the phase
    origin in seconds (time_origin, days)."""
    with netcdf_file(path, "r", mmap=False) as nc:
        v = nc.variables
        for need in ("tide_period", "tide_Eamp", "tide_Ephase"):
            if need not in v:
                raise ValueError("%s is not a spectral elevation file (no %s)" % (path, need))
        nodes = [int(x) for x in np.asarray(v["obc_nodes"][:])]
        period = np.asarray(v["tide_period"][:], dtype=np.float64)
        amp = np.asarray(v["tide_Eamp"][:], dtype=np.float64)      # (ntide, nobc)
        phase = np.asarray(v["tide_Ephase"][:], dtype=np.float64)
        eref = np.asarray(v["tide_Eref"][:], dtype=np.float64) if "tide_Eref" in v else np.zeros(len(nodes))
        origin = float(np.asarray(v["time_origin"].getValue() if "time_origin" in v else 0.0)) * 86400.0
    idx = []
    for nd in obc_nodes:
        if nd not in nodes:
            raise ValueError("%s: open-boundary node %d has no tide" % (path, nd))
        idx.append(nodes.index(nd))
    idx = np.array(idx, dtype=np.int64)
    tide = dict(period=period, apt=amp[:, idx].T.copy(), phai=phase[:, idx].T.copy(), emean=eref[idx].copy())
    return tide, origin


# --------------------------------------------------------------------------------------
# A run directory
# --------------------------------------------------------------------------------------
def _b(v, default=False):
    if v is None:
        return default
    if isinstance(v, bool):
        return v
    return str(v).strip().upper() in ("T", ".TRUE.", "TRUE")


def _s(v, default=""):
    return default if v is None else str(v).strip()


class FvcomRun:
    """An FVCOM case read from its run namelist (``<case>_run.nml``) and input files."""

    def __init__(self, nml_path, input_dir=None, limiter="LIMITED_NO", ghost_cells="GCN"):
        """``limiter`` and ``ghost_cells``: FVCOM's compile-time choices of the momentum
        advection limiter (LIMITED_NO, LIMITED_1, LIMITED_2) and of the solid-boundary
        treatment (GCN, GCY1, GCY2); the run namelist carries neither."""
        self.nml_path = os.path.abspath(nml_path)
        nml = read_namelist(nml_path)
        self.nml = nml
        base = os.path.dirname(self.nml_path)
        io = group(nml, "NML_IO")
        indir = input_dir or os.path.normpath(os.path.join(base, _s(io.get("INPUT_DIR"), ".")))
        self.input_dir = indir
        self.output_dir = os.path.normpath(os.path.join(base, _s(io.get("OUTPUT_DIR"), ".")))
        case_g = group(nml, "NML_CASE")
        self.title = _s(case_g.get("CASE_TITLE"), "fvcom case")
        self.casename = os.path.basename(self.nml_path).rsplit("_run.nml", 1)[0]
        start = parse_time(_s(case_g.get("START_DATE"), "seconds=0"))
        end = parse_time(_s(case_g.get("END_DATE"), "seconds=0"))
        if start is None or end is None or start[0] != end[0] or start[0] == "cycle":
            raise ValueError("START_DATE and END_DATE must both be relative times or both dates")
        self.start, self.end = start[1], end[1]
        # file times are seconds in the same frame as START_DATE: MJD for dates, the
        # relative origin otherwise; time_offset maps them to seconds since the start
        self.time_offset = self.start

        it = group(nml, "NML_INTEGRATION")
        ph = group(nml, "NML_PHYSICS")
        self._check_off(nml)
        dte = float(it.get("EXTSTEP_SECONDS"))
        isplit = int(it.get("ISPLIT"))
        self.dti = dte * isplit
        hm_type = _s(ph.get("HORIZONTAL_MIXING_TYPE"), "closure").lower()
        vm_type = _s(ph.get("VERTICAL_MIXING_TYPE"), "closure").lower()
        if _s(ph.get("HORIZONTAL_MIXING_KIND"), "constant").lower() != "constant":
            raise ValueError("HORIZONTAL_MIXING_KIND other than 'constant' is not on the supported path")
        if _s(ph.get("BOTTOM_ROUGHNESS_KIND"), "constant").lower() != "constant":
            raise ValueError("BOTTOM_ROUGHNESS_KIND other than 'constant' is not on the supported path")
        bpg = _s(ph.get("BAROCLINIC_PRESSURE_GRADIENT"), "sigma levels").lower()
        if bpg not in ("sigma levels", "z coordinates"):
            raise ValueError("BAROCLINIC_PRESSURE_GRADIENT '%s' is not 'sigma levels' or 'z coordinates'" % bpg)
        rt = group(nml, "NML_RIVER_TYPE")
        obc = group(nml, "NML_OPEN_BOUNDARY_CONTROL")
        params = default_params(
            DTE=dte, ISPLIT=isplit, IRAMP=int(it.get("IRAMP", 0)),
            MIN_DEPTH=float(it.get("MIN_DEPTH", 0.05)), STATIC_SSH_ADJ=float(it.get("STATIC_SSH_ADJ", 0.0)),
            HORIZONTAL_MIXING_TYPE=hm_type, HPRNU=float(ph.get("HORIZONTAL_PRANDTL_NUMBER", 1.0)),
            UMOL=float(ph.get("VERTICAL_MIXING_COEFFICIENT", 1e-4)),
            VPRNU=float(ph.get("VERTICAL_PRANDTL_NUMBER", 1.0)),
            CBCMIN=float(ph.get("BOTTOM_ROUGHNESS_MINIMUM", 0.0025)),
            VERTICAL_MIXING_TYPE=vm_type,
            WETTING_DRYING_ON=_b(ph.get("WETTING_DRYING_ON")),
            SCALAR_POSITIVITY_CONTROL=_b(ph.get("SCALAR_POSITIVITY_CONTROL"), True),
            BAROTROPIC=_b(ph.get("BAROTROPIC")),
            TEMPERATURE_ACTIVE=_b(ph.get("TEMPERATURE_ACTIVE"), True),
            SALINITY_ACTIVE=_b(ph.get("SALINITY_ACTIVE"), True),
            OBC_TS_TYPE=int(obc.get("OBC_TS_TYPE", 3)),
            RIVER_TS_SETTING=_s(rt.get("RIVER_TS_SETTING"), "specified").lower(),
            LIMITER=limiter, BAROCLINIC_PRESSURE_GRADIENT=bpg,
        )

        gc = group(nml, "NML_GRID_COORDINATES")
        if _s(gc.get("GRID_FILE_UNITS"), "meters").lower() != "meters":
            raise ValueError("GRID_FILE_UNITS other than 'meters' (spherical) is not on the supported path")
        p = lambda key, default=None: os.path.join(indir, _s(gc.get(key), default))  # noqa: E731
        x, y, nv = read_grid(p("GRID_FILE"))
        m = len(x)
        h = read_depth(p("DEPTH_FILE"), m)
        kb, psig = read_sigma(p("SIGMA_LEVELS_FILE"))
        lat = read_coriolis(p("CORIOLIS_FILE"), m) if _s(gc.get("CORIOLIS_FILE"), "none").lower() != "none" else None
        spg = read_sponge(p("SPONGE_FILE"), m) if _s(gc.get("SPONGE_FILE"), "none").lower() != "none" else []
        if _b(obc.get("OBC_ON")):
            obc_nodes, obc_types = read_obc(os.path.join(indir, _s(obc.get("OBC_NODE_LIST_FILE"))), m)
        else:
            obc_nodes, obc_types = [], []

        nriv = int(rt.get("RIVER_NUMBER", 0) or 0)
        rloc = _s(rt.get("RIVER_INFLOW_LOCATION"), "node").lower()
        rivers_nml = []
        if nriv > 0:
            kind = _s(rt.get("RIVER_KIND"), "variable").lower()
            if kind != "variable":
                raise ValueError("RIVER_KIND '%s' is not on the supported path (variable)" % kind)
            info = _s(rt.get("RIVER_INFO_FILE"), "default")
            src = self.nml_path if info.lower() == "default" else os.path.join(indir, info)
            rivers_nml = read_river_namelist(src)
            if len(rivers_nml) != nriv:
                raise ValueError("RIVER_NUMBER is %d but %d NML_RIVER groups were found" % (nriv, len(rivers_nml)))
        kbm1 = kb - 1
        rivers = []
        for r in rivers_nml:
            d = r["distribution"]
            if isinstance(d, str):
                if d.lower().startswith("unifor"):
                    d = None  # DZ of the river's node or cell, set below (SET_DISTRIBUTION)
                else:
                    raise ValueError("river distribution '%s' is not on the supported path "
                                     "(a list of %d weights, or 'uniform')" % (d, kbm1))
            else:
                d = np.atleast_1d(np.asarray(d, dtype=np.float64))
                if d.size < kbm1:
                    raise ValueError("river '%s': %d distribution weights for %d layers" % (r["name"], d.size, kbm1))
                if np.any(d[:kbm1] < 0.0):
                    raise ValueError("river '%s': negative distribution weight" % r["name"])
                d = d[:kbm1]
            rivers.append(dict(loc=r["location"], dist=d))
        # 'uniform' needs the sigma thicknesses, which are the same at every node for the
        # supported sigma types: the first node's DZ row
        if any(r["dist"] is None for r in rivers):
            probe = build_grid(x, y, nv, h, kb, p_sigma=psig)
            for r in rivers:
                if r["dist"] is None:
                    r["dist"] = probe["DZ"][1, :kbm1].copy()
        grid = build_grid(x, y, nv, h, kb, obc_nodes=obc_nodes, obc_types=obc_types, cor_lat=lat,
                          sponge=spg, horcon=float(ph.get("HORIZONTAL_MIXING_COEFFICIENT", 0.2)),
                          z0b=float(ph.get("BOTTOM_ROUGHNESS_LENGTHSCALE", 0.001)),
                          rivers=rivers, river_location=rloc,
                          static_ssh_adj=float(it.get("STATIC_SSH_ADJ", 0.0)), p_sigma=psig,
                          ghost_cells=ghost_cells)

        tide = None
        if obc_nodes and _b(obc.get("OBC_ELEVATION_FORCING_ON")):
            tide, origin = read_spectral_tide(os.path.join(indir, _s(obc.get("OBC_ELEVATION_FILE"))), obc_nodes)
            params["TIDE_REF_TIME"] = origin - self.time_offset
        self.rivers = RiverSeries(rivers_nml, indir, self.time_offset) if rivers_nml else None
        sf = group(nml, "NML_SURFACE_FORCING")
        self.wind = None
        if _b(sf.get("WIND_ON")):
            kind = _s(sf.get("WIND_KIND"), "constant").lower()
            wpath = os.path.join(indir, _s(sf.get("WIND_FILE"))) if kind == "variable" else None
            self.wind = WindSeries(grid["N"], _s(sf.get("WIND_TYPE"), "stress"), kind,
                                   float(sf.get("WIND_X", 0.0) or 0.0), float(sf.get("WIND_Y", 0.0) or 0.0),
                                   wpath, self.time_offset)

        self.heat = None
        if _b(sf.get("HEATING_ON")):
            kind = _s(sf.get("HEATING_KIND"), "constant").lower()
            hpath = os.path.join(indir, _s(sf.get("HEATING_FILE"))) if kind == "variable" else None
            self.heat = HeatSeries(grid["M"], kind, float(sf.get("HEATING_RADIATION", 0.0) or 0.0),
                                   float(sf.get("HEATING_NETFLUX", 0.0) or 0.0), hpath, self.time_offset)
            params.update(HEATING_ON=True,
                          HEATING_LONGWAVE_PERCTAGE=float(sf.get("HEATING_LONGWAVE_PERCTAGE", 0.78)),
                          HEATING_LONGWAVE_LENGTHSCALE=float(sf.get("HEATING_LONGWAVE_LENGTHSCALE", 1.4)),
                          HEATING_SHORTWAVE_LENGTHSCALE=float(sf.get("HEATING_SHORTWAVE_LENGTHSCALE", 6.3)))

        st = group(nml, "NML_STARTUP")
        stype = _s(st.get("STARTUP_TYPE"), "coldstart").lower()
        if stype != "coldstart":
            raise ValueError("STARTUP_TYPE '%s': only 'coldstart' is read from a namelist; restarts are "
                             "loaded with ncio.read_restart" % stype)
        ts = _s(st.get("STARTUP_TS_TYPE"), "constant").lower()
        tv, sv = st.get("STARTUP_T_VALS"), st.get("STARTUP_S_VALS")
        if ts == "constant":
            init = dict(kind="constant", t=float(np.atleast_1d(tv)[0]), s=float(np.atleast_1d(sv)[0]))
        elif ts == "linear_sigma":  # this library's linear-in-sigma start (not an FVCOM option)
            tv, sv = np.atleast_1d(tv), np.atleast_1d(sv)
            init = dict(kind="linear_sigma", t=(float(tv[0]), float(tv[-1])), s=(float(sv[0]), float(sv[-1])))
        else:
            raise ValueError("STARTUP_TS_TYPE '%s' is not on the supported path (constant)" % ts)

        nq = len(rivers)
        q0, t0, s0 = self.rivers.at(self.dti) if self.rivers else (np.zeros(0),) * 3
        forcing = dict(tide=tide, qdis=q0, tdis=t0, sdis=s0, wind=None)
        if self.wind is not None:
            sx, sy = self.wind.at(self.dti)
            forcing["wind"] = dict(kind="field", sx=sx, sy=sy)
        if self.heat is not None:
            sw, nf = self.heat.at(self.dti)
            forcing["heat"] = dict(swrad=sw, wtsurf=nf)
        assert len(q0) == nq
        self.case = dict(grid=grid, forcing=forcing, params=params, init=init, name=self.casename)

        nc = group(nml, "NML_NETCDF")
        self.nc_on = _b(nc.get("NC_ON"))
        first = parse_time(_s(nc.get("NC_FIRST_OUT"), "none"))
        inter = parse_time(_s(nc.get("NC_OUT_INTERVAL"), "none"))
        self.nc_first = None if first is None else (first[1] * self.dti if first[0] == "cycle"
                                                    else first[1] - (self.start if first[0] == "date" else 0.0))
        self.nc_interval = None if inter is None else (inter[1] * self.dti if inter[0] == "cycle" else inter[1])

    @staticmethod
    def _check_off(nml):
        sf = group(nml, "NML_SURFACE_FORCING")
        for key in ("HEATING_CALCULATE_ON", "PRECIPITATION_ON", "AIRPRESSURE_ON", "WAVE_ON", "ICE_MODEL"):
            if _b(sf.get(key)):
                raise ValueError("%s = T is not on the supported path" % key)
        if _b(sf.get("HEATING_ON")) and _s(sf.get("HEATING_TYPE"), "flux").lower() != "flux":
            raise ValueError("HEATING_TYPE '%s' is not on the supported path (flux)" % sf.get("HEATING_TYPE"))
        gw = group(nml, "NML_GROUNDWATER")
        if _b(gw.get("GROUNDWATER_ON")):
            raise ValueError("GROUNDWATER_ON = T is not on the supported path")
        obc = group(nml, "NML_OPEN_BOUNDARY_CONTROL")
        for key in ("OBC_TEMP_NUDGING", "OBC_SALT_NUDGING", "OBC_MEANFLOW", "OBC_LONGSHORE_FLOW_ON"):
            if _b(obc.get(key)):
                raise ValueError("%s = T is not on the supported path" % key)

    @property
    def steps(self):
        """Internal steps from START_DATE to END_DATE."""
        return int(round((self.end - self.start) / self.dti))

    def forcing_at(self, t):
        """``case["forcing"]`` with rivers and wind evaluated at ``t`` s after the start."""
        f = dict(self.case["forcing"])
        if self.rivers is not None:
            f["qdis"], f["tdis"], f["sdis"] = self.rivers.at(t)
        if self.wind is not None:
            sx, sy = self.wind.at(t)
            f["wind"] = dict(kind="field", sx=sx, sy=sy)
        if self.heat is not None:
            sw, nf = self.heat.at(t)
            f["heat"] = dict(swrad=sw, wtsurf=nf)
        return f

    def step(self, model):
        """One internal step: the forcing at the step's IntTime, then INTERNAL_STEP."""
        iint, _ = model.clock()
        if self.rivers is not None or self.wind is not None or self.heat is not None:
            model.set_forcing(self.forcing_at((iint + 1) * self.dti))
        model.internal_step()

    def run(self, model, steps=None, history=None):
        """Step ``model`` (an engine built from ``self.case``) ``steps`` internal steps
        (default: to END_DATE), writing a history record at NC_FIRST_OUT and every
        NC_OUT_INTERVAL after it to ``history`` (an ``ncio.History``) when given."""
        steps = self.steps if steps is None else int(steps)
        every = None
        if history is not None and self.nc_interval:
            every = max(1, int(round(self.nc_interval / self.dti)))
            first = int(round((self.nc_first or 0.0) / self.dti))
            if first == 0:
                history.write(model)
        for n in range(1, steps + 1):
            self.step(model)
            if every and n >= first and (n - first) % every == 0:
                history.write(model)
        return model


# --------------------------------------------------------------------------------------
# Writing a case as an FVCOM run directory
# --------------------------------------------------------------------------------------
def _w(path, lines):
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def _fmt(v):
    return repr(float(v))


def write_run(case, directory, name="case", days=1.0, river_series=None, wind_series=None,
              heat_series=None):
    """Write ``case`` as an FVCOM run directory (``<name>_run.nml`` and the input files
    it names) and return the namelist path.

    river_series: optional (times_s, flux, temp, salt) arrays (records x rivers);
    wind_series: optional (times_s, sx, sy) arrays (records x cells) of wind stress;
    heat_series: optional (times_s, short_wave, net_heat_flux) arrays (records x nodes).
    Without them the case's constant values are written as two records spanning the run.
    """
    g, p, fc = case["grid"], case["params"], case["forcing"]
    os.makedirs(directory, exist_ok=True)
    M, N, KB = g["M"], g["N"], g["KB"]
    vx = g["VX"][1:] + g.a.get("VXMIN", 0.0)
    vy = g["VY"][1:] + g.a.get("VYMIN", 0.0)
    nv = np.asarray(g["NV"][1:])
    lines = ["Node Number = %d" % M, "Cell Number = %d" % N]
    for i in range(N):  # back to counter-clockwise: N1, N3, N2
        lines.append("%d %d %d %d 1" % (i + 1, nv[i, 0], nv[i, 2], nv[i, 1]))
    for i in range(M):
        lines.append("%d %s %s 0.0" % (i + 1, _fmt(vx[i]), _fmt(vy[i])))
    _w(os.path.join(directory, name + "_grd.dat"), lines)
    h = g["H"][1:] - float(p.get("STATIC_SSH_ADJ", 0.0))
    _w(os.path.join(directory, name + "_dep.dat"),
       ["Node Number = %d" % M] + ["%s %s %s" % (_fmt(vx[i]), _fmt(vy[i]), _fmt(h[i])) for i in range(M)])
    lat = g["LAT"]
    _w(os.path.join(directory, name + "_cor.dat"),
       ["Node Number = %d" % M] + ["%s %s %s" % (_fmt(vx[i]), _fmt(vy[i]), _fmt(lat[i + 1])) for i in range(M)])
    spg = g.a.get("SPONGE_LIST", [])
    _w(os.path.join(directory, name + "_spg.dat"),
       ["Sponge Node Number = %d" % len(spg)] + ["%d %s %s" % (n, _fmt(r), _fmt(c)) for n, r, c in spg])
    nob = g["IOBCN"]
    obc_nodes = [int(g["I_OBC_N"][i]) for i in range(1, nob + 1)]
    obc_types = [int(g["TYPE_OBC"][i]) for i in range(1, nob + 1)]
    _w(os.path.join(directory, name + "_obc.dat"),
       ["OBC Node Number = %d" % nob] + ["%d %d %d" % (i + 1, obc_nodes[i], obc_types[i]) for i in range(nob)])
    psig = g.a.get("P_SIGMA", 1.0)
    _w(os.path.join(directory, "sigma.dat"),
       ["NUMBER OF SIGMA LEVELS = %d" % KB] +
       (["SIGMA COORDINATE TYPE = UNIFORM"] if psig == 1.0 else
        ["SIGMA COORDINATE TYPE = GEOMETRIC", "SIGMA POWER = %s" % _fmt(psig)]))

    dti = p["DTE"] * p["ISPLIT"]
    end = days * 86400.0
    tide = fc.get("tide")
    if tide is not None and nob:
        with netcdf_file(os.path.join(directory, name + "_el_obc.nc"), "w", version=1) as nc:
            nc.type = "FVCOM SPECTRAL ELEVATION FORCING FILE"
            nt = len(tide["period"])
            nc.createDimension("nobc", nob)
            nc.createDimension("tidal_components", nt)
            v = nc.createVariable("obc_nodes", "i", ("nobc",)); v[:] = obc_nodes
            v = nc.createVariable("tide_period", "d", ("tidal_components",)); v[:] = tide["period"]
            v = nc.createVariable("tide_Eref", "d", ("nobc",)); v[:] = tide["emean"]
            v = nc.createVariable("tide_Ephase", "d", ("tidal_components", "nobc")); v[:] = np.asarray(tide["phai"]).T
            v = nc.createVariable("tide_Eamp", "d", ("tidal_components", "nobc")); v[:] = np.asarray(tide["apt"]).T
            v = nc.createVariable("time_origin", "d", ()); v[()] = p.get("TIDE_REF_TIME", 0.0) / 86400.0
    nq = g["NUMQBC"]
    rloc = g["RIVER_LOC"]
    if nq:
        if river_series is None:
            tt = np.array([0.0, end + dti])
            river_series = (tt, np.tile(fc["qdis"], (2, 1)), np.tile(fc["tdis"], (2, 1)), np.tile(fc["sdis"], (2, 1)))
        tt, fl, te, sa = river_series
        with netcdf_file(os.path.join(directory, name + "_riv.nc"), "w", version=1) as nc:
            nc.type = "FVCOM RIVER FORCING FILE"
            nc.createDimension("time", None)
            nc.createDimension("rivers", nq)
            nc.createDimension("namelen", 26)
            names = np.array([list(("river%d" % (q + 1)).ljust(26)) for q in range(nq)], dtype="S1")
            v = nc.createVariable("river_names", "c", ("rivers", "namelen")); v[:] = names
            v = nc.createVariable("time", "d", ("time",)); v[:] = np.asarray(tt) / 86400.0
            v.units = "days since 0.0"
            for key, arr in (("river_flux", fl), ("river_temp", te), ("river_salt", sa)):
                v = nc.createVariable(key, "d", ("time", "rivers")); v[:] = np.asarray(arr)
        dist = np.asarray(g["VQDIST"])
        riv = []
        for q in range(1, nq + 1):
            loc = int(g["INODEQ"][q]) if rloc == "node" else int(g["ICELLQ"][q])
            riv += [" &NML_RIVER", " RIVER_NAME = 'river%d'" % q, " RIVER_FILE = '%s_riv.nc'" % name,
                    " RIVER_GRID_LOCATION = %d," % loc,
                    " RIVER_VERTICAL_DISTRIBUTION = " + " ".join(_fmt(w) for w in dist[q, :KB - 1]), " /", ""]
        _w(os.path.join(directory, "RIVERS_NAMELIST.nml"), riv)
    wind_lines = [" WIND_ON = F,"]
    if fc.get("wind") is not None or wind_series is not None:
        if wind_series is None:
            from .abi import wind_stress
            sx, sy = wind_stress(case)
            wind_series = (np.array([0.0, end + dti]), np.tile(sx[1:], (2, 1)), np.tile(sy[1:], (2, 1)))
        tt, sx, sy = wind_series
        with netcdf_file(os.path.join(directory, name + "_wnd.nc"), "w", version=1) as nc:
            nc.type = "FVCOM WIND FORCING FILE"
            nc.createDimension("time", None)
            nc.createDimension("nele", N)
            v = nc.createVariable("time", "d", ("time",)); v[:] = np.asarray(tt) / 86400.0
            v = nc.createVariable("uwind_stress", "d", ("time", "nele")); v[:] = np.asarray(sx)
            v = nc.createVariable("vwind_stress", "d", ("time", "nele")); v[:] = np.asarray(sy)
        wind_lines = [" WIND_ON = T,", " WIND_TYPE = 'stress',", " WIND_KIND = 'variable',",
                      " WIND_FILE = '%s_wnd.nc'," % name]
    heat_lines = [" HEATING_ON = F,"]
    if p.get("HEATING_ON"):
        if heat_series is None:
            from .abi import heat_flux
            sw, nf = heat_flux(case)
            heat_series = (np.array([0.0, end + dti]), np.tile(sw[1:], (2, 1)), np.tile(nf[1:], (2, 1)))
        tt, sw, nf = heat_series
        with netcdf_file(os.path.join(directory, name + "_hfx.nc"), "w", version=1) as nc:
            nc.type = "FVCOM HEAT FLUX FORCING FILE"
            nc.createDimension("time", None)
            nc.createDimension("node", M)
            v = nc.createVariable("time", "d", ("time",)); v[:] = np.asarray(tt) / 86400.0
            v = nc.createVariable("short_wave", "d", ("time", "node")); v[:] = np.asarray(sw)
            v = nc.createVariable("net_heat_flux", "d", ("time", "node")); v[:] = np.asarray(nf)
        heat_lines = [" HEATING_ON = T,", " HEATING_TYPE = 'flux',", " HEATING_KIND = 'variable',",
                      " HEATING_FILE = '%s_hfx.nc'," % name,
                      " HEATING_LONGWAVE_PERCTAGE = %s," % _fmt(p["HEATING_LONGWAVE_PERCTAGE"]),
                      " HEATING_LONGWAVE_LENGTHSCALE = %s," % _fmt(p["HEATING_LONGWAVE_LENGTHSCALE"]),
                      " HEATING_SHORTWAVE_LENGTHSCALE = %s," % _fmt(p["HEATING_SHORTWAVE_LENGTHSCALE"])]
    init = case["init"]
    if init["kind"] == "constant":
        tsl = [" STARTUP_TS_TYPE = 'constant',", " STARTUP_T_VALS = %s," % _fmt(init["t"]),
               " STARTUP_S_VALS = %s," % _fmt(init["s"])]
    else:
        tsl = [" STARTUP_TS_TYPE = 'linear_sigma',",
               " STARTUP_T_VALS = %s %s," % tuple(_fmt(v) for v in init["t"]),
               " STARTUP_S_VALS = %s %s," % tuple(_fmt(v) for v in init["s"])]
    L = lambda b: "T" if b else "F"  # noqa: E731
    nml = [
        " &NML_CASE", " CASE_TITLE = '%s'," % case.get("name", name), " START_DATE = 'seconds=0.0',",
        " END_DATE = 'seconds=%s'," % _fmt(end), " /",
        " &NML_STARTUP", " STARTUP_TYPE = 'coldstart',"] + tsl + [" /",
        " &NML_IO", " INPUT_DIR = './',", " OUTPUT_DIR = './',", " /",
        " &NML_INTEGRATION", " EXTSTEP_SECONDS = %s," % _fmt(p["DTE"]), " ISPLIT = %d," % p["ISPLIT"],
        " IRAMP = %d," % p["IRAMP"], " MIN_DEPTH = %s," % _fmt(p["MIN_DEPTH"]),
        " STATIC_SSH_ADJ = %s," % _fmt(p["STATIC_SSH_ADJ"]), " /",
        " &NML_NETCDF", " NC_ON = T,", " NC_FIRST_OUT = 'seconds=0.0',",
        " NC_OUT_INTERVAL = 'seconds=%s'," % _fmt(3600.0), " /",
        " &NML_SURFACE_FORCING"] + wind_lines + heat_lines + [" PRECIPITATION_ON = F,",
                                                              " AIRPRESSURE_ON = F,", " /",
        " &NML_PHYSICS", " HORIZONTAL_MIXING_TYPE = '%s'," % p["HORIZONTAL_MIXING_TYPE"],
        " HORIZONTAL_MIXING_KIND = 'constant',",
        " HORIZONTAL_MIXING_COEFFICIENT = %s," % _fmt(g["CC_HVC"][1]),
        " HORIZONTAL_PRANDTL_NUMBER = %s," % _fmt(p["HPRNU"]),
        " VERTICAL_MIXING_TYPE = '%s'," % p["VERTICAL_MIXING_TYPE"],
        " VERTICAL_MIXING_COEFFICIENT = %s," % _fmt(p["UMOL"]),
        " VERTICAL_PRANDTL_NUMBER = %s," % _fmt(p["VPRNU"]),
        " BOTTOM_ROUGHNESS_KIND = 'constant',",
        " BOTTOM_ROUGHNESS_LENGTHSCALE = %s," % _fmt(g["CC_Z0B"][1]),
        " BOTTOM_ROUGHNESS_MINIMUM = %s," % _fmt(p["CBCMIN"]),
        " SCALAR_POSITIVITY_CONTROL = %s," % L(p["SCALAR_POSITIVITY_CONTROL"]),
        " BAROTROPIC = %s," % L(p["BAROTROPIC"]),
        " BAROCLINIC_PRESSURE_GRADIENT = '%s'," % p.get("BAROCLINIC_PRESSURE_GRADIENT", "sigma levels"),
        " TEMPERATURE_ACTIVE = %s," % L(p["TEMPERATURE_ACTIVE"]),
        " SALINITY_ACTIVE = %s," % L(p["SALINITY_ACTIVE"]),
        " WETTING_DRYING_ON = %s," % L(p["WETTING_DRYING_ON"]), " /",
        " &NML_RIVER_TYPE", " RIVER_NUMBER = %d," % nq,
        " RIVER_TS_SETTING = '%s'," % p["RIVER_TS_SETTING"], " RIVER_INFLOW_LOCATION = '%s'," % rloc,
        " RIVER_INFO_FILE = 'RIVERS_NAMELIST.nml',", " RIVER_KIND = 'variable',", " /",
        " &NML_OPEN_BOUNDARY_CONTROL", " OBC_ON = %s," % L(nob > 0),
        " OBC_NODE_LIST_FILE = '%s_obc.dat'," % name,
        " OBC_ELEVATION_FORCING_ON = %s," % L(tide is not None and nob > 0),
        " OBC_ELEVATION_FILE = '%s_el_obc.nc'," % name, " OBC_TS_TYPE = %d," % p["OBC_TS_TYPE"], " /",
        " &NML_GRID_COORDINATES", " GRID_FILE = %s_grd.dat," % name, " GRID_FILE_UNITS = 'meters',",
        " SIGMA_LEVELS_FILE = 'sigma.dat',", " DEPTH_FILE = '%s_dep.dat'," % name,
        " CORIOLIS_FILE = '%s_cor.dat'," % name, " SPONGE_FILE = '%s_spg.dat'," % name, " /",
    ]
    path = os.path.join(directory, name + "_run.nml")
    _w(path, nml)
    return path

