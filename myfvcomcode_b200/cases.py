"""Seeded synthetic FVCOM cases.

No public dataset is named for this path, so every case is generated here with the
shapes, sizes and forcing the workloads call for:

* ``estuary_channel``: the idealised estuary channel, 20 km x 4 km, a 100 x 20 structured
  grid split diagonally (2,121 nodes, 4,000 cells), depth linear 5 -> 20 m seaward, M2
  tide of 1.0 m on the 21 seaward nodes, one 100 m^3/s fresh river at the head,
  T = 15 C / S = 30 initially, MY2.5, DTE = 2 s, ISPLIT = 10, no wetting and drying,
  a sponge layer (radius 6 km, coefficient 0.01) at the open boundary.
  ``nx``/``ny``/``kb`` shrink it for quick tests.  ``ghost_cells`` (both cases) selects
  FVCOM's solid-boundary treatment: "GCN", "GCY1" or "GCY2".
* ``coastal_mesh``: the large coastal mesh, a Delaunay triangulation of jittered lattice
  points in a 200 km x 100 km box (200,000 points by default), bathymetry
  5 m + 195 m x a smoothed Gaussian random field (correlation length 10 km) with a
  2 m intertidal strip along the coast, wetting and drying on, 40 sigma layers, M2+S2
  open-boundary tide (0.8/0.3 m, seeded phases), T/S stratified 20 -> 8 C and 30 -> 35
  linearly in sigma, uniform 10 m/s wind at a seeded heading, a sponge layer (radius
  10 km, coefficient 0.01) along the open boundary.

The node order of every triangle is produced counter-clockwise, as FVCOM grid files
store it, and then swapped to the clockwise order FVCOM uses internally
(FVCOM_source/mod_input.F:3739-3741).
"""
from __future__ import annotations

import numpy as np

from .grid import build_grid, _f4

M2_PERIOD = 44712.0
S2_PERIOD = 43200.0


def _ccw_to_fvcom(tri):
    tri = np.asarray(tri, dtype=np.int64)
    return np.stack([tri[:, 0], tri[:, 2], tri[:, 1]], axis=1) + 1


def _structured(nx, ny, lx, ly, flip=()):
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    vx = X.ravel()
    vy = Y.ravel()

    def nid(i, j):
        return i * (ny + 1) + j

    tri = []
    for i in range(nx):
        for j in range(ny):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if (i, j) in flip:
                tri.append((a, b, d))
                tri.append((b, c, d))
            else:
                tri.append((a, b, c))
                tri.append((a, c, d))
    return vx, vy, np.array(tri), nid


def default_params(**kw):
    """Run-time parameters (the namelist keys the step reads), FVCOM defaults where the
    Estuary example (Examples/Estuary/run/tst_run.nml) gives them."""
    p = dict(
        DTE=2.0, ISPLIT=10, IRAMP=360, MIN_DEPTH=0.05, STATIC_SSH_ADJ=0.0,
        HORIZONTAL_MIXING_TYPE="closure", HPRNU=1.0,
        UMOL=1.0e-4, VPRNU=1.0, CBCMIN=0.0025,
        WETTING_DRYING_ON=False, SCALAR_POSITIVITY_CONTROL=True,
        BAROTROPIC=False, TEMPERATURE_ACTIVE=True, SALINITY_ACTIVE=True,
        OBC_TS_TYPE=3, RIVER_TS_SETTING="specified",
        VERTICAL_MIXING_TYPE="closure",
    )
    p.update(kw)
    return p


def estuary_channel(nx=100, ny=20, kb=11, lx=20000.0, ly=4000.0, river_q=100.0,
                    river_location="node", lat=30.0, river=True, sponge=True, ghost_cells="GCN", **pkw):
    # The lower seaward corner quad is split along its other diagonal so that no cell
    # has one open and one solid side (tge.F:563-580 rejects such cells).
    vx, vy, tri, nid = _structured(nx, ny, lx, ly, flip={(nx - 1, 0)})
    nv = _ccw_to_fvcom(tri)
    h = 5.0 + 15.0 * vx / lx
    obc = [nid(nx, j) + 1 for j in range(ny + 1)]
    if river_location == "node":
        rloc = nid(0, ny // 2) + 1
    else:
        # Head cell on the x = 0 boundary at mid-channel: cell (i=0, j) second triangle.
        rloc = 2 * (ny // 2) + 2
    kbm1 = kb - 1
    rivers = [dict(loc=rloc, dist=[1.0 / kbm1] * kbm1)] if river else []
    # Sponge layer at the open boundary, as FVCOM's Estuary example carries one
    # (Examples/Estuary/tstinp/tst_spg.dat): centred on the middle open-boundary node,
    # radius 0.3 of the channel length, coefficient 0.01.  Without it the corner where
    # the open boundary meets the wall grows grid-scale noise after about 0.6 day.
    spg = [(obc[len(obc) // 2], 0.3 * lx, 0.01)] if sponge else ()
    g = build_grid(vx, vy, nv, h, kb, obc_nodes=obc, obc_types=[1] * len(obc),
                   cor_lat=lat, sponge=spg, horcon=0.2, z0b=0.001,
                   rivers=rivers, river_location=river_location, ghost_cells=ghost_cells)
    n_obc = len(obc)
    tide = dict(period=np.array([M2_PERIOD]), apt=np.full((n_obc, 1), 1.0),
                phai=np.zeros((n_obc, 1)), emean=np.zeros(n_obc))
    nq = len(rivers)
    forcing = dict(tide=tide, qdis=np.full(nq, river_q), tdis=np.full(nq, 15.0),
                   sdis=np.zeros(nq), wind=None)
    params = default_params(**pkw)
    init = dict(kind="constant", t=15.0, s=30.0)
    return dict(grid=g, forcing=forcing, params=params, init=init,
                name="estuary-channel-%dx%d-k%d" % (nx, ny, kb - 1))


def _grf(rng, lx, ly, corr, res=1000.0):
    from scipy.ndimage import gaussian_filter
    nxg = int(lx / res) + 1
    nyg = int(ly / res) + 1
    w = rng.standard_normal((nxg, nyg))
    f = gaussian_filter(w, sigma=corr / res, mode="reflect")
    f = (f - f.min()) / (f.max() - f.min())
    return f, res


def _bilinear(f, res, x, y):
    nxg, nyg = f.shape
    gx = np.clip(x / res, 0, nxg - 1 - 1e-9)
    gy = np.clip(y / res, 0, nyg - 1 - 1e-9)
    i0 = np.floor(gx).astype(int)
    j0 = np.floor(gy).astype(int)
    tx = gx - i0
    ty = gy - j0
    return ((1 - tx) * (1 - ty) * f[i0, j0] + tx * (1 - ty) * f[i0 + 1, j0]
            + (1 - tx) * ty * f[i0, j0 + 1] + tx * ty * f[i0 + 1, j0 + 1])


def coastal_mesh(npts=200000, kb=41, lx=200000.0, ly=100000.0, seed=1234, lat=40.0,
                 wind_speed=10.0, dte=2.0, blend=6000.0, sponge=(10000.0, 0.01), ghost_cells="GCN", **pkw):
    """Jittered-lattice Delaunay coastal mesh; ``npts`` sets the approximate node count.

    ``sponge`` = (radius m, coefficient) of a sponge layer centred on every open-boundary
    node (None: no sponge).  Without it the open boundary's south-east corner grows a
    current that ends the run after about 4.5 simulated hours.
    """
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    nxp = max(int(round(np.sqrt(npts * lx / ly))), 4)
    nyp = max(int(round(npts / nxp)), 3)
    xs = np.linspace(0.0, lx, nxp)
    ys = np.linspace(0.0, ly, nyp)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    dx, dy = xs[1] - xs[0], ys[1] - ys[0]
    jx = rng.uniform(-0.3, 0.3, X.shape) * dx
    jy = rng.uniform(-0.3, 0.3, Y.shape) * dy
    interior_x = (X > 0) & (X < lx)
    interior_y = (Y > 0) & (Y < ly)
    X = X + np.where(interior_x & interior_y, jx, 0.0)
    Y = Y + np.where(interior_x & interior_y, jy, 0.0)
    vx = X.ravel()
    vy = Y.ravel()
    tri = Delaunay(np.stack([vx, vy], axis=1)).simplices
    # Orient counter-clockwise and drop slivers on the straight hull.
    p0, p1, p2 = tri[:, 0], tri[:, 1], tri[:, 2]
    cross = (vx[p1] - vx[p0]) * (vy[p2] - vy[p0]) - (vx[p2] - vx[p0]) * (vy[p1] - vy[p0])
    keep = np.abs(cross) > 1e-6 * dx * dy
    tri = tri[keep]
    cross = cross[keep]
    tri = np.where((cross < 0)[:, None], tri[:, [0, 2, 1]], tri)
    # Number the cells in the same column-major lattice order as the nodes (x strip, then
    # y), as mesh generators emit them; Delaunay returns triangles in arbitrary order.
    cxs = (vx[tri[:, 0]] + vx[tri[:, 1]] + vx[tri[:, 2]]) / 3.0
    cys = (vy[tri[:, 0]] + vy[tri[:, 1]] + vy[tri[:, 2]]) / 3.0
    order = np.lexsort((cys, np.floor(cxs / dx)))
    tri = tri[order]
    nv = _ccw_to_fvcom(tri)
    f, res = _grf(rng, lx, ly, 10000.0)
    h = 5.0 + 195.0 * _bilinear(f, res, vx, vy)
    # Intertidal shelf strip along the western coast: depth runs -1 m .. +1 m over the
    # first 4 km, blending into the deep field by 10 km.
    strip = -1.0 + 2.0 * np.clip(vx / 4000.0, 0.0, 1.0)
    w = np.clip((vx - 4000.0) / blend, 0.0, 1.0)
    h = np.where(vx < 4000.0, strip, (1 - w) * 1.0 + w * h)
    # Open boundary: the eastern side x = lx without its two corner nodes, so that no
    # cell has one open and one solid side (tge.F:563-580).
    obc = list(np.nonzero(np.isclose(vx, lx) & (vy > 0.0) & (vy < ly))[0] + 1)
    obc.sort(key=lambda n: vy[n - 1])
    spg = ()
    if sponge is not None:
        radius, coef = sponge
        spg = [(n, radius, coef) for n in obc]
    g = build_grid(vx, vy, nv, h, kb, obc_nodes=obc, obc_types=[1] * len(obc),
                   cor_lat=lat, sponge=spg, horcon=0.2, z0b=0.001, rivers=[],
                   river_location="node", ghost_cells=ghost_cells)
    n_obc = len(obc)
    ph = rng.uniform(0.0, 360.0, 2)
    tide = dict(period=np.array([M2_PERIOD, S2_PERIOD]),
                apt=np.tile(np.array([0.8, 0.3]), (n_obc, 1)),
                phai=np.tile(ph, (n_obc, 1)), emean=np.zeros(n_obc))
    heading = rng.uniform(0.0, 2 * np.pi)
    forcing = dict(tide=tide, qdis=np.zeros(0), tdis=np.zeros(0), sdis=np.zeros(0),
                   wind=dict(kind="speed", u=wind_speed * np.cos(heading),
                             v=wind_speed * np.sin(heading)))
    params = default_params(DTE=dte, WETTING_DRYING_ON=True, **pkw)
    init = dict(kind="linear_sigma", t=(20.0, 8.0), s=(30.0, 35.0))
    return dict(grid=g, forcing=forcing, params=params, init=init,
                name="coastal-%dk-k%d" % (round(g["M"] / 1000), kb - 1))


def simple_drag(u, v):
    """Wind speed to stress, PSIMPLE_DRAG (FVCOM_source/mod_bulk.F:58-92)."""
    u = np.asarray(u, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    wds = np.sqrt(u * u + v * v)
    cd = np.full_like(wds, _f4(1.2e-3))
    cd = np.where(wds >= 11.0, (0.49 + 0.065 * wds) * 1.0e-3, cd)
    cd = np.where(wds >= 25.0, (0.49 + 0.065 * 25.0) * 1.0e-3, cd)
    return 1.2 * cd * u * wds, 1.2 * cd * v * wds
