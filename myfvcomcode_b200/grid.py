"""FVCOM grid metrics: the arrays FVCOM's GRID_METRICS builds before the first step.

This module plays FVCOM's set-up role so the time-step library can be driven
without the Fortran host.  It reproduces, array for array, what the reference
computes at start-up:

* TRIANGLE_GRID_EDGE  (FVCOM_source/tge.F:29-866): NBE, ISBCE, ISONB, NTVE/NBVE/NBVT,
  NTSN/NBSN, the element edges IEC/IENODE/ISBC/XIJC/YIJC/DLTXC/DLTYC and the
  control-volume half-edges NIEC/NTRG/DLTXE/DLTYE, EPOR.
* CELL_AREA           (FVCOM_source/cell_area.F:40-352): ART, ART1, ART2.
* SHAPE_COEF_GCN      (FVCOM_source/shape_coef_gcn.F:29-368): A1U, A2U, AWX, AWY, AW0, ALPHA.
* EDGE_LEN            (FVCOM_source/edge_len.F:29-241): DLTXNCVE/DLTYNCVE, DLTXTRIE/DLTYTRIE,
  DLTXECEC/DLTYECEC, DLTXNEC/DLTYNEC.
* DEPTH_GRADIENT      (FVCOM_source/depth_grad.F:33-90): SITA_GD, PHPN.
* SETUP_OBC           (FVCOM_source/mod_obcs.F:868-1173): NEXT_OBC, NADJC_OBC/ADJC_OBC,
  FLUXF_OBC, DLTN_OBC, IUCP.
* SETUP_CENTER_COORDS / SETUP_CORIOLIS / SETUP_SPONGE / SIGMA_GEOMETRIC /
  SETUP_SIGMA_DERIVATIVES / SET_WATER_DEPTH (FVCOM_source/mod_setup.F:62-1091,
  FVCOM_source/mod_startup.F:1408-1495).
* SET_RIVER_BNDRY_METRICS (FVCOM_source/mod_force.F:3447-3581).

Array convention (shared with the C ABI in include/fvg.h): every per-node, per-cell,
per-edge and per-half-edge array carries FVCOM's 1-based index with a ghost row 0,
shape (len+1,) or (len+1, cols) with cols 0-based; column-major (Fortran order) when
handed to C, so element (i, j) of a 2-D array sits at a[j*(len+1) + i].

The mesh arrays are set-up data, not the hot path; the arithmetic follows the
reference's expression order so the metrics equal FVCOM's, but nothing here is
timed.
"""
from __future__ import annotations

import math
import numpy as np

ONE_THIRD = 1.0 / 3.0
PI = 3.141592653589793238
PI2 = 2.0 * PI
DEG2RAD = PI2 / 360.0
GRAV = 9.81


def _f4(x: float) -> float:
    """Value of a default-kind (single precision) Fortran literal once promoted to FP64."""
    return float(np.float32(x))


def fsign(a, b):
    """Fortran SIGN(a, b) with a processor that does not honour negative zero."""
    return np.where(np.asarray(b) >= 0.0, abs(a), -abs(a))


def _nxt(j):
    """J+1-INT((J+1)/4)*3 for a 1-based local vertex index J in 1..3."""
    return j + 1 - ((j + 1) // 4) * 3


def _nxt2(j):
    """J+2-INT((J+2)/4)*3."""
    return j + 2 - ((j + 2) // 4) * 3


class Grid:
    """FVCOM mesh arrays for one serial domain (MT == M, NT == N)."""

    def __init__(self):
        self.a = {}

    def __getitem__(self, k):
        return self.a[k]

    def __setitem__(self, k, v):
        self.a[k] = v


def build_grid(vx_in, vy_in, nv_cw, h_in, kb, obc_nodes=(), obc_types=(),
               cor_lat=None, sponge=(), horcon=0.2, z0b=0.001,
               rivers=None, river_location="node", static_ssh_adj=0.0, p_sigma=1.0,
               ghost_cells="GCN"):
    """Build every mesh array the mode-split step reads.

    vx_in, vy_in, h_in: node coordinates (m) and depth (m), length M (0-based input).
    nv_cw: (N, 3) 1-based node numbers of each cell in FVCOM's internal clockwise order
      (the order READ_COLDSTART_GRID produces after its node 2/3 swap,
      FVCOM_source/mod_input.F:3739-3741).
    kb: number of sigma levels; p_sigma: the power of GEOMETRIC sigma levels, 1.0 for
      UNIFORM (SIGMA_GEOMETRIC, FVCOM_source/mod_setup.F:848-877).
    obc_nodes/obc_types: 1-based open-boundary nodes and their TYPE_OBC (1..10).
    cor_lat: per-node latitude in degrees used for the Coriolis parameter.
    sponge: iterable of (node, radius, coefficient) as in the *_spg.dat file.
    horcon: HORIZONTAL_MIXING_COEFFICIENT (constant kind); z0b: BOTTOM_ROUGHNESS_LENGTHSCALE.
    rivers: list of dicts {"loc": node-or-cell (1-based), "dist": per-layer weights}.
    ghost_cells: FVCOM's solid-boundary treatment: "GCN" (no ghost cell, gradients of
      boundary cells are zero), "GCY1" (ghost cell at the foot of the perpendicular from
      the cell centre to the boundary edge) or "GCY2" (ghost cell at the edge midpoint)
      (SHAPE_COEF_GCN / SHAPE_COEF_GCY, shape_coef_gcy.F:29-655).
    """
    if ghost_cells not in ("GCN", "GCY1", "GCY2"):
        raise ValueError("ghost_cells must be GCN, GCY1 or GCY2")
    g = Grid()
    M = len(vx_in)
    N = len(nv_cw)
    g["M"], g["N"], g["KB"] = M, N, kb
    vx = np.zeros(M + 1)
    vy = np.zeros(M + 1)
    vx[1:] = np.asarray(vx_in, dtype=np.float64)
    vy[1:] = np.asarray(vy_in, dtype=np.float64)
    # SETUP_CENTER_COORDS (mod_setup.F:89-110): shift to the lower-left corner.
    vxmin = vx[1:].min()
    vymin = vy[1:].min()
    vx = vx - vxmin
    vy = vy - vymin
    vx[0] = 0.0
    vy[0] = 0.0
    nv = np.zeros((N + 1, 3), dtype=np.int32)
    nv[1:] = np.asarray(nv_cw, dtype=np.int32)
    h = np.zeros(M + 1)
    h[1:] = np.asarray(h_in, dtype=np.float64) + static_ssh_adj
    xc = np.zeros(N + 1)
    yc = np.zeros(N + 1)
    xc[1:] = ONE_THIRD * (vx[nv[1:, 0]] + vx[nv[1:, 1]] + vx[nv[1:, 2]])
    yc[1:] = ONE_THIRD * (vy[nv[1:, 0]] + vy[nv[1:, 1]] + vy[nv[1:, 2]])
    g["VX"], g["VY"], g["NV"], g["H"], g["XC"], g["YC"] = vx, vy, nv, h, xc, yc
    g["VXMIN"], g["VYMIN"] = vxmin, vymin

    _tge(g, list(obc_nodes))
    _cell_area(g)
    if ghost_cells == "GCN":
        _shape_coef(g)
    else:
        _shape_coef_gcy(g, ghost_cells)
    g["GHOST_CELLS"] = ghost_cells
    _edge_len(g)
    _depth_gradient(g)
    _obc_setup(g, list(obc_nodes), list(obc_types))
    _sigma(g, kb, p_sigma)
    g["P_SIGMA"] = float(p_sigma)
    _constants(g, cor_lat, sponge, horcon, z0b)
    _rivers(g, rivers or [], river_location)
    return g


# --------------------------------------------------------------------------------------
# TRIANGLE_GRID_EDGE (tge.F:29-866)
# --------------------------------------------------------------------------------------
def _tge(g, obc_nodes):
    M, N = g["M"], g["N"]
    nv = g["NV"]
    # Neighbour search via shared edges (tge.F:141-172).  NBE(I,1) is the cell across
    # the edge opposite local node 1 (nodes 2,3), NBE(I,2) across nodes 1,3, NBE(I,3)
    # across nodes 1,2.
    nbe = np.zeros((N + 1, 3), dtype=np.int32)
    edge_owner = {}
    pairs = ((1, 2), (0, 2), (0, 1))
    for i in range(1, N + 1):
        for j, (p, q) in enumerate(pairs):
            a, b = int(nv[i, p]), int(nv[i, q])
            key = (a, b) if a < b else (b, a)
            edge_owner.setdefault(key, []).append((i, j))
    for key, lst in edge_owner.items():
        if len(lst) == 2:
            (i1, j1), (i2, j2) = lst
            nbe[i1, j1] = i2
            nbe[i2, j2] = i1
        elif len(lst) > 2:
            raise ValueError("non-manifold edge %s" % (key,))
    if np.any(nbe[1:].sum(axis=1) == 0):
        raise ValueError("element with no neighbours (tge.F:190-197)")
    isbce = np.zeros(N + 1, dtype=np.int32)
    isonb = np.zeros(M + 1, dtype=np.int32)
    bnd = nbe[1:].min(axis=1) == 0
    isbce[1:][bnd] = 1
    for i in np.nonzero(bnd)[0] + 1:
        if nbe[i, 0] == 0:
            isonb[nv[i, 1]] = 1; isonb[nv[i, 2]] = 1
        if nbe[i, 1] == 0:
            isonb[nv[i, 0]] = 1; isonb[nv[i, 2]] = 1
        if nbe[i, 2] == 0:
            isonb[nv[i, 0]] = 1; isonb[nv[i, 1]] = 1

    # NBVE/NBVT in ascending cell order, then reordered around the node (tge.F:240-389).
    cells_of = [[] for _ in range(M + 1)]
    for i in range(1, N + 1):
        for jj in range(3):
            cells_of[nv[i, jj]].append(i)
    ntve = np.zeros(M + 1, dtype=np.int32)
    for i in range(1, M + 1):
        ntve[i] = len(cells_of[i])
    mx = int(ntve.max())
    nbve = np.zeros((M + 1, mx + 1), dtype=np.int32)
    nbvt = np.zeros((M + 1, mx + 1), dtype=np.int32)
    nbsn = np.zeros((M + 1, mx + 3), dtype=np.int32)
    ntsn = np.zeros(M + 1, dtype=np.int32)

    def local(c, node):
        if nv[c, 0] == node:
            return 1
        if nv[c, 1] == node:
            return 2
        return 3

    for i in range(1, M + 1):
        cl = cells_of[i]
        nt = len(cl)
        if isonb[i] == 0:
            ring = [cl[0]]
            tj = [local(cl[0], i)]
            for _ in range(1, nt + 1):
                ii, jj = ring[-1], tj[-1]
                nxt = int(nbe[ii, _nxt(jj) - 1])
                ring.append(nxt)
                tj.append(local(nxt, i))
            if ring[0] != ring[nt] or tj[0] != tj[nt]:
                raise ValueError("NBVE ring of node %d does not close (tge.F:317-327)" % i)
            for j in range(nt + 1):
                nbve[i, j] = ring[j]
                nbvt[i, j] = tj[j]
            for j in range(nt):
                nbsn[i, j] = nv[ring[j], _nxt(tj[j]) - 1]
            nbsn[i, nt] = nbsn[i, 0]
            ntsn[i] = nt + 1
        else:
            start = []
            for c in cl:
                jj = local(c, i)
                if nbe[c, _nxt2(jj) - 1] == 0:
                    start.append((c, jj))
            if len(start) != 1:
                raise ValueError("boundary node %d: %d starting cells (tge.F:352-355)" % (i, len(start)))
            ring = [start[0][0]]
            tj = [start[0][1]]
            for _ in range(1, nt):
                ii, jj = ring[-1], tj[-1]
                nxt = int(nbe[ii, _nxt(jj) - 1])
                ring.append(nxt)
                tj.append(local(nxt, i))
            for j in range(nt):
                nbve[i, j] = ring[j]
                nbvt[i, j] = tj[j]
            nbve[i, nt] = 0
            nbsn[i, 0] = i
            for j in range(nt):
                nbsn[i, j + 1] = nv[ring[j], _nxt(tj[j]) - 1]
            nbsn[i, nt + 1] = nv[ring[nt - 1], _nxt2(tj[nt - 1]) - 1]
            nbsn[i, nt + 2] = i
            ntsn[i] = nt + 3

    # Element edges (tge.F:435-524).
    iec, ienode = [], []
    iset = np.zeros((N + 1, 3), dtype=bool)
    for i in range(1, N + 1):
        for j in range(1, 4):
            if not iset[i, j - 1]:
                iney = int(nbe[i, j - 1])
                iset[i, j - 1] = True
                if iney:
                    for jn in range(3):
                        if nbe[iney, jn] == i:
                            iset[iney, jn] = True
                iec.append((i, iney))
                ienode.append((int(nv[i, _nxt(j) - 1]), int(nv[i, _nxt2(j) - 1])))
    ne = len(iec)
    IEC = np.zeros((ne + 1, 2), dtype=np.int32)
    IEN = np.zeros((ne + 1, 2), dtype=np.int32)
    IEC[1:] = np.array(iec, dtype=np.int32)
    IEN[1:] = np.array(ienode, dtype=np.int32)
    isbc = np.zeros(ne + 1, dtype=np.int32)
    isbc[1:] = ((IEC[1:, 0] == 0) | (IEC[1:, 1] == 0)).astype(np.int32)
    vx, vy, xc, yc = g["VX"], g["VY"], g["XC"], g["YC"]
    dltxc = np.zeros(ne + 1)
    dltyc = np.zeros(ne + 1)
    xijc = np.zeros(ne + 1)
    yijc = np.zeros(ne + 1)
    dltxc[1:] = vx[IEN[1:, 1]] - vx[IEN[1:, 0]]
    dltyc[1:] = vy[IEN[1:, 1]] - vy[IEN[1:, 0]]
    xijc[1:] = (vx[IEN[1:, 0]] + vx[IEN[1:, 1]]) / 2.0
    yijc[1:] = (vy[IEN[1:, 0]] + vy[IEN[1:, 1]]) / 2.0

    # Open-boundary node marker and boundary cell types (tge.F:540-588).
    for nd in obc_nodes:
        isonb[nd] = 2
    s = isonb[nv[1:, 0]] + isonb[nv[1:, 1]] + isonb[nv[1:, 2]]
    if np.any(s > 4):
        raise ValueError("boundary cell with two open sides (tge.F:566-580)")
    isbce[1:][s == 4] = 2
    for i in range(1, N + 1):
        if isbce[i] == 2:
            continue
        b0, b1, b2 = nbe[i]
        if (b0 + b1 + b2 == 0) or (b0 + b1 == 0) or (b1 + b2 == 0) or (b0 + b2 == 0):
            isbce[i] = 3

    # Control-volume half-edges (tge.F:611-769).  Serial domain: IEC(I,1) <= N always.
    niec, ntrg, dxe, dye, xije, yije = [], [], [], [], [], []
    for i in range(1, ne + 1):
        ia, ib = int(IEC[i, 0]), int(IEC[i, 1])
        n1, n2 = int(IEN[i, 0]), int(IEN[i, 1])
        if isbc[i] == 0:
            for (c, a, b) in ((ia, n1, n2), (ib, n2, n1)):
                niec.append((a, b)); ntrg.append(c)
                xije.append((xc[c], xijc[i])); yije.append((yc[c], yijc[i]))
                dxe.append(xijc[i] - xc[c]); dye.append(yijc[i] - yc[c])
        else:
            if ia == 0:
                raise ValueError("IEC(I,1)==0 (tge.F:711-714)")
            niec.append((n1, n2)); ntrg.append(ia)
            xije.append((xc[ia], xijc[i])); yije.append((yc[ia], yijc[i]))
            dxe.append(xijc[i] - xc[ia]); dye.append(yijc[i] - yc[ia])
    ncv = len(ntrg)
    if ncv != 3 * N:
        raise ValueError("NCV != 3N (tge.F:762-765)")
    NIEC = np.zeros((ncv + 1, 2), dtype=np.int32)
    NIEC[1:] = np.array(niec, dtype=np.int32)
    NTRG = np.zeros(ncv + 1, dtype=np.int32)
    NTRG[1:] = ntrg
    DLTXE = np.zeros(ncv + 1); DLTXE[1:] = dxe
    DLTYE = np.zeros(ncv + 1); DLTYE[1:] = dye
    XIJE = np.zeros((ncv + 1, 2)); XIJE[1:] = xije
    YIJE = np.zeros((ncv + 1, 2)); YIJE[1:] = yije
    epor = np.ones(N + 1)
    epor[1:][isbce[1:] == 2] = 0.0

    g.a.update(NBE=nbe, ISBCE=isbce, ISONB=isonb, NTVE=ntve, NBVE=nbve, NBVT=nbvt,
               NTSN=ntsn, NBSN=nbsn, NE=ne, IEC=IEC, IENODE=IEN, ISBC=isbc,
               DLTXC=dltxc, DLTYC=dltyc, XIJC=xijc, YIJC=yijc, NCV=ncv, NCV_I=ncv,
               NIEC=NIEC, NTRG=NTRG, DLTXE=DLTXE, DLTYE=DLTYE, XIJE=XIJE, YIJE=YIJE,
               EPOR=epor)


# --------------------------------------------------------------------------------------
# CELL_AREA (cell_area.F:40-352)
# --------------------------------------------------------------------------------------
def _cell_area(g):
    M, N = g["M"], g["N"]
    vx, vy, nv, xc, yc = g["VX"], g["VY"], g["NV"], g["XC"], g["YC"]
    art = np.zeros(N + 1)
    n1, n2, n3 = nv[1:, 0], nv[1:, 1], nv[1:, 2]
    art[1:] = ((vx[n2] - vx[n1]) * (vy[n3] - vy[n1]) - (vx[n3] - vx[n1]) * (vy[n2] - vy[n1]))
    art = np.abs(0.5 * art)
    art1 = np.zeros(M + 1)
    ntve, nbve, nbvt, isonb = g["NTVE"], g["NBVE"], g["NBVT"], g["ISONB"]
    for i in range(1, M + 1):
        nt = int(ntve[i])
        xx, yy = [], []
        for j in range(nt):
            ii = nbve[i, j]
            j1 = int(nbvt[i, j])
            j2 = _nxt(j1)
            xx.append((vx[nv[ii, j1 - 1]] + vx[nv[ii, j2 - 1]]) * 0.5 - vx[i])
            yy.append((vy[nv[ii, j1 - 1]] + vy[nv[ii, j2 - 1]]) * 0.5 - vy[i])
            xx.append(xc[ii] - vx[i])
            yy.append(yc[ii] - vy[i])
        if isonb[i] == 0:
            xx.append(xx[0]); yy.append(yy[0])
            cnt = 2 * nt
        else:
            ii = nbve[i, nt - 1]
            j1 = int(nbvt[i, nt - 1])
            j2 = _nxt2(j1)
            xx.append((vx[nv[ii, j1 - 1]] + vx[nv[ii, j2 - 1]]) * 0.5 - vx[i])
            yy.append((vy[nv[ii, j1 - 1]] + vy[nv[ii, j2 - 1]]) * 0.5 - vy[i])
            xx.append(vx[i] - vx[i]); yy.append(vy[i] - vy[i])
            xx.append(xx[0]); yy.append(yy[0])
            cnt = 2 * nt + 2
        acc = 0.0
        for j in range(cnt):
            acc = acc + 0.5 * (xx[j + 1] * yy[j] - xx[j] * yy[j + 1])
        art1[i] = abs(acc)
    art2 = np.zeros(M + 1)
    for i in range(1, M + 1):
        s = 0.0
        for j in range(int(ntve[i])):
            s = s + art[nbve[i, j]]
        art2[i] = s
    art[0] = art[1]
    art1[0] = art1[1]
    g.a.update(ART=art, ART1=art1, ART2=art2)


# --------------------------------------------------------------------------------------
# SHAPE_COEF_GCN (shape_coef_gcn.F:29-368)
# --------------------------------------------------------------------------------------
def _shape_coef(g):
    M, N = g["M"], g["N"]
    vx, vy, nv, xc, yc = g["VX"], g["VY"], g["NV"], g["XC"], g["YC"]
    nbe, isbce, art = g["NBE"], g["ISBCE"], g["ART"]
    a1u = np.zeros((N + 1, 4))
    a2u = np.zeros((N + 1, 4))
    awx = np.zeros((N + 1, 3))
    awy = np.zeros((N + 1, 3))
    aw0 = np.zeros((N + 1, 3))
    alpha = np.zeros(N + 1)
    for i in range(1, N + 1):
        if isbce[i] == 0:
            y1 = yc[nbe[i, 0]] - yc[i]; y2 = yc[nbe[i, 1]] - yc[i]; y3 = yc[nbe[i, 2]] - yc[i]
            x1 = xc[nbe[i, 0]] - xc[i]; x2 = xc[nbe[i, 1]] - xc[i]; x3 = xc[nbe[i, 2]] - xc[i]
            x1 = x1 / 1000.0; x2 = x2 / 1000.0; x3 = x3 / 1000.0
            y1 = y1 / 1000.0; y2 = y2 / 1000.0; y3 = y3 / 1000.0
            delt = (x1 * y2 - x2 * y1) ** 2 + (x1 * y3 - x3 * y1) ** 2 + (x2 * y3 - x3 * y2) ** 2
            delt = delt * 1000.0
            sxy = x1 * y1 + x2 * y2 + x3 * y3
            syy = y1 ** 2 + y2 ** 2 + y3 ** 2
            sxx = x1 ** 2 + x2 ** 2 + x3 ** 2
            a1u[i, 0] = ((y1 + y2 + y3) * sxy - (x1 + x2 + x3) * syy) / delt
            a1u[i, 1] = (syy * x1 - sxy * y1) / delt
            a1u[i, 2] = (syy * x2 - sxy * y2) / delt
            a1u[i, 3] = (syy * x3 - sxy * y3) / delt
            a2u[i, 0] = ((x1 + x2 + x3) * sxy - (y1 + y2 + y3) * sxx) / delt
            a2u[i, 1] = (sxx * y1 - sxy * x1) / delt
            a2u[i, 2] = (sxx * y2 - sxy * x2) / delt
            a2u[i, 3] = (sxx * y3 - sxy * x3) / delt
        x1 = vx[nv[i, 0]] - xc[i]; x2 = vx[nv[i, 1]] - xc[i]; x3 = vx[nv[i, 2]] - xc[i]
        y1 = vy[nv[i, 0]] - yc[i]; y2 = vy[nv[i, 1]] - yc[i]; y3 = vy[nv[i, 2]] - yc[i]
        ai = (y2 - y3, y3 - y1, y1 - y2)
        bi = (x3 - x2, x1 - x3, x2 - x1)
        ci = (x2 * y3 - x3 * y2, x3 * y1 - x1 * y3, x1 * y2 - x2 * y1)
        for j in range(3):
            aw0[i, j] = -ci[j] / 2.0 / art[i]
            awx[i, j] = -ai[j] / 2.0 / art[i]
            awy[i, j] = -bi[j] / 2.0 / art[i]
    pi7 = 3.1415926
    for i in range(1, N + 1):
        if isbce[i] == 1:
            jj = 0
            for j in range(1, 4):
                if nbe[i, j - 1] == 0:
                    jj = j
            j1, j2 = _nxt(jj), _nxt2(jj)
            deltx = vx[nv[i, j1 - 1]] - vx[nv[i, j2 - 1]]
            delty = vy[nv[i, j1 - 1]] - vy[nv[i, j2 - 1]]
            alpha[i] = math.atan2(delty, deltx)
            alpha[i] = alpha[i] - pi7 / 2.0
    ang1 = 359.9 / 180.0 * pi7
    ang2 = -0.1 / 180.0 * pi7
    ntve, nbve, isonb = g["NTVE"], g["NBVE"], g["ISONB"]
    for i in range(1, M + 1):
        nt = int(ntve[i])
        if isonb[i] == 1 and nt > 2:
            angle = alpha[nbve[i, nt - 1]] - alpha[nbve[i, 0]]
            if angle > ang1:
                angle = 100000.0
            elif angle > pi7:
                angle = angle - 2.0 * pi7
            elif angle < -pi7:
                angle = angle + 2.0 * pi7
            elif angle < ang2:
                angle = 100000.0
            for j in range(2, nt):
                ii = nbve[i, j - 1]
                if isbce[ii] != 1:
                    alpha[ii] = alpha[nbve[i, 0]] + angle / _f4(nt - 1) * _f4(j - 1)
    g.a.update(A1U=a1u, A2U=a2u, AWX=awx, AWY=awy, AW0=aw0, ALPHA=alpha)


def _foot(xa, ya, xb, yb, xc, yc):
    """Foot of the perpendicular from (xc, yc) onto the line through (xa, ya) and (xb, yb),
    in the reference's line-intersection form (shape_coef_gcy.F:117-125)."""
    deltx = xa - xb
    delty = ya - yb
    aa1 = -delty
    bb1 = deltx
    cc1 = -aa1 * xa - bb1 * ya
    aa2 = bb1
    bb2 = -aa1
    cc2 = -aa2 * xc - bb2 * yc
    x = -(cc1 * bb2 - cc2 * bb1) / (aa1 * bb2 - aa2 * bb1)
    y = -(cc1 * aa2 - cc2 * aa1) / (bb1 * aa2 - bb2 * aa1)
    return x, y


def _shape_coef_gcy(g, variant):
    """SHAPE_COEF_GCY (shape_coef_gcy.F:29-655): the least-squares weights of every cell,
    boundary cells included, with a ghost point in place of each missing neighbour: on a
    solid edge the foot of the perpendicular from the centre (GCY1) or the edge midpoint
    (GCY2), on an open-boundary edge twice the centre-to-foot offset.  The formulas are
    the reference's, including its first A2U weight, which multiplies (X1+X2+X3) by the
    sum of X squared where the GCN weights use the sum of X*Y."""
    M, N = g["M"], g["N"]
    vx, vy, nv, xc, yc = g["VX"], g["VY"], g["NV"], g["XC"], g["YC"]
    nbe, isbce, art = g["NBE"], g["ISBCE"], g["ART"]
    a1u = np.zeros((N + 1, 4))
    a2u = np.zeros((N + 1, 4))
    awx = np.zeros((N + 1, 3))
    awy = np.zeros((N + 1, 3))
    aw0 = np.zeros((N + 1, 3))
    alpha = np.zeros(N + 1)
    pi7 = 3.1415926

    def node(i, j):  # node j (1-based) of cell i
        return nv[i, j - 1]

    def nbr(i, j):
        return nbe[i, j - 1]

    for i in range(1, N + 1):
        b = isbce[i]
        pts = [None, None, None]  # (x, y) offsets of the three neighbours or ghosts
        if b == 0:
            for j in range(1, 4):
                pts[j - 1] = (xc[nbr(i, j)] - xc[i], yc[nbr(i, j)] - yc[i])
        elif b in (1, 2):
            jj = 0
            for j in range(1, 4):
                if nbr(i, j) == 0:
                    jj = j
            j1, j2 = _nxt(jj), _nxt2(jj)
            na, nb_ = node(i, j1), node(i, j2)
            if b == 2 or variant == "GCY1":
                deltx = vx[na] - vx[nb_]
                delty = vy[na] - vy[nb_]
                alpha[i] = math.atan2(delty, deltx) - pi7 / 2.0
                xt, yt = _foot(vx[na], vy[na], vx[nb_], vy[nb_], xc[i], yc[i])
            else:
                xt, yt = (vx[na] + vx[nb_]) / 2.0, (vy[na] + vy[nb_]) / 2.0
            ghost = (xt - xc[i], yt - yc[i]) if b == 1 else ((xt - xc[i]) * 2.0, (yt - yc[i]) * 2.0)
            for j in range(1, 4):
                pts[j - 1] = ghost if j == jj else (xc[nbr(i, j)] - xc[i], yc[nbr(i, j)] - yc[i])
        elif b == 3:
            jj = 0
            for j in range(1, 4):
                if nbr(i, j) != 0:
                    jj = j
            j1, j2 = _nxt(jj), _nxt2(jj)
            n0, na, nb_ = node(i, jj), node(i, j1), node(i, j2)
            if variant == "GCY1":
                xt1, yt1 = _foot(vx[n0], vy[n0], vx[nb_], vy[nb_], xc[i], yc[i])
                xt2, yt2 = _foot(vx[n0], vy[n0], vx[na], vy[na], xc[i], yc[i])
            else:
                xt1, yt1 = (vx[n0] + vx[nb_]) / 2.0, (vy[n0] + vy[nb_]) / 2.0
                xt2, yt2 = (vx[n0] + vx[na]) / 2.0, (vy[n0] + vy[na]) / 2.0
            # slot j1 lies opposite node j1: the edge (jj, j2), ghost 1; slot j2: ghost 2
            pts[jj - 1] = (xc[nbr(i, jj)] - xc[i], yc[nbr(i, jj)] - yc[i])
            pts[j1 - 1] = (xt1 - xc[i], yt1 - yc[i])
            pts[j2 - 1] = (xt2 - xc[i], yt2 - yc[i])
        (x1, y1), (x2, y2), (x3, y3) = pts
        x1 = x1 / 1000.0; x2 = x2 / 1000.0; x3 = x3 / 1000.0
        y1 = y1 / 1000.0; y2 = y2 / 1000.0; y3 = y3 / 1000.0
        delt = (x1 * y2 - x2 * y1) ** 2 + (x1 * y3 - x3 * y1) ** 2 + (x2 * y3 - x3 * y2) ** 2
        delt = delt * 1000.0
        sxy = x1 * y1 + x2 * y2 + x3 * y3
        syy = y1 ** 2 + y2 ** 2 + y3 ** 2
        sxx = x1 ** 2 + x2 ** 2 + x3 ** 2
        sxx_b = x1 * x1 + x2 * x2 + x3 * x3
        a1u[i, 0] = ((y1 + y2 + y3) * sxy - (x1 + x2 + x3) * syy) / delt
        a1u[i, 1] = (syy * x1 - sxy * y1) / delt
        a1u[i, 2] = (syy * x2 - sxy * y2) / delt
        a1u[i, 3] = (syy * x3 - sxy * y3) / delt
        a2u[i, 0] = ((x1 + x2 + x3) * sxx_b - (y1 + y2 + y3) * sxx) / delt
        a2u[i, 1] = (sxx * y1 - sxy * x1) / delt
        a2u[i, 2] = (sxx * y2 - sxy * x2) / delt
        a2u[i, 3] = (sxx * y3 - sxy * x3) / delt
        x1 = vx[nv[i, 0]] - xc[i]; x2 = vx[nv[i, 1]] - xc[i]; x3 = vx[nv[i, 2]] - xc[i]
        y1 = vy[nv[i, 0]] - yc[i]; y2 = vy[nv[i, 1]] - yc[i]; y3 = vy[nv[i, 2]] - yc[i]
        ai = (y2 - y3, y3 - y1, y1 - y2)
        bi = (x3 - x2, x1 - x3, x2 - x1)
        ci = (x2 * y3 - x3 * y2, x3 * y1 - x1 * y3, x1 * y2 - x2 * y1)
        for j in range(3):
            aw0[i, j] = -ci[j] / 2.0 / art[i]
            awx[i, j] = -ai[j] / 2.0 / art[i]
            awy[i, j] = -bi[j] / 2.0 / art[i]
    ang1 = 359.9 / 180.0 * pi7
    ang2 = -0.1 / 180.0 * pi7
    ntve, nbve, isonb = g["NTVE"], g["NBVE"], g["ISONB"]
    for i in range(1, M + 1):
        nt = int(ntve[i])
        if isonb[i] == 1 and nt > 2:
            angle = alpha[nbve[i, nt - 1]] - alpha[nbve[i, 0]]
            if angle > ang1:
                angle = 100000.0
            elif angle > pi7:
                angle = angle - 2.0 * pi7
            elif angle < -pi7:
                angle = angle + 2.0 * pi7
            elif angle < ang2:
                angle = 100000.0
            for j in range(2, nt):
                ii = nbve[i, j - 1]
                if isbce[ii] != 1:
                    alpha[ii] = alpha[nbve[i, 0]] + angle / _f4(nt - 1) * _f4(j - 1)
    g.a.update(A1U=a1u, A2U=a2u, AWX=awx, AWY=awy, AW0=aw0, ALPHA=alpha)


# --------------------------------------------------------------------------------------
# EDGE_LEN (edge_len.F:29-241)
# --------------------------------------------------------------------------------------
def _edge_len(g):
    M = g["M"]
    vx, vy, nv = g["VX"], g["VY"], g["NV"]
    niec, xije, yije, ncv_i = g["NIEC"], g["XIJE"], g["YIJE"], g["NCV_I"]
    dxn = np.zeros((ncv_i + 1, 2))
    dyn = np.zeros((ncv_i + 1, 2))
    xi = 0.5 * (xije[1:, 0] + xije[1:, 1])
    yi = 0.5 * (yije[1:, 0] + yije[1:, 1])
    dxn[1:, 0] = xi - vx[niec[1:, 0]]
    dyn[1:, 0] = yi - vy[niec[1:, 0]]
    dxn[1:, 1] = xi - vx[niec[1:, 1]]
    dyn[1:, 1] = yi - vy[niec[1:, 1]]
    ntsn, nbsn, ntve, nbve, nbvt = g["NTSN"], g["NBSN"], g["NTVE"], g["NBVE"], g["NBVT"]
    if ntsn.max() > 13 or ntve.max() > 13:
        raise ValueError("more than 12 neighbours around a node (edge_len.F:98-170)")
    W = 12
    dxtrie = np.zeros((M + 1, W))
    dytrie = np.zeros((M + 1, W))
    dxecec = np.zeros((M + 1, W))
    dyecec = np.zeros((M + 1, W))
    dxnec = np.zeros((M + 1, W))
    dynec = np.zeros((M + 1, W))
    for i in range(1, M + 1):
        for j in range(int(ntsn[i]) - 1):
            i1, i2 = nbsn[i, j], nbsn[i, j + 1]
            dytrie[i, j] = vy[i1] - vy[i2]
            dxtrie[i, j] = vx[i2] - vx[i1]
        for j in range(int(ntve[i])):
            i1 = nbve[i, j]
            jt = int(nbvt[i, j])
            j1, j2 = _nxt(jt), _nxt2(jt)
            x11 = 0.5 * (vx[i] + vx[nv[i1, j1 - 1]])
            y11 = 0.5 * (vy[i] + vy[nv[i1, j1 - 1]])
            x33 = 0.5 * (vx[i] + vx[nv[i1, j2 - 1]])
            y33 = 0.5 * (vy[i] + vy[nv[i1, j2 - 1]])
            dyecec[i, j] = y11 - y33
            dxecec[i, j] = x33 - x11
            dynec[i, j] = vy[i] - y11
            dxnec[i, j] = x11 - vx[i]
    g.a.update(DLTXNCVE=dxn, DLTYNCVE=dyn, DLTXTRIE=dxtrie, DLTYTRIE=dytrie,
               DLTXECEC=dxecec, DLTYECEC=dyecec, DLTXNEC=dxnec, DLTYNEC=dynec)


# --------------------------------------------------------------------------------------
# DEPTH_GRADIENT (depth_grad.F:33-90)
# --------------------------------------------------------------------------------------
def _depth_gradient(g):
    M = g["M"]
    vx, vy, h, art2 = g["VX"], g["VY"], g["H"], g["ART2"]
    ntsn, nbsn = g["NTSN"], g["NBSN"]
    sita = np.zeros(M + 1)
    phpn = np.zeros(M + 1)
    for i in range(1, M + 1):
        px = 0.0
        py = 0.0
        for j in range(int(ntsn[i]) - 1):
            i1, i2 = nbsn[i, j], nbsn[i, j + 1]
            f1 = 0.50 * (h[i1] + h[i2])
            px = px + f1 * (vy[i1] - vy[i2])
            py = py + f1 * (vx[i2] - vx[i1])
        px = px / art2[i]
        py = py / art2[i]
        if px == 0.0 and py == 0.0:
            sita[i] = 0.0
            phpn[i] = 0.0
        else:
            sita[i] = math.atan2(py, px)
            phpn[i] = math.sqrt(py * py + px * px)
    g.a.update(SITA_GD=sita, PHPN=phpn)


# --------------------------------------------------------------------------------------
# SETUP_OBC (mod_obcs.F:868-1173) and SEPARATE_OBC (mod_obcs.F:803-861)
# --------------------------------------------------------------------------------------
def _obc_setup(g, obc_nodes, obc_types):
    M, N = g["M"], g["N"]
    n_obc = len(obc_nodes)
    g["IOBCN"] = n_obc
    vx, vy, nv, xc, yc = g["VX"], g["VY"], g["NV"], g["XC"], g["YC"]
    isonb, ntsn, nbsn, ntve, nbve = g["ISONB"], g["NTSN"], g["NBSN"], g["NTVE"], g["NBVE"]
    I_OBC_N = np.zeros(n_obc + 1, dtype=np.int32)
    TYPE_OBC = np.zeros(n_obc + 1, dtype=np.int32)
    I_OBC_N[1:] = obc_nodes
    TYPE_OBC[1:] = obc_types
    iucp = np.ones(N + 1)
    nadjn = np.zeros(n_obc + 1, dtype=np.int32)
    adjn = np.zeros((n_obc + 1, 2), dtype=np.int32)
    for i in range(1, n_obc + 1):
        inode = I_OBC_N[i]
        for j in range(int(ntsn[inode]) - 1):
            jn = nbsn[inode, j]
            if isonb[jn] == 2 and inode != jn:
                nadjn[i] += 1
                if nadjn[i] > 2:
                    raise ValueError("open-boundary node with more than two open neighbours")
                adjn[i, nadjn[i] - 1] = jn
        if nadjn[i] == 0:
            raise ValueError("no adjacent open-boundary node for %d (mod_obcs.F:912-918)" % i)
    nadjc = np.zeros(n_obc + 1, dtype=np.int32)
    adjc = np.zeros((n_obc + 1, 2), dtype=np.int32)
    nx = np.zeros(n_obc + 1)
    ny = np.zeros(n_obc + 1)
    for i in range(1, n_obc + 1):
        i1 = I_OBC_N[i]
        for which in range(int(min(nadjn[i], 2))):
            i2 = adjn[i, which]
            for j in range(int(ntve[i1])):
                ic = nbve[i1, j]
                if i2 in (nv[ic, 0], nv[ic, 1], nv[ic, 2]):
                    dxn = vx[i2] - vx[i1]; dyn = vy[i2] - vy[i1]
                    dxc = xc[ic] - vx[i1]; dyc = yc[ic] - vy[i1]
                    cross = 1.0 if (dxc * dyn - dyc * dxn) >= 0.0 else -1.0
                    if which == 0:
                        nx[i] = cross * dyn / math.sqrt(dxn ** 2 + dyn ** 2)
                        ny[i] = -cross * dxn / math.sqrt(dxn ** 2 + dyn ** 2)
                    else:
                        tx = nx[i] + cross * dyn / math.sqrt(dxn ** 2 + dyn ** 2)
                        ty = ny[i] - cross * dxn / math.sqrt(dxn ** 2 + dyn ** 2)
                        nx[i] = tx / math.sqrt(tx ** 2 + ty ** 2)
                        ny[i] = ty / math.sqrt(tx ** 2 + ty ** 2)
                    nadjc[i] += 1
                    adjc[i, nadjc[i] - 1] = ic
                    if TYPE_OBC[i] % 2 == 1:
                        iucp[ic] = 0.0
    fluxf = np.zeros((n_obc + 1, 2))
    for i in range(1, n_obc + 1):
        if nadjn[i] == 1:
            fluxf[i, 0] = 1.0
            fluxf[i, 1] = 0.0
        else:
            n1, n2, n3 = I_OBC_N[i], adjn[i, 0], adjn[i, 1]
            e1 = math.sqrt((vx[n1] - vx[n2]) ** 2 + (vy[n1] - vy[n2]) ** 2)
            e2 = math.sqrt((vx[n1] - vx[n3]) ** 2 + (vy[n1] - vy[n3]) ** 2)
            fluxf[i, 0] = e1 / (e1 + e2)
            fluxf[i, 1] = e2 / (e1 + e2)
    next_obc = np.zeros(n_obc + 1, dtype=np.int32)
    for i in range(1, n_obc + 1):
        dotmax = -1.0
        inode = I_OBC_N[i]
        for j in range(int(ntsn[inode]) - 1):
            jn = nbsn[inode, j]
            if isonb[jn] != 2 and inode != jn:
                dx = vx[jn] - vx[inode]; dy = vy[jn] - vy[inode]
                ddx = dx / math.sqrt(dx ** 2 + dy ** 2)
                ddy = dy / math.sqrt(dx ** 2 + dy ** 2)
                dot = ddx * nx[i] + ddy * ny[i]
                if dot > dotmax:
                    dotmax = dot
                    next_obc[i] = jn
        if next_obc[i] == 0:
            raise ValueError("open-boundary node %d has no interior neighbour" % inode)
    dltn = np.zeros(n_obc + 1)
    for i in range(1, n_obc + 1):
        i1, i2 = I_OBC_N[i], next_obc[i]
        dltn[i] = abs((vx[i2] - vx[i1]) * nx[i] + (vy[i2] - vy[i1]) * ny[i])
    # SEPARATE_OBC: list of each OBC type group (mod_obcs.F:832-858).
    groups = [[] for _ in range(5)]
    for i in range(1, n_obc + 1):
        t = int(TYPE_OBC[i])
        groups[(t - 1) // 2].append(i)
    if any(len(gr) for gr in groups[2:]):
        raise ValueError("only open-boundary types 1-4 (specified or clamped elevation) are supported")
    g.a.update(I_OBC_N=I_OBC_N, TYPE_OBC=TYPE_OBC, IUCP=iucp, NADJC_OBC=nadjc, ADJC_OBC=adjc,
               FLUXF_OBC=fluxf, NEXT_OBC=next_obc, DLTN_OBC=dltn, NXOBC=nx, NYOBC=ny,
               OBC_LST1=np.array(groups[0], dtype=np.int32),
               OBC_LST2=np.array(groups[1], dtype=np.int32))


# --------------------------------------------------------------------------------------
# Sigma levels: SIGMA_GEOMETRIC with P_SIGMA = 1 (uniform), SETUP_SIGMA_DERIVATIVES and
# the cell versions of SET_WATER_DEPTH (mod_setup.F:848-877, 1009-1047;
# mod_startup.F:1460-1491).
# --------------------------------------------------------------------------------------
def _sigma(g, kb, p_sigma=1.0):
    M, N = g["M"], g["N"]
    nv = g["NV"]
    # ZTMP(K) = -((K-1)/FLOAT(KB-1))**P_SIGMA: the quotient is a default-real (single
    # precision) division because FLOAT returns default real; **1.0 leaves it unchanged.
    if p_sigma == 1.0:
        ztmp = np.array([-float(np.float32(k - 1) / np.float32(kb - 1)) for k in range(1, kb + 1)])
    else:
        # Geometric levels symmetric about mid-depth (mod_setup.F:854-860): the same
        # single-precision quotient, raised to the FP64 power and halved.
        if kb % 2 == 0:
            raise ValueError("GEOMETRIC sigma with a power other than 1 needs an odd KB (mod_setup.F:805)")
        half = (kb + 1) // 2
        p = float(p_sigma)
        ztmp = np.zeros(kb)
        for k in range(1, half + 1):
            ztmp[k - 1] = -(float(np.float32(k - 1) / np.float32(half - 1)) ** p) / 2.0
        for k in range(half + 1, kb + 1):
            ztmp[k - 1] = (float(np.float32(kb - k) / np.float32(half - 1)) ** p) / 2.0 - 1.0
    z = np.zeros((M + 1, kb))
    z[1:, :] = ztmp[None, :]
    z1 = np.zeros((N + 1, kb))
    z1[1:, :] = (z[nv[1:, 0], :] + z[nv[1:, 1], :] + z[nv[1:, 2], :]) / 3.0

    def deriv(zz_in):
        L = zz_in.shape[0]
        dz = np.zeros((L, kb))
        zz = np.zeros((L, kb))
        dzz = np.zeros((L, kb))
        dz[1:, :kb - 1] = zz_in[1:, :kb - 1] - zz_in[1:, 1:kb]
        zz[1:, :kb - 1] = 0.5 * (zz_in[1:, :kb - 1] + zz_in[1:, 1:kb])
        zz[1:, kb - 1] = 2.0 * zz[1:, kb - 2] - zz[1:, kb - 3]
        dzz[1:, :kb - 2] = zz[1:, :kb - 2] - zz[1:, 1:kb - 1]
        dzz[:, kb - 2] = 0.0
        dz[:, kb - 1] = 0.0
        return dz, zz, dzz

    dz, zz, dzz = deriv(z)
    dz1, zz1, dzz1 = deriv(z1)
    h = g["H"]
    h1 = np.zeros(N + 1)
    h1[1:] = (h[nv[1:, 0]] + h[nv[1:, 1]] + h[nv[1:, 2]]) / 3.0
    g.a.update(Z=z, ZZ=zz, DZ=dz, DZZ=dzz, Z1=z1, ZZ1=zz1, DZ1=dz1, DZZ1=dzz1, H1=h1)


# --------------------------------------------------------------------------------------
# Coriolis, gravity, sponge, mixing and roughness coefficients
# (mod_setup.F:314-516).
# --------------------------------------------------------------------------------------
def _constants(g, cor_lat, sponge, horcon, z0b):
    M, N = g["M"], g["N"]
    nv = g["NV"]
    lat = np.zeros(M + 1)
    if cor_lat is not None:
        lat[1:] = np.broadcast_to(np.asarray(cor_lat, dtype=np.float64), (M,))
    cor = np.zeros(N + 1)
    cor[1:] = ONE_THIRD * (lat[nv[1:, 0]] + lat[nv[1:, 1]] + lat[nv[1:, 2]])
    cor = 2.0 * 7.292e-5 * np.sin(cor * DEG2RAD)
    cor = np.where((cor < 1.0e-5) & (cor > 0.0), 1.0e-5, cor)
    cor = np.where((cor > -1.0e-5) & (cor < 0.0), -1.0e-5, cor)
    grav_n = np.full(M + 1, GRAV)
    grav_e = np.full(N + 1, GRAV)
    sp = np.zeros(N + 1)
    vx, vy, xc, yc = g["VX"], g["VY"], g["XC"], g["YC"]
    for (node, r, c) in sponge:
        xs, ys = vx[node], vy[node]
        d = np.sqrt((xc[1:] - xs) ** 2 + (yc[1:] - ys) ** 2) / r
        cs = c * (1.0 - d)
        sp[1:] = np.where(d <= 1.0, np.maximum(cs, sp[1:]), sp[1:])
    cc_hvc = np.full(N + 1, float(horcon)); cc_hvc[0] = 0.0
    nn_hvc = np.full(M + 1, float(horcon)); nn_hvc[0] = 0.0
    cc_z0b = np.full(N + 1, float(z0b)); cc_z0b[0] = 0.0
    g.a.update(COR=cor, GRAV_N=grav_n, GRAV_E=grav_e, CC_SPONGE=sp, CC_HVC=cc_hvc,
               NN_HVC=nn_hvc, CC_Z0B=cc_z0b, LAT=lat, SPONGE_LIST=[tuple(x) for x in sponge])


# --------------------------------------------------------------------------------------
# SET_RIVER_BNDRY_METRICS (mod_force.F:3447-3581)
# --------------------------------------------------------------------------------------
def _rivers(g, rivers, location):
    nq = len(rivers)
    kbm1 = g["KB"] - 1
    g["NUMQBC"] = nq
    g["RIVER_LOC"] = location
    vx, vy, h, nv, nbe = g["VX"], g["VY"], g["H"], g["NV"], g["NBE"]
    isonb, isbce, ntsn, nbsn, art1 = g["ISONB"], g["ISBCE"], g["NTSN"], g["NBSN"], g["ART1"]
    inodeq = np.zeros(nq + 1, dtype=np.int32)
    icellq = np.zeros(nq + 1, dtype=np.int32)
    n_icellq = np.zeros((nq + 1, 2), dtype=np.int32)
    rdisq = np.zeros((nq + 1, 2))
    qarea = np.zeros(nq + 1)
    angleq = np.zeros(nq + 1)
    vqdist = np.zeros((nq + 1, kbm1))
    for q, r in enumerate(rivers, start=1):
        vqdist[q, :] = np.asarray(r["dist"], dtype=np.float64)
        if location == "node":
            j = int(r["loc"])
            if isonb[j] != 1:
                raise ValueError("river node %d is not a solid-boundary node (mod_force.F:3471)" % j)
            inodeq[q] = j
            i1, i2, i3 = nbsn[j, 1], nbsn[j, 0], nbsn[j, ntsn[j] - 2]
            dy12 = vy[i1] - vy[i2]; dy32 = vy[i3] - vy[i2]
            dx12 = vx[i1] - vx[i2]; dx32 = vx[i3] - vx[i2]
            a1 = math.atan2(dy12, dx12)
            a2 = math.atan2(dy32, dx32)
            if a1 < a2:
                a1 = a1 + 2.0 * 3.1415927
            dxy = math.sqrt(dx12 ** 2 + dy12 ** 2) + math.sqrt(dx32 ** 2 + dy32 ** 2)
            qarea[q] = 0.5 * dxy * h[j]
            angleq[q] = (a1 - a2) / 2.0 + a2
        elif location == "edge":
            ii = int(r["loc"])
            if isbce[ii] != 1:
                raise ValueError("river cell %d is not a solid-boundary cell (mod_force.F:3519)" % ii)
            zeros = [j for j in range(1, 4) if nbe[ii, j - 1] == 0]
            if len(zeros) != 1:
                raise ValueError("river cell %d has the wrong number of solid sides" % ii)
            jt = zeros[0]
            j1, j2 = _nxt(jt), _nxt2(jt)
            i1, i2 = nv[ii, j1 - 1], nv[ii, j2 - 1]
            icellq[q] = ii
            n_icellq[q] = (i1, i2)
            htmp = 0.5 * (h[i1] + h[i2])
            dy12 = vy[i1] - vy[i2]
            dx12 = vx[i1] - vx[i2]
            a1 = math.atan2(dy12, dx12)
            qarea[q] = math.sqrt(dx12 ** 2 + dy12 ** 2) * htmp
            # 3.1415927/2.0 is a default-real (single precision) expression.
            angleq[q] = a1 + float(np.float32(3.1415927) / np.float32(2.0))
            areatmp = art1[i1] + art1[i2]
            rdisq[q, 0] = art1[i1] / areatmp
            rdisq[q, 1] = art1[i2] / areatmp
        else:
            raise ValueError("RIVER_INFLOW_LOCATION must be 'node' or 'edge'")
    g.a.update(INODEQ=inodeq, ICELLQ=icellq, N_ICELLQ=n_icellq, RDISQ=rdisq, QAREA=qarea,
               ANGLEQ=angleq, VQDIST=vqdist)
