"""Mesh-metric invariants of the FVCOM set-up stand-in (tge.F, cell_area.F, edge_len.F)."""
import numpy as np
import pytest

from myfvcomcode_b200 import cases


@pytest.mark.parametrize("nx,ny", [(4, 2), (10, 3)])
def test_channel_counts(nx, ny):
    c = cases.estuary_channel(nx=nx, ny=ny, kb=4, lx=1000.0 * nx, ly=1000.0 * ny)
    g = c["grid"]
    M, N = g["M"], g["N"]
    assert M == (nx + 1) * (ny + 1) and N == 2 * nx * ny
    assert g["NCV"] == 3 * N                       # tge.F:762
    assert g["NE"] == (3 * N + (g["ISBC"] == 1).sum()) // 2
    # every cell has exactly three edges
    cnt = np.zeros(N + 1, int)
    for e in range(1, g["NE"] + 1):
        cnt[g["IEC"][e, 0]] += 1
        if g["IEC"][e, 1] > 0:
            cnt[g["IEC"][e, 1]] += 1
    assert (cnt[1:] == 3).all()


def test_areas_partition_domain():
    c = cases.estuary_channel(nx=12, ny=4, kb=4, lx=6000.0, ly=2000.0)
    g = c["grid"]
    total = 6000.0 * 2000.0
    assert abs(g["ART"][1:].sum() - total) < 1e-6 * total
    assert abs(g["ART1"][1:].sum() - total) < 1e-6 * total      # median-dual CVs tile the mesh
    assert abs(g["ART2"][1:].sum() - 3 * total) < 1e-6 * total  # each cell counted at its 3 nodes


def test_rings_close_and_half_edges_balance():
    c = cases.coastal_mesh(npts=800, kb=4, lx=8000.0, ly=4000.0, seed=3)
    g = c["grid"]
    M = g["M"]
    for i in range(1, M + 1):
        nt = g["NTSN"][i]
        ring = g["NBSN"][i, :nt]
        assert ring[0] == ring[nt - 1]                 # closed ring (tge.F:338, 387)
        if g["ISONB"][i] == 0:
            assert g["NBVE"][i, 0] == g["NBVE"][i, g["NTVE"][i]]
    # sum over a node's CV half-edges of the signed edge vectors closes the CV
    sx = np.zeros(M + 1)
    sy = np.zeros(M + 1)
    for he in range(1, g["NCV"] + 1):
        a, b = g["NIEC"][he]
        sx[a] -= g["DLTXE"][he]; sx[b] += g["DLTXE"][he]
        sy[a] -= g["DLTYE"][he]; sy[b] += g["DLTYE"][he]
    interior = g["ISONB"][1:] == 0
    assert np.abs(sx[1:][interior]).max() < 1e-6
    assert np.abs(sy[1:][interior]).max() < 1e-6


def test_uniform_sigma_is_single_precision_quotient():
    c = cases.estuary_channel(nx=4, ny=2, kb=11, lx=4000.0, ly=2000.0)
    z = c["grid"]["Z"][1]
    assert z[1] == -float(np.float32(1.0) / np.float32(10.0))   # mod_setup.F:855
    assert z[0] == 0.0 and z[-1] == -1.0


def test_shape_coefficients_reproduce_linear_field():
    c = cases.coastal_mesh(npts=900, kb=4, lx=9000.0, ly=4500.0, seed=5)
    g = c["grid"]
    xc, yc, nbe = g["XC"], g["YC"], g["NBE"]
    u = 0.3 + 2e-4 * xc - 5e-5 * yc
    for i in range(1, g["N"] + 1):
        if g["ISBCE"][i] != 0:
            continue
        k = nbe[i]
        vals = np.array([u[i], u[k[0]], u[k[1]], u[k[2]]])
        assert abs(g["A1U"][i] @ vals - 2e-4) < 1e-9
        assert abs(g["A2U"][i] @ vals + 5e-5) < 1e-9


def test_ghost_cell_coefficients():
    """SHAPE_COEF_GCY: boundary cells get least-squares weights from their ghost points
    (GCN leaves them zero); GCY1 and GCY2 differ only on solid-boundary cells; on interior
    cells the weights equal GCN's except the first A2U weight, which the reference's GCY
    routine forms with the sum of X squared in place of the sum of X*Y."""
    import numpy as np
    from myfvcomcode_b200 import cases
    kw = dict(npts=1500, kb=5, lx=20000.0, ly=10000.0, seed=7)
    g0 = cases.coastal_mesh(**kw)["grid"]
    g1 = cases.coastal_mesh(ghost_cells="GCY1", **kw)["grid"]
    g2 = cases.coastal_mesh(ghost_cells="GCY2", **kw)["grid"]
    isbce = np.asarray(g0["ISBCE"])
    solid = isbce == 1
    obc = isbce == 2
    interior = isbce == 0
    interior[0] = False
    assert solid.sum() > 10 and obc.sum() > 5
    assert np.all(g0["A1U"][solid] == 0.0) and np.all(np.abs(g1["A1U"][solid]).sum(axis=1) > 0)
    assert np.array_equal(g1["A1U"][interior], g0["A1U"][interior])
    assert np.array_equal(g1["A2U"][interior][:, 1:], g0["A2U"][interior][:, 1:])
    assert not np.array_equal(g1["A2U"][interior][:, 0], g0["A2U"][interior][:, 0])
    assert np.array_equal(g1["A1U"][~solid & (isbce != 3)], g2["A1U"][~solid & (isbce != 3)])
    assert not np.array_equal(g1["A1U"][solid], g2["A1U"][solid])
