"""FVCOM run directories: namelist parsing, grid and forcing files, time-varying forcing.

CPU tests check the readers against the reference's own formats (mod_input.F,
mod_force.F, mod_nctools.F), a write -> read round trip that must rebuild every mesh
array bit for bit, the bracketing rules of river (nearest record) and wind (linear)
forcing, and the oracle stepped through ``FvcomRun``.  The GPU test runs the same
file-driven case with forcing that changes every step on the library and the oracle
and requires bitwise equal states.
"""
import os

import numpy as np
import pytest

from myfvcomcode_b200 import cases, fvcom_input as fi

# The reference's own Estuary example (Examples/Estuary/run/tst_run.nml of the FVCOM
# tree), located by FVCOM_ESTUARY_NML; the test that reads it is skipped when unset.
ESTUARY = os.environ.get("FVCOM_ESTUARY_NML", "")

NML_TEXT = """
 &NML_CASE
 CASE_TITLE      = 'IDEAL ''QUOTED'' CASE'   ! a comment with a / slash
 START_DATE      = 'seconds=0.0'
 END_DATE        = 'days=1.5'
 /
 &NML_PHYSICS
 WETTING_DRYING_ON = .TRUE., BAROTROPIC = F,
 VERTICAL_MIXING_COEFFICIENT = 1.0D-4,
 HORIZONTAL_MIXING_COEFFICIENT = 2.E-1
 EMPTY_KEY =              ,
 /
 &NML_GRID_COORDINATES
 GRID_FILE       = tst_grd.dat  ,
 PROJECTION_REFERENCE  = 'proj=tmerc +lon_0=-70d10'
 /
 &NML_RIVER
 RIVER_NAME = 'r1'
 RIVER_VERTICAL_DISTRIBUTION = 3*0.2 0.4
 /
 &NML_RIVER
 RIVER_NAME = 'r2', RIVER_GRID_LOCATION = 12,
 RIVER_VERTICAL_DISTRIBUTION = 'uniform'
 /
"""


def test_parse_namelist():
    nml = fi.parse_namelist(NML_TEXT)
    case = fi.group(nml, "NML_CASE")
    assert case["CASE_TITLE"] == "IDEAL 'QUOTED' CASE"
    assert case["END_DATE"] == "days=1.5"
    ph = fi.group(nml, "nml_physics")
    assert ph["WETTING_DRYING_ON"] is True and ph["BAROTROPIC"] is False
    assert ph["VERTICAL_MIXING_COEFFICIENT"] == 1.0e-4
    assert ph["HORIZONTAL_MIXING_COEFFICIENT"] == 0.2
    assert ph["EMPTY_KEY"] is None
    gc = fi.group(nml, "NML_GRID_COORDINATES")
    assert gc["GRID_FILE"] == "tst_grd.dat"
    assert gc["PROJECTION_REFERENCE"] == "proj=tmerc +lon_0=-70d10"
    rivers = nml["NML_RIVER"]
    assert len(rivers) == 2
    assert rivers[0]["RIVER_VERTICAL_DISTRIBUTION"] == [0.2, 0.2, 0.2, 0.4]
    assert rivers[1]["RIVER_GRID_LOCATION"] == 12 and rivers[1]["RIVER_VERTICAL_DISTRIBUTION"] == "uniform"
    assert fi.group(nml, "NML_ABSENT") == {}


def test_parse_time():
    assert fi.parse_time("seconds=3600.") == ("relative", 3600.0)
    assert fi.parse_time("days=3.0") == ("relative", 3.0 * 86400.0)
    assert fi.parse_time("cycle = 200") == ("cycle", 200.0)
    assert fi.parse_time("none") is None
    kind, t = fi.parse_time("1858-11-18 00:00:00")
    assert kind == "date" and t == 86400.0


def test_bracket_rules():
    t = np.array([0.0, 100.0, 300.0])
    assert fi.bracket(t, 0.0) == (0, 1, 0.0)
    assert fi.bracket(t, 100.0) == (0, 1, 1.0)   # prev < now <= next
    p, n, w = fi.bracket(t, 150.0)
    assert (p, n) == (1, 2) and w == 0.25
    with pytest.raises(ValueError):
        fi.bracket(t, 300.5)
    with pytest.raises(ValueError):
        fi.bracket(t, -1.0)


def _series_case(tmp_path, case, end_s, heat=False):
    """Write ``case`` with a river that steps 100 -> 300 m^3/s and a wind stress that
    grows linearly over the run (and, with ``heat``, surface heating that turns from
    warming to cooling); return the namelist path."""
    g = case["grid"]
    nq, N, M = g["NUMQBC"], g["N"], g["M"]
    heat_series = None
    if heat:
        case = dict(case, params=dict(case["params"], HEATING_ON=True, HEATING_LONGWAVE_PERCTAGE=0.78,
                                      HEATING_LONGWAVE_LENGTHSCALE=1.4, HEATING_SHORTWAVE_LENGTHSCALE=6.3),
                    forcing=dict(case["forcing"], heat=dict(swrad=300.0, wtsurf=200.0)))
        ht = np.array([0.0, 0.5 * end_s, end_s + 1000.0])
        heat_series = (ht, np.tile([[300.0], [150.0], [0.0]], (1, M)), np.tile([[200.0], [0.0], [-250.0]], (1, M)))
    tt = np.array([0.0, 250.0, 520.0, end_s + 1000.0])
    flux = np.array([[100.0] * nq, [100.0] * nq, [300.0] * nq, [300.0] * nq])
    temp = np.tile(np.array([[15.0] * nq]), (4, 1)) + np.arange(4)[:, None]
    salt = np.zeros((4, nq))
    wt = np.array([0.0, end_s + 1000.0])
    rng = np.random.default_rng(3)
    base = rng.uniform(0.05, 0.15, N)
    sx = np.stack([0.0 * base, 2.0 * base])
    sy = np.stack([0.0 * base, -1.0 * base])
    return fi.write_run(case, str(tmp_path), name="tst", days=end_s / 86400.0,
                        river_series=(tt, flux, temp, salt), wind_series=(wt, sx, sy),
                        heat_series=heat_series)


def test_round_trip_rebuilds_the_mesh(tmp_path, small_channel_edge):
    case = small_channel_edge
    path = fi.write_run(case, str(tmp_path), name="rt", days=0.1)
    run = fi.FvcomRun(path)
    a, b = case["grid"].a, run.case["grid"].a
    checked = 0
    for k, v in a.items():
        if isinstance(v, np.ndarray):
            assert k in b, k
            assert np.array_equal(v, b[k]), k
            checked += 1
    assert checked > 60
    for k, v in case["params"].items():
        assert run.case["params"][k] == v, k
    assert run.case["init"] == case["init"]
    for k in ("period", "apt", "phai", "emean"):
        assert np.array_equal(np.asarray(case["forcing"]["tide"][k], dtype=float),
                              np.asarray(run.case["forcing"]["tide"][k], dtype=float)), k
    assert np.array_equal(run.case["forcing"]["qdis"], case["forcing"]["qdis"])
    assert run.steps == int(round(0.1 * 86400.0 / (case["params"]["DTE"] * case["params"]["ISPLIT"])))


def test_round_trip_geometric_sigma(tmp_path):
    case = cases.estuary_channel(nx=8, ny=4, kb=7, lx=1600.0, ly=800.0, river=False)
    from myfvcomcode_b200.grid import build_grid
    g0 = case["grid"]
    g = build_grid(g0["VX"][1:] + g0["VXMIN"], g0["VY"][1:] + g0["VYMIN"], g0["NV"][1:], g0["H"][1:], 7,
                   obc_nodes=list(g0["I_OBC_N"][1:]), obc_types=list(g0["TYPE_OBC"][1:]),
                   cor_lat=30.0, sponge=g0["SPONGE_LIST"], p_sigma=2.0)
    z = g["Z"][1]
    assert z[0] == 0.0 and z[-1] == -1.0 and np.all(np.diff(z) < 0.0)
    assert np.allclose(z + z[::-1], -1.0)  # symmetric about mid-depth
    case = dict(case, grid=g)
    run = fi.FvcomRun(fi.write_run(case, str(tmp_path), name="geo", days=0.01))
    assert np.array_equal(run.case["grid"]["Z"], g["Z"])


def test_forcing_schedule(tmp_path, small_channel_edge):
    end = 2000.0
    run = fi.FvcomRun(_series_case(tmp_path, small_channel_edge, end))
    dti = run.dti
    assert dti == 20.0
    q, t, s = run.rivers.at(240.0)
    assert np.all(q == 100.0)
    q, t, s = run.rivers.at(300.0)     # prev weight (520-300)/270 > 0.5: previous record
    assert np.all(q == 100.0) and np.all(t == 16.0)
    q, t, s = run.rivers.at(385.0)     # prev weight exactly 0.5: next record
    assert np.all(q == 300.0) and np.all(t == 17.0)
    q, t, s = run.rivers.at(400.0)     # prev weight 0.444: next record
    assert np.all(q == 300.0) and np.all(t == 17.0)
    sx, sy = run.wind.at(1000.0)
    w = 1000.0 / (end + 1000.0)
    assert sx[0] == 0.0 and np.allclose(sx[1:], w * run.wind.u[1] + (1 - w) * run.wind.u[0])


def test_oracle_steps_with_changing_forcing(tmp_path, small_channel_edge):
    from oracle.oracle import Oracle
    run = fi.FvcomRun(_series_case(tmp_path, small_channel_edge, 1000.0))
    a = Oracle(run.case)
    run.run(a, steps=30)
    # the same steps without the forcing updates differ (the river steps up at 400 s,
    # the wind grows every step)
    b = Oracle(run.case)
    b.run(30)
    assert np.isfinite(a.get("el")).all() and np.isfinite(a.get("u")).all()
    assert not np.array_equal(a.get("u"), b.get("u"))
    # a forcing update with unchanged values changes nothing
    c, d = Oracle(run.case), Oracle(run.case)
    for _ in range(3):
        c.set_forcing(run.case["forcing"])
        c.internal_step()
        d.internal_step()
    for n in ("el", "u", "t1", "s1", "q2"):
        assert np.array_equal(c.get(n), d.get(n)), n


def test_history_written_every_interval(tmp_path, small_channel):
    from scipy.io import netcdf_file
    from oracle.oracle import Oracle
    from myfvcomcode_b200 import ncio
    path = fi.write_run(small_channel, str(tmp_path), name="h", days=0.05)
    run = fi.FvcomRun(path)
    run.nc_interval = 10 * run.dti
    o = Oracle(run.case)
    hist = ncio.History(os.path.join(str(tmp_path), "h_0001.nc"), run.case)
    run.run(o, steps=25, history=hist)
    hist.close()
    with netcdf_file(os.path.join(str(tmp_path), "h_0001.nc"), "r", mmap=False) as nc:
        assert list(nc.variables["iint"][:]) == [0, 10, 20]


@pytest.mark.skipif(not ESTUARY or not os.path.exists(ESTUARY),
                    reason="FVCOM_ESTUARY_NML does not name the reference's Estuary example")
def test_reads_the_estuary_example():
    from oracle.oracle import Oracle
    run = fi.FvcomRun(ESTUARY)
    g = run.case["grid"]
    assert (g["M"], g["N"], g["KB"], g["IOBCN"], g["NUMQBC"]) == (845, 1570, 11, 25, 3)
    assert run.dti == 50.0 and run.steps == 5184 and run.nc_interval == 3600.0
    assert g["RIVER_LOC"] == "edge" and np.allclose(g["VQDIST"][1:], 0.1)
    assert np.all(run.case["forcing"]["qdis"] == 200.0)
    assert run.case["params"]["WETTING_DRYING_ON"] is True and run.case["params"]["IRAMP"] == 500
    o = Oracle(run.case)
    run.run(o, steps=40)
    assert np.isfinite(o.get("el")).all() and np.isfinite(o.get("u")).all()


def test_heat_series(tmp_path, small_channel_edge):
    run = fi.FvcomRun(_series_case(tmp_path, small_channel_edge, 1000.0, heat=True))
    assert run.case["params"]["HEATING_ON"] is True
    assert run.case["params"]["HEATING_SHORTWAVE_LENGTHSCALE"] == 6.3
    sw, nf = run.heat.at(250.0)   # a quarter of the way from the first to the last record
    assert sw[0] == 0.0 and np.allclose(sw[1:], 225.0) and np.allclose(nf[1:], 100.0)


@pytest.mark.gpu
@pytest.mark.parametrize("heat", [False, True])
def test_file_driven_run_matches_oracle(tmp_path, small_channel_edge, heat):
    """Forcing from files, changing every step, through the library and the oracle: the
    north-star tolerance on zeta, u, v, T, S (the tidal cos, BROUGH log, VDIF_Q powers
    and the short-wave exp are device functions), wet flags exact."""
    import tests.parity as parity
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    run = fi.FvcomRun(_series_case(tmp_path, small_channel_edge, 1000.0, heat=heat))
    f, o = Fvcom(run.case), Oracle(run.case)
    run.run(f, steps=30)
    run.run(o, steps=30)
    f.sync()
    bad = parity.compare(f, o, ["el", "ua", "va", "u", "v", "t1", "s1"], rtol=1e-9)
    assert not bad, bad
    for n in ("iswetn", "iswetc"):
        assert np.array_equal(f.get(n), o.get(n)), n
    assert f.clock() == o.clock()
    f.close()
