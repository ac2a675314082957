"""Surface heating, HEATING_TYPE 'flux' (vdif_ts.F:118-150, bcond_gcn.F:683-694).

Known answers on the oracle: after one internal step the heat a column gains over an
unheated twin is DTI*RAMP/(SPCP*ROSEA) times the net flux minus the short-wave that
leaves through the bottom, RAD(KB) = SW*(RHEAT*exp(-D/ZETA1) + (1-RHEAT)*exp(-D/ZETA2));
cooling stops for water at or below -2 C.  On the GPU the library follows the oracle to
1e-9 relative (the short-wave profile uses the device's exp, so not bit for bit).
"""
import numpy as np
import pytest

from myfvcomcode_b200 import cases

SPRO = 4.2174e3 * 1.023e3


def _heated(case, swrad, wtsurf, **kw):
    p = dict(case["params"], HEATING_ON=True, HEATING_LONGWAVE_PERCTAGE=0.78,
             HEATING_LONGWAVE_LENGTHSCALE=1.4, HEATING_SHORTWAVE_LENGTHSCALE=6.3, **kw)
    f = dict(case["forcing"], heat=dict(swrad=swrad, wtsurf=wtsurf))
    return dict(case, params=p, forcing=f)


@pytest.fixture(scope="module")
def channel():
    return cases.estuary_channel(nx=24, ny=6, kb=6, lx=4800.0, ly=1200.0, IRAMP=0, river=False)


def _column_heat(model, g):
    t = model.get3("t1")[:, : g["KB"] - 1]
    dz = g["DZ"][:, : g["KB"] - 1]
    return (t * dz).sum(axis=1) * model.get("d")


def _interior_wet(model, g):
    ok = model.get("iswetn") == 1
    ok[0] = False
    ok[np.asarray(g["I_OBC_N"][1:], dtype=int)] = False
    return ok


def test_net_heat_flux_known_answer(channel):
    from oracle.oracle import Oracle
    g = channel["grid"]
    q_net, sw = 400.0, 250.0
    a, b = Oracle(_heated(channel, sw, q_net)), Oracle(channel)
    a.internal_step()
    b.internal_step()
    ok = _interior_wet(a, g)
    gain = (_column_heat(a, g) - _column_heat(b, g))[ok]
    D = a.get("d")[ok]
    dti = channel["params"]["DTE"] * channel["params"]["ISPLIT"]
    leak = sw * (0.78 * np.exp(-D / 1.4) + 0.22 * np.exp(-D / 6.3))
    want = dti * (q_net - leak) / SPRO
    assert np.allclose(gain, want, rtol=1e-9, atol=0.0)
    # the short-wave is absorbed near the surface: the warming falls off with depth
    dT = (a.get3("t1") - b.get3("t1"))[ok, : g["KB"] - 1]
    assert np.all(dT[:, 0] > dT[:, -1])


def test_no_cooling_below_freezing(channel):
    from oracle.oracle import Oracle
    g = channel["grid"]
    cold = dict(channel, init=dict(channel["init"], t=-3.0))
    a, b = Oracle(_heated(cold, 0.0, -300.0)), Oracle(cold)
    a.internal_step()
    b.internal_step()
    ok = _interior_wet(a, g)
    assert np.array_equal(a.get3("t1")[ok], b.get3("t1")[ok])
    warm = dict(channel, init=dict(channel["init"], t=10.0))
    c, d = Oracle(_heated(warm, 0.0, -300.0)), Oracle(warm)
    c.internal_step()
    d.internal_step()
    assert np.all(_column_heat(c, g)[ok] < _column_heat(d, g)[ok])


def test_heating_off_ignores_heat_forcing(channel):
    from oracle.oracle import Oracle
    c = _heated(channel, 500.0, 500.0)
    c["params"]["HEATING_ON"] = False
    a, b = Oracle(c), Oracle(channel)
    a.run(3)
    b.run(3)
    assert np.array_equal(a.get("t1"), b.get("t1"))


@pytest.mark.gpu
def test_heating_matches_oracle(channel):
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    import tests.parity as parity
    rng = np.random.default_rng(5)
    M = channel["grid"]["M"]
    c = _heated(channel, rng.uniform(100.0, 400.0, M + 1), rng.uniform(-200.0, 300.0, M + 1))
    f, o = Fvcom(c), Oracle(c)
    f.run(20)
    o.run(20)
    bad = parity.compare(f, o, ["el", "u", "v", "t1", "s1"], rtol=1e-9)
    assert not bad, bad
    assert np.array_equal(f.get("iswetn"), o.get("iswetn"))
    # the forcing can change between steps
    sw2 = rng.uniform(0.0, 100.0, M + 1)
    nf2 = rng.uniform(-100.0, 100.0, M + 1)
    for m in (f, o):
        m.set_forcing(dict(c["forcing"], heat=dict(swrad=sw2, wtsurf=nf2)))
        m.run(5)
    bad = parity.compare(f, o, ["el", "u", "v", "t1", "s1"], rtol=1e-9)
    assert not bad, bad
    f.close()
