"""Parity of the CUDA library with the CPU oracle, on a B200.

Per routine: both engines start from the same bits (the oracle state copied into the
library), run one reference routine and must agree bit for bit, except where the routine
evaluates a transcendental function the reference computes at run time (cos of the tide,
log of the roughness, real powers in MY2.5), where CUDA's libm and the host's differ in the
last place; those are held to 1e-13 relative.

Whole steps: from the same cold start both engines advance; zeta, u, v, T and S must agree
to 1e-9 relative after 1000 external steps (100 internal steps at ISPLIT=10) on the
estuary channel workload.
"""
import numpy as np
import pytest

from tests import parity

pytestmark = pytest.mark.gpu

TRANSCENDENTAL = {"BCOND_ELF", "BROUGH", "VDIF_Q", "EXTERNAL_STEP", "INT_FORCING"}

ROUTINES = [
    ("INT_FORCING", 0, ["qdis", "wusurf", "wvsurf"]),
    ("ADJUST2D3D", 1, ["u", "v"]),
    ("BCOND_UV3D_SOLID", 0, ["u", "v"]),
    ("BROUGH", 0, ["cbc", "wubot", "wvbot", "taubm", "wubot_n", "wvbot_n", "taubm_n"]),
    ("ADVECTION3D", 0, ["advx", "advy"]),
    ("BAROPG", 0, ["drhox", "drhoy", "rho", "rho1"]),
    ("INT_PRE_EXT", 0, ["adx2d", "ady2d", "drx2d", "dry2d", "advua", "advva", "pstx", "psty",
                        "uard", "vard", "egf", "uard_obcn"]),
    ("EXTEL_EDGE", 1, ["elf", "xflux_obcn"]),
    ("EXTEL_EDGE", 3, ["elf", "xflux_obcn"]),
    ("BCOND_ELF", 2, ["elf"]),
    ("N2E2D_ELF", 0, ["elf1"]),
    ("WET_JUDGE", 0, ["iswetn", "iswetc", "elf", "elf1"]),
    ("FLUX_OBN", 4, ["fluxobn"]),
    ("ADVAVE", 0, ["advua", "advva", "pstx", "psty"]),
    ("EXTUV_EDGE", 2, ["uaf", "vaf"]),
    ("BCOND_UV2D", 0, ["uaf", "vaf"]),
    ("EXT_UPDATE", 3, ["el", "d", "dtfa", "egf", "el1", "d1", "ua", "va", "uard", "vard", "iswetce"]),
    ("EXT_UPDATE", 4, ["el", "d", "uard_obcn", "ua", "va"]),
    ("EXTERNAL_STEP", 1, ["el", "elf", "ua", "va", "d1", "uard", "egf", "fluxobn"]),
    ("ADJUST2D3D", 2, ["u", "v", "uard", "vard"]),
    ("VERTVL", 0, ["wts", "dtfa", "w"]),
    ("VISCOFH", 0, ["viscofh"]),
    ("ADV_UV", 0, ["uf", "vf", "viscofm"]),
    ("VDIF_UV", 0, ["uf", "vf", "tps", "wubot", "wvbot"]),
    ("BCOND_UV3D", 0, ["uf", "vf"]),
    ("WREAL", 0, ["ww"]),
    ("ADV_Q", 0, ["q2f"]),
    ("ADV_Q", 1, ["q2lf"]),
    ("FCT_Q", 0, ["q2f"]),
    ("FCT_Q", 1, ["q2lf"]),
    ("VDIF_Q", 0, ["q2", "q2l", "q2f", "q2lf", "l", "km", "kh", "kq"]),
    ("TURB_UPDATE", 0, ["q2", "q2l", "km1"]),
    ("ADV_TS", 1, ["tf1", "pfpxb", "pfpyb", "ah_bottom", "xflux_obc"]),
    ("ADV_TS", 2, ["sf1", "pfpxb", "pfpyb", "ah_bottom", "xflux_obc"]),
    ("FCT_TS", 1, ["tf1"]),
    ("FCT_TS", 2, ["sf1"]),
    ("VDIF_TS", 1, ["tf1"]),
    ("VDIF_TS", 2, ["sf1"]),
    ("BCOND_TS", 1, ["tf1", "sf1"]),
    ("BCOND_TS", 2, ["tf1", "sf1"]),
    ("TS_UPDATE", 1, ["t1", "t"]),
    ("TS_UPDATE", 2, ["s1", "s"]),
    ("DENS2", 0, ["rho1", "rho"]),
    ("INT_FINAL", 0, ["u", "v", "et", "dt", "et1", "dt1", "iswetct", "iswetnt"]),
]


def _engines(case, steps):
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    ora = Oracle(case)
    ora.run(steps)
    gpu = Fvcom(case)
    return ora, gpu


@pytest.mark.parametrize("case_name", ["small_channel", "small_channel_edge", "small_coastal"])
def test_each_routine_matches_oracle(case_name, request):
    failures = routine_failures(request.getfixturevalue(case_name), 4)
    assert not failures, failures


def routine_failures(case, warm):
    """Run every routine of ROUTINES on the library and the oracle from the oracle's state
    after ``warm`` internal steps; return the routines whose outputs differ (bitwise, or
    beyond 1e-13 relative for the TRANSCENDENTAL ones)."""
    ora, gpu = _engines(case, warm)
    wind = case["forcing"].get("wind")
    failures = {}
    for name, arg, outs in ROUTINES:
        parity.copy_state(ora, gpu)
        if name == "EXTUV_EDGE" and wind is not None:
            # the oracle keeps WUSURF2 from BCOND_GCN(9,0); the library forms it in EXTUV
            from myfvcomcode_b200.abi import wind_stress
            sx, sy = wind_stress(case)
            r = ora.ramp()
            ora.set("wusurf2", sx * r * 0.001)
            ora.set("wvsurf2", sy * r * 0.001)
        gpu.routine(name, arg)
        ora.routine(name, arg)
        tracer = 2 if (name in ("ADV_TS",) and arg == 2) else 1
        bad = parity.compare(gpu, ora, outs, rtol=1e-13 if name in TRANSCENDENTAL else 0.0, tracer=tracer)
        if bad:
            failures["%s(%d)" % (name, arg)] = bad
    gpu.close()
    return failures


@pytest.mark.parametrize("case_name", ["small_channel", "small_channel_edge", "small_coastal"])
def test_internal_steps_match_oracle(case_name, request):
    case = request.getfixturevalue(case_name)
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    ora = Oracle(case)
    gpu = Fvcom(case)
    ora.run(20)
    gpu.run(20)
    bad = parity.compare(gpu, ora, ["el", "ua", "va", "u", "v", "w", "t1", "s1", "q2", "q2l", "km", "kh",
                                    "rho1", "wts", "d1"], rtol=1e-10)
    assert not bad, bad
    assert np.array_equal(gpu.get("iswetn"), ora.get("iswetn"))
    assert np.array_equal(gpu.get("iswetc"), ora.get("iswetc"))
    assert gpu.clock() == ora.clock()


def test_estuary_channel_1000_external_steps_within_1e9():
    """The plain FP64 path against the FP64 oracle on the 2,121-node / 4,000-cell channel:
    zeta, u, v, T and S after 1000 external steps (north-star tolerance 1e-9 relative)."""
    from myfvcomcode_b200 import cases
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    case = cases.estuary_channel()
    ora = Oracle(case)
    gpu = Fvcom(case)
    ora.run(100)
    gpu.run(100)
    bad = parity.compare(gpu, ora, ["el", "u", "v", "t1", "s1"], rtol=1e-9)
    assert not bad, bad


def test_plain_path_is_bitwise_deterministic(small_coastal):
    from myfvcomcode_b200.engine import Fvcom
    a = Fvcom(small_coastal)
    b = Fvcom(small_coastal)
    a.run(6)
    b.run(6)
    for n in ("el", "ua", "u", "v", "t1", "s1", "q2", "km", "wts"):
        assert np.array_equal(a.get(n), b.get(n)), n


def test_graph_replay_equals_plain_launches(small_channel):
    from myfvcomcode_b200.engine import Fvcom
    a = Fvcom(small_channel)
    b = Fvcom(small_channel)
    b.use_graph(False)
    a.run(5)
    b.run(5)
    for n in ("el", "ua", "u", "t1", "s1", "q2l", "kh"):
        assert np.array_equal(a.get(n), b.get(n)), n


@pytest.mark.parametrize("threads,layers", [(32, 1), (64, 3), (256, 7)])
def test_launch_shape_does_not_change_results(small_coastal, threads, layers):
    from myfvcomcode_b200.engine import Fvcom
    a = Fvcom(small_coastal)
    b = Fvcom(small_coastal)
    b.set_tuning("col_threads", threads)
    b.set_tuning("col_layers", layers)
    assert (b.get_tuning("col_threads"), b.get_tuning("col_layers")) == (threads, layers)
    a.run(4)
    b.run(4)
    for n in ("el", "ua", "u", "v", "w", "t1", "s1", "q2", "q2l", "km", "viscofh", "wts"):
        assert np.array_equal(a.get(n), b.get(n)), n


def test_autotuner_returns_a_timed_shape(small_channel):
    from myfvcomcode_b200 import autotune
    r = autotune.autotune(small_channel, cands=[(64, 1), (128, 5)], steps=2, warmup=1)
    assert (r["col_threads"], r["col_layers"]) in [(64, 1), (128, 5)]
    assert len(r["table"]) == 2 and all(t[0] > 0 for t in r["table"])


def test_set_forcing_and_external_step(small_coastal):
    import ctypes as C
    from myfvcomcode_b200 import abi
    from myfvcomcode_b200.engine import Fvcom
    a, b, c = Fvcom(small_coastal), Fvcom(small_coastal), Fvcom(small_coastal)
    _, _, fs, keep = abi.make_structs(small_coastal)
    b.lib.fvg_set_forcing.argtypes = [C.c_void_p, C.c_void_p]
    assert b.lib.fvg_set_forcing(b.h, C.byref(fs)) == 0  # the same forcing: no change
    ws = abi.wind_stress(small_coastal)
    sx = np.ascontiguousarray(ws[0] * 2.0)
    sy = np.ascontiguousarray(ws[1] * 2.0)
    fs2 = abi.FvgForcing()
    C.pointer(fs2)[0] = fs
    fs2.wstress_x = sx.ctypes.data_as(C.POINTER(C.c_double))
    fs2.wstress_y = sy.ctypes.data_as(C.POINTER(C.c_double))
    assert c.lib.fvg_set_forcing(c.h, C.byref(fs2)) == 0
    for m in (a, b, c):
        m.run(3)
    assert np.array_equal(a.get("el"), b.get("el")) and np.array_equal(a.get("u"), b.get("u"))
    assert not np.array_equal(a.get("u"), c.get("u"))
    # one EXTERNAL_STEP through its own entry point equals the routine call
    d, e = Fvcom(small_coastal), Fvcom(small_coastal)
    d.lib.fvg_external_step.argtypes = [C.c_void_p, C.c_int32]
    assert d.lib.fvg_external_step(d.h, 1) == 0
    e.routine("EXTERNAL_STEP", 1)
    for n in ("el", "ua", "va", "elf"):
        assert np.array_equal(d.get(n), e.get(n)), n
    assert d.lib.fvg_external_step(d.h, 0) == 1


LIMITED_ROUTINES = [
    ("ADVECTION3D", 0, ["advx", "advy"]),
    ("INT_PRE_EXT", 0, ["adx2d", "ady2d", "drx2d", "dry2d", "advua", "advva", "pstx", "psty"]),
    ("ADVAVE", 0, ["advua", "advva", "pstx", "psty"]),
    ("ADV_UV", 0, ["uf", "vf", "viscofm"]),
    ("EXTERNAL_STEP", 1, ["el", "elf", "ua", "va", "d1", "uard", "egf", "fluxobn"]),
]


@pytest.mark.parametrize("limiter", ["LIMITED_1", "LIMITED_2"])
@pytest.mark.parametrize("case_name", ["small_channel", "small_coastal"])
def test_limited_schemes_match_oracle(case_name, limiter, request):
    """The limited momentum advection (slope limiter, and LIMITED_1's clamp) per routine
    bit for bit (EXTERNAL_STEP to 1e-13: its tide is a device cos), and 20 whole steps."""
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    base = request.getfixturevalue(case_name)
    case = dict(base, params=dict(base["params"], LIMITER=limiter))
    ora, gpu = Oracle(case), Fvcom(case)
    ora.run(4)
    failures = {}
    for name, arg, outs in LIMITED_ROUTINES:
        parity.copy_state(ora, gpu)
        gpu.routine(name, arg)
        ora.routine(name, arg)
        bad = parity.compare(gpu, ora, outs, rtol=1e-13 if name in TRANSCENDENTAL else 0.0)
        if bad:
            failures["%s(%d)" % (name, arg)] = bad
    assert not failures, failures
    a, b = Oracle(case), Fvcom(case)
    a.run(20)
    b.run(20)
    bad = parity.compare(b, a, ["el", "ua", "va", "u", "v", "t1", "s1"], rtol=1e-10)
    assert not bad, bad
    b.set_precision("fp32flux")
    b.run(5)
    assert np.isfinite(b.get("u")).all() and np.isfinite(b.get("el")).all()


@pytest.mark.parametrize("case_name", ["small_channel", "small_coastal"])
def test_z_level_pressure_gradient_matches_oracle(case_name, request):
    """BAROCLINIC_PRESSURE_GRADIENT = 'z coordinates' (PHY_BAROPG): the routine bit for
    bit from the same state, and 20 whole steps to 1e-10."""
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    base = request.getfixturevalue(case_name)
    case = dict(base, params=dict(base["params"], BAROCLINIC_PRESSURE_GRADIENT="z coordinates"))
    ora, gpu = Oracle(case), Fvcom(case)
    ora.run(4)
    parity.copy_state(ora, gpu)
    gpu.routine("BAROPG", 0)
    ora.routine("BAROPG", 0)
    bad = parity.compare(gpu, ora, ["drhox", "drhoy", "rho1"])
    assert not bad, bad
    a, b = Oracle(case), Fvcom(case)
    a.run(20)
    b.run(20)
    bad = parity.compare(b, a, ["el", "ua", "va", "u", "v", "t1", "s1", "rho1"], rtol=1e-10)
    assert not bad, bad


GCY_ROUTINES = [
    ("BCOND_UV3D_SOLID", 0, ["u", "v"]),
    ("ADVECTION3D", 0, ["advx", "advy"]),
    ("INT_PRE_EXT", 0, ["adx2d", "ady2d", "drx2d", "dry2d", "advua", "advva", "pstx", "psty"]),
    ("ADVAVE", 0, ["advua", "advva", "pstx", "psty"]),
    ("BCOND_UV2D", 0, ["uaf", "vaf"]),
    ("EXTERNAL_STEP", 1, ["el", "elf", "ua", "va", "d1", "uard", "egf", "fluxobn"]),
    ("ADV_UV", 0, ["uf", "vf", "viscofm"]),
    ("BCOND_UV3D", 0, ["uf", "vf"]),
]


@pytest.mark.parametrize("ghost", ["GCY1", "GCY2"])
@pytest.mark.parametrize("case_name", ["channel_edge", "coastal"])
def test_ghost_cells_match_oracle(case_name, ghost):
    """GCY (ghost velocities in the gradients, the GCY flux masks, no tangential projection)
    per routine bit for bit (EXTERNAL_STEP to 1e-13) and whole internal steps from the
    same state to 1e-12, with and without LIMITED_1; 20 free-running steps to 1e-10
    without it.  LIMITED_1's clamp is discontinuous: a last-place difference of the
    device's tidal cos can switch it on one edge, after which free-running runs part at
    1e-9 and more although every single step agrees to 1e-15 (measured)."""
    from myfvcomcode_b200 import cases
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    if case_name == "channel_edge":
        base = cases.estuary_channel(nx=24, ny=6, kb=6, lx=4800.0, ly=1200.0, IRAMP=10,
                                     river_location="edge", ghost_cells=ghost)
    else:
        base = cases.coastal_mesh(npts=1500, kb=7, lx=20000.0, ly=10000.0, seed=7, IRAMP=20, ghost_cells=ghost)
    for lim in ("LIMITED_NO", "LIMITED_1"):
        case = dict(base, params=dict(base["params"], LIMITER=lim))
        ora, gpu = Oracle(case), Fvcom(case)
        ora.run(4)
        failures = {}
        for name, arg, outs in GCY_ROUTINES:
            parity.copy_state(ora, gpu)
            gpu.routine(name, arg)
            ora.routine(name, arg)
            bad = parity.compare(gpu, ora, outs, rtol=1e-13 if name in TRANSCENDENTAL else 0.0)
            if bad:
                failures["%s(%d)" % (name, arg)] = bad
        assert not failures, (lim, failures)
        for step in range(10):
            parity.copy_state(ora, gpu)
            ora.internal_step()
            gpu.internal_step()
            bad = parity.compare(gpu, ora, ["el", "ua", "va", "u", "v", "t1", "s1"], rtol=1e-12)
            assert not bad, (lim, step, bad)
        if lim == "LIMITED_NO":
            a, b = Oracle(case), Fvcom(case)
            a.run(20)
            b.run(20)
            bad = parity.compare(b, a, ["el", "ua", "va", "u", "v", "t1", "s1"], rtol=1e-10)
            assert not bad, (lim, bad)


@pytest.mark.parametrize("case_name", ["small_channel", "small_coastal"])
def test_staged_momentum_kernels_equal_per_cell_kernels(case_name, request):
    """ADVECTION_EDGE_GCN and ADV_UV_EDGE_GCN as tile-staged kernels (neighbours in shared
    memory, each edge evaluated once per tile) against the one-thread-per-cell kernels:
    bit for bit in FP64, and the routines against the oracle above run staged."""
    from myfvcomcode_b200.engine import Fvcom
    case = request.getfixturevalue(case_name)
    a, b = Fvcom(case), Fvcom(case)
    a.set_tuning("staged", 2)
    b.set_tuning("staged", 0)
    assert a.get_tuning("staged") == 2 and b.get_tuning("staged") == 0
    a.run(4)
    b.run(4)
    for n in ("el", "ua", "u", "v", "advx", "advy", "uf", "vf", "viscofm", "t1", "s1", "q2", "km"):
        assert np.array_equal(a.get(n), b.get(n)), n
