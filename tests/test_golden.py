"""The frozen fixture tests/golden/channel_100x20_k10_1000ext.npz (made by
tests/golden/make_golden.py from the oracle): the full estuary channel, 100 x 20 grid,
10 layers, after 100 internal steps = 1000 external steps from cold start.

* CPU: the oracle reproduces the fixture bit for bit (sha256 of el, u, v, t1, s1).
* GPU: the CUDA library, run the same 1000 external steps, matches the fixture within the
  parity tolerance of 1e-9 relative (to each field's maximum magnitude) in zeta, u, v, T, S.
"""
import os

import numpy as np
import pytest

from tests.golden import make_golden as mg

RTOL = 1e-9


def _fixture():
    return dict(np.load(mg.FIXTURE))


def test_oracle_reproduces_golden_bitwise():
    from oracle.oracle import Oracle
    fx = _fixture()
    ora = Oracle(mg.case())
    ora.run(mg.INTERNAL_STEPS)
    got = mg.summarize(ora)
    assert str(got["sha256"]) == str(fx["sha256"])
    for f in mg.SAMPLED:
        assert np.array_equal(got[f + "_val"], fx[f + "_val"])
    ora.close()


def test_golden_fixture_is_physical():
    fx = _fixture()
    el = fx["el"][1:]
    assert np.all(np.isfinite(el)) and 0.05 < np.abs(el).max() < 2.0
    assert np.all((fx["s1_val"] >= -1e-9) & (fx["s1_val"] <= 30.0 + 1e-9))
    assert np.all(np.abs(fx["t1_val"] - 15.0) < 1e-6)


@pytest.mark.gpu
def test_library_matches_golden():
    from myfvcomcode_b200.engine import Fvcom
    fx = _fixture()
    gpu = Fvcom(mg.case())
    gpu.run(mg.INTERNAL_STEPS)
    el = gpu.get("el")
    scale = np.abs(fx["el"]).max()
    assert np.abs(el - fx["el"]).max() <= RTOL * scale
    for f in mg.SAMPLED:
        a = gpu.get3(f)[1:, : gpu.KB - 1].reshape(-1, order="F")[fx[f + "_idx"]]
        b = fx[f + "_val"]
        scale = max(np.abs(b).max(), 1e-30)
        assert np.abs(a - b).max() <= RTOL * scale, f
    gpu.close()
