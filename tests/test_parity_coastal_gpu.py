"""Parity on the benchmarked configuration's own generator, on a B200.

The bench times the large coastal mesh: a seeded Delaunay triangulation of jittered
points in 200 km x 100 km, Gaussian-random-field bathymetry with a 2 m intertidal strip,
wetting and drying, M2+S2 open-boundary tide, 10 m/s wind, 40 sigma layers.  These tests
run the same generator at 60,000 points (about 119,000 cells, every feature of the
200,000-point mesh: high-valence nodes, wet/dry fronts, open-boundary corners) so that the
oracle finishes in seconds:

* every reference routine from the oracle's state after two internal steps, bit for bit
  (1e-13 relative where the device evaluates a transcendental), as on the small meshes;
* three internal steps of the plain FP64 library against the oracle from the same cold
  start: zeta, the 2-D and 3-D velocities, w, T, S, q2, q2l, KM, KH within 1e-12 of each
  field's maximum, and the wet/dry flags equal.  Both measures of ``parity.errors`` are
  reported in the failure message.
"""
import numpy as np
import pytest

from tests import parity
from tests.test_parity_gpu import routine_failures

pytestmark = pytest.mark.gpu

FIELDS = ["el", "ua", "va", "u", "v", "w", "t1", "s1", "q2", "q2l", "km", "kh", "d1", "wts"]


@pytest.fixture(scope="module")
def coastal60k():
    from myfvcomcode_b200 import cases
    return cases.coastal_mesh(npts=60000, kb=41, seed=1234)


def test_routines_match_oracle_on_coastal_60k(coastal60k):
    failures = routine_failures(coastal60k, 2)
    assert not failures, failures


def test_three_internal_steps_match_oracle_on_coastal_60k(coastal60k):
    from myfvcomcode_b200.engine import Fvcom
    from oracle.oracle import Oracle
    ora = Oracle(coastal60k)
    gpu = Fvcom(coastal60k)
    ora.run(3)
    gpu.run(3)
    errs = parity.errors(gpu, ora, FIELDS)
    bad = {n: e for n, e in errs.items() if not e["max_norm"] <= 1e-12}
    assert not bad, errs
    for n in ("iswetn", "iswetc", "iswetnt", "iswetct"):
        assert np.array_equal(gpu.get(n), ora.get(n)), n
    assert gpu.clock() == ora.clock()
    gpu.close()
