"""Batched ensembles: union models of perturbed members and groups of models.

CPU: the union model built by ensemble.union_case, run on the oracle, reproduces every
member run alone bit for bit (the union only renumbers; each gather stays in its member).
GPU: the same on the CUDA library, and a group of models stepped by one graph per step
equals the models stepped one by one.
"""
import numpy as np
import pytest

FIELDS = ("el", "ua", "u", "v", "t1", "s1", "q2", "km")


def _specs(n, seed=3):
    from myfvcomcode_b200 import ensemble
    return ensemble.perturbed_members(None, n, seed=seed)


def test_member_perturbations_are_seeded_and_bounded():
    from myfvcomcode_b200 import ensemble
    a = ensemble.perturbed_members(None, 64, seed=11)
    b = ensemble.perturbed_members(None, 64, seed=11)
    assert a == b
    assert all(0.8 <= s["wind_scale"] <= 1.2 and 0.9 <= s["tide_scale"] <= 1.1 for s in a)
    assert abs(np.std([s["t_offset"] for s in a]) - 0.5) < 0.15


def test_union_on_oracle_equals_members_alone(small_coastal):
    from myfvcomcode_b200 import ensemble
    from oracle.oracle import Oracle
    specs = _specs(2)
    u = ensemble.union_case(small_coastal, specs)
    assert u["grid"]["M"] == 2 * small_coastal["grid"]["M"]
    ou = Oracle(u)
    ou.run(3)
    for m, sp in enumerate(specs):
        om = Oracle(ensemble.member_case(small_coastal, sp))
        om.run(3)
        for f in FIELDS:
            assert np.array_equal(ensemble.member_slice(u, m, f, ou), om.get(f)), (m, f)
        om.close()
    ou.close()


@pytest.mark.gpu
def test_union_on_gpu_equals_members_alone(small_channel):
    from myfvcomcode_b200 import ensemble
    from myfvcomcode_b200.engine import Fvcom
    specs = _specs(3, seed=5)
    u = ensemble.union_case(small_channel, specs)
    fu = Fvcom(u)
    fu.run(4)
    for m, sp in enumerate(specs):
        fm = Fvcom(ensemble.member_case(small_channel, sp))
        fm.run(4)
        for f in FIELDS:
            assert np.array_equal(ensemble.member_slice(u, m, f, fu), fm.get(f)), (m, f)
        fm.close()


@pytest.mark.gpu
def test_group_equals_models_alone(small_channel, small_coastal):
    from myfvcomcode_b200.engine import Fvcom, Group
    a, b = Fvcom(small_channel), Fvcom(small_coastal)
    b.set_precision("fp32flux")
    ga, gb = Fvcom(small_channel), Fvcom(small_coastal)
    gb.set_precision("fp32flux")
    grp = Group([ga, gb])
    grp.run(5)
    a.run(5)
    b.run(5)
    for f in FIELDS:
        assert np.array_equal(ga.get(f), a.get(f)), f
        assert np.array_equal(gb.get(f), b.get(f)), f
    assert ga.clock() == a.clock()
    assert grp.time_steps(2) > 0.0
    grp.close()
