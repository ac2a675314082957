"""NetCDF-3 history and restart files (myfvcomcode_b200/ncio.py).

CPU (oracle): a run stopped after 3 internal steps, written to a restart file, read into
a fresh model and continued for 2 steps equals the 5-step run bit for bit; the history
file carries FVCOM's variable names, units and the model's values.
GPU: the same restart round trip on the CUDA library.
"""
import numpy as np
import pytest
from scipy.io import netcdf_file

from myfvcomcode_b200 import ncio

CHECK = ("el", "ua", "u", "v", "t1", "s1", "q2", "q2l", "km", "kh", "w", "rho1", "iswetn")


def _roundtrip(make, tmp_path):
    a = make()
    a.run(5)
    b = make()
    b.run(3)
    path = str(tmp_path / "restart.nc")
    ncio.write_restart(path, b)
    c = make()
    ncio.read_restart(path, c)
    c.run(2)
    assert c.clock() == a.clock()
    for f in CHECK:
        assert np.array_equal(a.get(f), c.get(f)), f


def test_restart_continues_bitwise_on_oracle(small_coastal, tmp_path):
    from oracle.oracle import Oracle
    _roundtrip(lambda: Oracle(small_coastal), tmp_path)


def test_history_file_has_fvcom_names_and_values(small_channel, tmp_path):
    from oracle.oracle import Oracle
    o = Oracle(small_channel)
    path = str(tmp_path / "hist.nc")
    h = ncio.History(path, small_channel)
    o.run(2)
    h.write(o)
    o.run(1)
    h.write(o)
    h.close()
    nc = netcdf_file(path, "r", mmap=False)
    for name in ("x", "y", "xc", "yc", "nv", "h", "siglay", "siglev", "time", "zeta", "u", "v", "ww",
                 "ua", "va", "temp", "salinity", "km", "kh", "kq", "q2", "q2l"):
        assert name in nc.variables, name
    assert nc.variables["zeta"].units == b"meters"
    assert nc.variables["temp"].long_name == b"temperature"
    assert nc.variables["u"].shape == (2, o.KB - 1, o.N)
    assert np.allclose(nc.variables["zeta"][1], o.get("el")[1:].astype(np.float32))
    t1 = o.get3("t1")[1:, :-1].T
    assert np.allclose(nc.variables["temp"][1], t1.astype(np.float32))
    assert list(nc.variables["iint"][:]) == [2, 3]
    nc.close()


@pytest.mark.gpu
def test_restart_continues_bitwise_on_gpu(small_coastal, tmp_path):
    from myfvcomcode_b200.engine import Fvcom
    _roundtrip(lambda: Fvcom(small_coastal), tmp_path)
