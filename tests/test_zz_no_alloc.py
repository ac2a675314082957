"""fvg_budget_fields (budgets from caller-owned device arrays, fixed-size device scratch,
no allocation) against fvg_budget on the same state, through the C ABI.

The file name sorts last so the test also runs after every other GPU test in a session.
"""
import ctypes as C

import numpy as np
import pytest

FVG_ERR_CAPACITY = 8
MAX_NODES = 4194304


def _bind(lib):
    f = lib.fvg_budget_fields
    f.argtypes = [C.c_void_p] * 5 + [C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_double)]
    f.restype = C.c_int
    return f


def _device_fields(gpu, case):
    import torch
    g = case["grid"]
    kbm1 = gpu.KB - 1

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda:0")

    d = dev(gpu.get("d"))
    art1 = dev(np.asarray(g["ART1"], dtype=np.float64))
    t1 = dev(gpu.get3("t1")[:, :kbm1].reshape(-1, order="F"))
    s1 = dev(gpu.get3("s1")[:, :kbm1].reshape(-1, order="F"))
    dz = dev(np.asarray(g["DZ"], dtype=np.float64)[:, :kbm1].reshape(-1, order="F"))
    return d, art1, t1, s1, dz


@pytest.mark.gpu
def test_budget_fields_matches_budget_twice(small_channel):
    import torch
    from myfvcomcode_b200.engine import Fvcom, load_library
    gpu = Fvcom(small_channel)
    gpu.run(3)
    ref = np.array(gpu.budget())
    fields = _device_fields(gpu, small_channel)
    f = _bind(load_library())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    got = []
    for _ in range(2):
        out = (C.c_double * 3)()
        rc = f(*[C.c_void_p(t.data_ptr()) for t in fields], gpu.M, gpu.KB - 1, stream, out)
        assert rc == 0
        got.append(np.array(out[:]))
    for g in got:
        np.testing.assert_allclose(g, ref, rtol=1e-12, atol=0.0)
    assert np.array_equal(got[0], got[1])
    gpu.close()


@pytest.mark.gpu
def test_budget_fields_rejects_mesh_beyond_scratch(small_channel):
    import torch
    from myfvcomcode_b200.engine import load_library
    f = _bind(load_library())
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = C.c_void_p(buf.data_ptr())
    out = (C.c_double * 3)(7.0, 7.0, 7.0)
    # Rejected on the host from the sizes alone; nothing is launched.
    assert f(p, p, p, p, p, MAX_NODES + 1, 10, None, out) == FVG_ERR_CAPACITY
    assert f(p, p, p, p, p, 8, 0, None, out) == 1
    assert list(out) == [7.0, 7.0, 7.0]
