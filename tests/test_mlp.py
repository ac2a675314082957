"""The learned closure's network: the CUDA training kernels' loss and gradient against
the float64 numpy restatement (oracle/mlp_oracle.py), which is itself checked against
central finite differences; the FP32 forward pass; and that training converges."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, mo.MI)).astype(np.float32)
    # a smooth target the network can represent
    y = np.stack([np.tanh(x[:, 0] - 0.5 * x[:, 1]), x[:, 2] * x[:, 3] * 0.3,
                  np.sin(x[:, 4]) + 0.1 * x[:, 7]], axis=1).astype(np.float32)
    return x, y


def _params(seed=1):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(mo.NPAR) * 0.2).astype(np.float32)


def test_oracle_gradient_matches_finite_differences():
    x, y = _data(5)
    p = _params().astype(np.float64)
    loss, g = mo.loss_grad(p, x, y)
    rng = np.random.default_rng(2)
    for q in rng.choice(mo.NPAR, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (mo.loss_grad(pp, x, y)[0] - mo.loss_grad(pm, x, y)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 + 1e-5 * abs(fd), q


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


@pytest.mark.gpu
def test_cuda_gradient_matches_oracle():
    from myfvcomcode_b200.engine import Mlp
    x, y = _data(300)  # several blocks of 64 and a partial block
    p = _params()
    net = Mlp(seed=0)
    net.set_params(p)
    dx, dy = _dev(x), _dev(y)
    loss, g = net.loss_grad(dx.data_ptr(), dy.data_ptr(), 300)
    loss_o, g_o = mo.loss_grad(p.astype(np.float64), x, y)
    assert abs(loss - loss_o) <= 1e-5 * loss_o
    scale = np.abs(g_o).max()
    assert np.abs(g - g_o).max() <= 2e-5 * scale
    net.close()


@pytest.mark.gpu
def test_cuda_forward_matches_oracle():
    from myfvcomcode_b200.engine import Mlp
    import torch
    x, _ = _data(1000, seed=4)
    p = _params(5)
    net = Mlp(seed=0)
    net.set_params(p)
    dx = _dev(x)
    out = torch.zeros((1000, 3), dtype=torch.float32, device="cuda:0")
    net.forward(dx.data_ptr(), 1000, out.data_ptr())
    ref, _ = mo.forward(p.astype(np.float64), x.astype(np.float64))
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())
    net.close()


@pytest.mark.gpu
def test_training_converges_and_is_deterministic():
    from myfvcomcode_b200.engine import Mlp
    x, y = _data(20000, seed=6)
    dx, dy = _dev(x), _dev(y)
    hists, params = [], []
    for _ in range(2):
        net = Mlp(seed=7)
        hists.append(net.train(dx.data_ptr(), dy.data_ptr(), 20000, epochs=8, batch=512, lr=2e-3, seed=9))
        params.append(net.params())
        net.close()
    h = hists[0]
    assert h[-1] < 0.1 * h[0]
    assert np.array_equal(hists[0], hists[1]) and np.array_equal(params[0], params[1])


@pytest.mark.gpu
def test_tensor_core_forward_matches_bf16_arithmetic():
    import ctypes as C
    import torch
    from myfvcomcode_b200.engine import Mlp
    n = 1000  # not a multiple of the 128-row tile
    x, _ = _data(n, seed=8)
    p = _params(9)
    net = Mlp(seed=0)
    net.set_params(p)
    dx = _dev(x)
    out = torch.zeros((n, 3), dtype=torch.float32, device="cuda:0")
    f = net.lib.fvg_mlp_forward_bf16
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    assert f(net.h, dx.data_ptr(), n, out.data_ptr()) == 0
    got = out.cpu().numpy().astype(np.float64)
    emu = mo.forward_bf16(p.astype(np.float64), x.astype(np.float64))
    ref, _ = mo.forward(p.astype(np.float64), x.astype(np.float64))
    scale = np.abs(ref).max()
    # same arithmetic up to FP32 summation order and rounding of the activations
    assert np.abs(got - emu).max() <= 2e-2 * scale
    assert np.sqrt(np.mean((got - emu) ** 2)) <= 2e-3 * scale
    # and within BF16 noise of the FP32 network
    assert np.sqrt(np.mean((got - ref) ** 2)) <= 2e-2 * scale
    net.close()
