"""Tensor-core surrogate MLP against the numpy reference (oracle/mlp_ref.py),
which rounds inputs, weights and hidden activations to bf16 at the same points
as the kernels and accumulates in f64."""
import numpy as np
import pytest

import mlp_ref as R
from _gpu_util import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 70000])
def test_forward_matches_reference(n):
    import torch

    from agimp.surrogate import MLP
    rng = np.random.default_rng(n)
    P = R.init_params(rng).astype(np.float32)
    X = rng.normal(0, 1, (n, R.IN)).astype(np.float32)
    m = MLP(params=P)
    Y = m.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    assert m.errors() == 0
    ref, _ = R.forward(P, X)
    scale = np.abs(ref).max()
    # bf16 rounding of hidden activations may differ by one ulp (2^-8 relative)
    # where the kernels' exp differs from numpy's in the last bits
    assert np.abs(Y - ref).max() <= 1e-2 * scale + 1e-3, np.abs(Y - ref).max()
    assert np.median(np.abs(Y - ref)) <= 1e-4 * scale + 1e-6
    m.close()


def _grad_gpu(m, X, T):
    import ctypes

    import torch
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    g = torch.zeros(R.NPARAM, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert m._L.agimp_mlp_grad(m._h, ctypes.c_void_p(Xd.data_ptr()), ctypes.c_void_p(Td.data_ptr()), len(X),
                               ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(loss.data_ptr()), st) == 0
    torch.cuda.synchronize()
    return float(loss.item()), g.cpu().numpy()


@pytest.mark.parametrize("n", [100, 128, 5000, 200000])
def test_gradient_matches_oracle(n):
    """Loss and every parameter block's gradient against the numpy backward
    pass with the same bf16 rounding points (relative Frobenius error)."""
    from agimp.surrogate import MLP
    rng = np.random.default_rng(10 + n)
    P = R.init_params(rng).astype(np.float32)
    X = rng.normal(0, 1, (n, R.IN)).astype(np.float32)
    T = rng.normal(0, 1, (n, R.OUT)).astype(np.float32)
    m = MLP(params=P)
    loss, g = _grad_gpu(m, X, T)
    assert m.errors() == 0
    lref, gref = R.loss_and_grad(P, X, T)
    assert abs(loss - lref) <= 2e-3 * abs(lref)
    o = 0
    for name, shape in R.SIZES:
        k = int(np.prod(shape))
        a, b = g[o:o + k], gref[o:o + k]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 1e-2, (name, rel)
        o += k
    m.close()


def test_training_reduces_loss():
    """Adam steps on the tensor-core gradient fit a smooth 7 -> 4 map."""
    import ctypes

    import torch

    from agimp.surrogate import MLP
    rng = np.random.default_rng(0)
    n = 65536
    X = rng.uniform(-1, 1, (n, R.IN)).astype(np.float32)
    T = np.stack([np.tanh(X[:, 0] + 0.5 * X[:, 1]), X[:, 2] * X[:, 3], np.sin(X[:, 4]), X[:, 5] - X[:, 6]], 1)
    T = T.astype(np.float32)
    m = MLP(seed=1)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    hist = []
    for it in range(300):
        assert m._L.agimp_mlp_train_step(m._h, ctypes.c_void_p(Xd.data_ptr()), ctypes.c_void_p(Td.data_ptr()), n,
                                         ctypes.c_float(3e-3), ctypes.c_void_p(loss.data_ptr()), st) == 0
        if it % 50 == 0 or it == 299:
            hist.append(float(loss.item()))
    assert m.errors() == 0
    assert hist[-1] < 0.05 * hist[0], hist
    m.close()
