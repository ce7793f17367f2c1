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
