"""The coordinate MLP's hand-written kernels (BF16 tensor-core GEMMs with
FP32 accumulation) against the FP64 restatement (oracle/mlp_ref.py):
forward values and gradients, and a training run that fits a surface."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, size=(n, 8)).astype(np.float32)
    t = (np.sin(2 * x[:, 0]) * np.cos(3 * x[:, 1]) + 0.3 * x[:, 4]).astype(np.float32)
    return x, t


@pytest.mark.parametrize("n", [1, 37, 1000, 5000])
def test_gradients_match_fp64(n):
    from randomtilings_b200.mlp import CoordinateMLP

    m = CoordinateMLP(seed=3)
    x, t = _batch(n, n)
    loss, g = m.loss_grad(x, t)
    p = m.params
    rloss, rg, ry = mlp_ref.loss_grad(p, x, t)
    y = m.predict(x)
    # tolerances: FP32 accumulation in a different order; BF16 storage is emulated by the restatement
    assert np.allclose(y, ry, rtol=2e-3, atol=2e-3)
    assert abs(loss - rloss) <= 2e-3 * max(1.0, rloss)
    at = 0
    for name, shape in mlp_ref.SIZES:
        k = int(np.prod(shape))
        a, b = g[at:at + k].astype(np.float64), rg[at:at + k]
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b) + 1e-6, name
        at += k
    # and against the un-rounded FP64 model the gradient is still close (BF16 storage only)
    _, fg, _ = mlp_ref.loss_grad(p, x, t, bf16_like_gpu=False)
    assert np.linalg.norm(g - fg) <= 5e-2 * np.linalg.norm(fg)


def test_training_fits_a_surface():
    from randomtilings_b200.mlp import CoordinateMLP

    m = CoordinateMLP(seed=1)
    x, t = _batch(200000, 7)
    m.set_data(x, t)
    xv, tv = _batch(4096, 8)
    before = float(np.mean((m.predict(xv) - tv) ** 2))
    m.train(400, batch=8192, lr=2e-3, seed=5)
    after = float(np.mean((m.predict(xv) - tv) ** 2))
    assert after < before / 20, (before, after)
