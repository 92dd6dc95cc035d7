"""The FP64 oracle of the flux network, pinned on the CPU: its backward pass against
central finite differences of its own forward pass (exact arithmetic), and its BF16
rounding against torch's conversion."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo


@pytest.mark.parametrize("width,depth", [(128, 3), (64, 2), (32, 1)])
def test_oracle_gradient_matches_finite_differences(width, depth):
    rng = np.random.default_rng(3)
    shp = mo.shapes(width, depth)
    assert mo.shapes() == mo.SHAPES
    n = sum(k * m + m for k, m in shp)
    p = rng.normal(0, 0.2, n)
    x = rng.normal(0, 1, (4, 17))
    t = rng.normal(0, 1, (4, 8))
    loss, g = mo.loss_and_grad(p, x, t, bf16_rounding=False, shp=shp)
    assert g.size == n
    idx = rng.choice(n, 60, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_and_grad(pp, x, t, False, shp)[0] - mo.loss_and_grad(pm, x, t, False, shp)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(4)
    a = np.concatenate([rng.normal(0, 1, 5000), rng.normal(0, 1e-20, 100), [0.0, -0.0, 1.0, 3.0, 65504.0]])
    ref = torch.tensor(a.astype(np.float32)).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(mo.bf16(a), ref)


def test_adam_step_reference_values():
    p, g = np.array([1.0, -2.0]), np.array([0.5, -0.25])
    m, v = np.zeros(2), np.zeros(2)
    p1, m1, v1 = mo.adam_step(p, g, m, v, 1, lr=0.1)
    # first Adam step moves every parameter by lr against the sign of its gradient
    assert np.allclose(p1, p - 0.1 * np.sign(g), atol=1e-6)
