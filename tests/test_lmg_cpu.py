"""The learned preconditioner's oracle (oracle/cnn.py) checked against finite
differences on the CPU: the exact (FP64, unrounded) network's analytic
gradient must match central differences of its loss."""
import numpy as np
import pytest

from oracle import cnn as ref


def small_problem(n=2, h=16, w=16, seed=3):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, h + 2, w + 2))
    e = np.zeros_like(r)
    r[:, 1:-1, 1:-1] = rng.standard_normal((n, h, w))
    e[:, 1:-1, 1:-1] = rng.standard_normal((n, h, w))
    Kx = np.zeros_like(r)
    Ky = np.zeros_like(r)
    Kx[:, 1:-1, 2:-1] = rng.uniform(0.01, 5.0, (n, h, w - 1))
    Ky[:, 2:-1, 1:-1] = rng.uniform(0.01, 5.0, (n, h - 1, w))
    return r, Kx, Ky, e


@pytest.mark.parametrize("anorm", [False, True])
def test_oracle_gradient_matches_finite_differences(anorm):
    r, Kx, Ky, e = small_problem()
    p = ref.init_params(seed=1, out_scale=0.5).astype(np.float64)
    loss, g = ref.net_loss_grad(p, r, Kx, Ky, e, 30.0, 30.0, bf16=False, anorm=anorm)
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(p.size - 17, 24, replace=False), np.arange(p.size - 17, p.size)])
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = ref.net_loss_grad(pp, r, Kx, Ky, e, 30.0, 30.0, bf16=False, anorm=anorm)
        lm, _ = ref.net_loss_grad(pm, r, Kx, Ky, e, 30.0, 30.0, bf16=False, anorm=anorm)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])
    assert loss > 0


def test_untrained_output_is_jacobi():
    """With the output layer at zero, M(r) = r / diag(A)."""
    r, Kx, Ky, _ = small_problem()
    p = ref.init_params(seed=1, out_scale=0.0)
    M, A = ref.net_forward(p, r, Kx, Ky, 30.0, 30.0)
    np.testing.assert_allclose(M, A["z"], rtol=0, atol=0)
