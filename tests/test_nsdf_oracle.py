"""CPU checks of the neural-SDF oracle itself (no GPU)."""
import numpy as np

from oracle import nsdf_oracle as no

BOX = ([-10.0, -6.0, -20.0], [10.0, 11.0, 30.0])


def _params(seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.15, no.NUM_PARAMS)
    return p


def test_softplus_fit_is_accurate():
    x = np.linspace(-20, 20, 4001)
    ref = np.logaddexp(0.0, x)
    assert np.abs(no.softplus(x) - ref).max() < 3e-6
    sig = 1 / (1 + np.exp(-x))
    assert np.abs(no.softplus_deriv(x) - sig).max() < 2e-4


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _params(1)
    pts = np.stack([rng.uniform(BOX[0][k], BOX[1][k], 64) for k in range(3)], 1)
    labels = rng.normal(0, 1, 64)
    loss, grad, _ = no.loss_grad(p, pts, labels, *BOX, 0.5, bf16_round=False)
    idx = np.concatenate([rng.choice(no.NUM_PARAMS - 1, 60, replace=False), [no.OFF_B5]])
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _, _ = no.loss_grad(q, pts, labels, *BOX, 0.5, bf16_round=False)
        q[i] -= 2 * eps
        lm, _, _ = no.loss_grad(q, pts, labels, *BOX, 0.5, bf16_round=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(grad[i]), (i, fd, grad[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0])
    r = no.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[4] == 0.0
    assert abs(r[3] - -3.140625) < 1e-9


def test_adam_step_moves_against_gradient():
    p = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    q, m, v = no.adam(p, g, np.zeros(4), np.zeros(4), 1, 1e-3)
    assert np.allclose(q, -1e-3 * np.sign(g), atol=1e-9)
