"""The learned field's CPU restatement (oracle/surrogate.py), the reference
the GPU training and inference kernels will be checked against (CPU).

Bars: parameter and position gradients against central differences to 1e-6
relative (FP64); hashed rows inside the table; a short Adam fit of a smooth
potential lowers the loss tenfold.
"""
import numpy as np
import pytest


def _field(seed=0):
    from oracle.surrogate import Field
    return Field(lo=[-5, -5, -5], hi=[5, 5, 5], hidden=(16, 16), outputs=2, seed=seed,
                 levels=4, log2_table=8, features=2, base=4, finest=32)


def _loss(f, x, w):
    return float((f.forward(x) * w).sum())


def test_parameter_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    f = _field()
    f.grid.table = rng.normal(0, 0.5, size=f.grid.table.shape)  # away from the tiny initial values
    x = rng.uniform(-4.5, 4.5, size=(24, 3))
    w = rng.normal(size=(24, 2))
    f.forward(x)
    gW, gb, gt, _ = f.backward(w)
    h = 1e-6
    checks = [(f.W[0], gW[0], (3, 5)), (f.W[1], gW[1], (2, 7)), (f.W[2], gW[2], (4, 1)), (f.b[1], gb[1], (3,))]
    used = np.argwhere(np.abs(gt) > 1e-3)
    for i in rng.choice(len(used), 4, replace=False):
        checks.append((f.grid.table, gt, tuple(used[i])))
    for arr, grad, idx in checks:
        old = arr[idx]
        arr[idx] = old + h
        up = _loss(f, x, w)
        arr[idx] = old - h
        dn = _loss(f, x, w)
        arr[idx] = old
        fd = (up - dn) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, grad[idx])


def test_position_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    f = _field(seed=3)
    f.grid.table = rng.normal(0, 0.5, size=f.grid.table.shape)
    x = rng.uniform(-4.0, 4.0, size=(10, 3))
    g = f.position_grad(x)
    h = 1e-6
    for a in range(3):
        xp, xm = x.copy(), x.copy()
        xp[:, a] += h
        xm[:, a] -= h
        fd = (f.forward(xp) - f.forward(xm)) / (2 * h)
        np.testing.assert_allclose(g[:, :, a], fd, rtol=1e-6, atol=1e-6)


def test_hashed_rows_stay_in_the_table():
    from oracle.surrogate import HashGrid
    g = HashGrid([-50] * 3, [50] * 3, levels=16, log2_table=18, features=2)
    x = np.random.default_rng(4).uniform(-50, 50, size=(256, 3))
    _, _, cache = g.encode(x)
    for rows, weights in cache:
        assert rows.min() >= 0 and rows.max() < g.T
        np.testing.assert_allclose(weights.sum(axis=1), 1.0, rtol=1e-12)


def test_adam_fit_of_a_smooth_potential():
    rng = np.random.default_rng(5)
    f = _field(seed=6)
    x = rng.uniform(-4.5, 4.5, size=(512, 3))
    r = np.linalg.norm(x, axis=1)
    target = np.stack([1.0 / (1.0 + r), np.cos(r)], 1)
    params = f.W + f.b + [f.grid.table]
    m = [np.zeros_like(p) for p in params]
    v = [np.zeros_like(p) for p in params]
    lr, b1, b2 = 1e-2, 0.9, 0.99
    losses = []
    for step in range(1, 301):
        y = f.forward(x)
        d = y - target
        losses.append(float((d * d).mean()))
        gW, gb, gt, _ = f.backward(2 * d / d.size)
        for k, (p, g) in enumerate(zip(params, gW + gb + [gt])):
            m[k] = b1 * m[k] + (1 - b1) * g
            v[k] = b2 * v[k] + (1 - b2) * g * g
            p -= lr * (m[k] / (1 - b1 ** step)) / (np.sqrt(v[k] / (1 - b2 ** step)) + 1e-12)
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])
