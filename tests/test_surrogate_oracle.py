"""The learned field's CPU restatement (oracle/surrogate.py), the reference
the GPU training and inference kernels are checked against (CPU).

Bars: forces against central differences of the potential to 1e-6 relative;
every parameter gradient of the force-matching loss (it passes twice through
the network) against central differences to 1e-6 relative (FP64); the
bfloat16 inference arithmetic within a few per cent of FP64; a short Adam
fit of a smooth potential lowers the loss tenfold.
"""
import numpy as np


def _field(seed=0, outputs=2):
    from oracle.surrogate import Field
    f = Field(lo=[-5, -5, -5], hi=[5, 5, 5], hidden=16, outputs=outputs, scale=(0.7, 2.0)[:outputs], seed=seed,
              levels=4, log2_table=8, features=2, base=4, finest=32)
    rng = np.random.default_rng(seed + 10)
    f.grid.table = rng.normal(0, 0.5, size=f.grid.table.shape)  # away from the tiny initial values
    f.b1 = rng.normal(0, 0.1, size=f.b1.shape)
    f.b2 = rng.normal(0, 0.1, size=f.b2.shape)
    return f


def test_levels_dense_then_hashed():
    f = _field()
    assert f.grid.dense(0) and not f.grid.dense(3)
    rng = np.random.default_rng(0)
    x = rng.uniform(-5, 5, size=(200, 3))
    for l in range(f.grid.L):
        rows, w, _ = f.grid.corners(x, l)
        assert rows.min() >= 0 and rows.max() < f.grid.T
        np.testing.assert_allclose(w.sum(1), 1.0, rtol=1e-12)


def test_forces_are_minus_the_potential_gradient():
    rng = np.random.default_rng(2)
    f = _field(seed=3)
    x = rng.uniform(-4.0, 4.0, size=(12, 3))
    _, F, _ = f.forward(x)
    h = 1e-6
    for a in range(3):
        d = np.zeros(3)
        d[a] = h
        up, _, _ = f.forward(x + d)
        dn, _, _ = f.forward(x - d)
        fd = -(up - dn) / (2 * h)
        np.testing.assert_allclose(F[:, :, a], fd, rtol=1e-6, atol=1e-7)


def test_loss_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    f = _field()
    x = rng.uniform(-4.5, 4.5, size=(20, 3))
    U = rng.normal(size=(20, 2))
    Fs = rng.normal(size=(20, 2, 3))
    loss, dt, dmlp = f.loss_and_grad(x, U, Fs)
    v = f.mlp_vector()
    h = 1e-6

    def loss_at():
        return f.loss_and_grad(x, U, Fs)[0]

    idx = rng.choice(len(v), 40, replace=False)
    for i in idx:
        old = v[i]
        v[i] = old + h
        f.set_mlp_vector(v)
        up = loss_at()
        v[i] = old - h
        f.set_mlp_vector(v)
        dn = loss_at()
        v[i] = old
        f.set_mlp_vector(v)
        fd = (up - dn) / (2 * h)
        assert abs(fd - dmlp[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, dmlp[i])
    used = np.argwhere(np.abs(dt) > 1e-4)
    for k in rng.choice(len(used), 12, replace=False):
        t = tuple(used[k])
        old = f.grid.table[t]
        f.grid.table[t] = old + h
        up = loss_at()
        f.grid.table[t] = old - h
        dn = loss_at()
        f.grid.table[t] = old
        fd = (up - dn) / (2 * h)
        assert abs(fd - dt[t]) <= 1e-6 * max(1.0, abs(fd)), (t, fd, dt[t])


def test_bf16_inference_is_close_to_fp64():
    rng = np.random.default_rng(4)
    f = _field(seed=5)
    x = rng.uniform(-4.0, 4.0, size=(400, 3))
    u, F, _ = f.forward(x)
    ub, Fb = f.infer_bf16(x)
    assert np.abs(ub - u).max() <= 0.03 * np.abs(u).max()
    assert np.linalg.norm(Fb - F, axis=-1).mean() <= 0.03 * np.linalg.norm(F, axis=-1).mean()


def test_adam_fit_lowers_the_loss():
    from oracle.surrogate import Field, adam_step
    rng = np.random.default_rng(6)
    f = Field(lo=[-5, -5, -5], hi=[5, 5, 5], hidden=16, outputs=1, scale=1.0, seed=7,
              levels=4, log2_table=10, features=2, base=4, finest=32)
    x = rng.uniform(-4.0, 4.0, size=(512, 3))
    r2 = (x * x).sum(1, keepdims=True)
    U = np.exp(-r2 / 8.0)
    Fs = (x / 4.0 * U)[:, None, :]
    tm, tv = np.zeros_like(f.grid.table), np.zeros_like(f.grid.table)
    v = f.mlp_vector()
    mv, vv = np.zeros_like(v), np.zeros_like(v)
    first = None
    for t in range(1, 301):
        loss, dt, dm = f.loss_and_grad(x, U, Fs, lam_u=1.0, u0=0.1, f0=0.1)
        first = loss if first is None else first
        adam_step(f.grid.table, dt, tm, tv, t, 1e-2)
        adam_step(v, dm, mv, vv, t, 1e-2)
        f.set_mlp_vector(v)
    assert loss < 0.1 * first, (first, loss)


def test_far_fields_are_minus_their_gradients():
    """The far parts of the range-separated pair terms (the training labels):
    every field's second entry is minus the gradient of its value."""
    from oracle.surrogate import far_fields, field_layout
    rng = np.random.default_rng(8)
    xyz = rng.normal(size=(60, 3)) * 4
    q = rng.normal(size=60) * 0.3
    ab = np.tile([4 * 0.1 * 3.3 ** 12, 4 * 0.1 * 3.3 ** 6], (60, 1))
    for gas in (2, 3, 1):
        fields, _, _ = field_layout(gas, True, True)
        args = (xyz, q, ab, ab * 1.1, fields, 12.0, 25.0, 6.0, 8.0, True)
        for p in (np.array([[9.0, 1.0, -2.0]]), np.array([[0.5, 7.1, 3.0]])):
            o = far_fields(p, *args)
            h = 1e-5
            for a in range(3):
                fd = (far_fields(p + h * np.eye(3)[a], *args)[0, :, 0] - far_fields(p - h * np.eye(3)[a], *args)[0, :, 0]) / (2 * h)
                np.testing.assert_allclose(o[0, :, 1 + a], -fd, rtol=1e-6, atol=1e-9)
