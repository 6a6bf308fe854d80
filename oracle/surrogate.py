"""TEST INFRASTRUCTURE ONLY (the checker, never the product).

A numpy FP64 restatement of the learned field the engine trains and runs on
the GPU (massccs_b200/csrc/field_device.cuh, field.cu).  The reference has
no learned field, so no reference file restates this; the model is the
published multiresolution hash encoding (Mueller et al., Instant-NGP, 2022)
feeding a two-hidden-layer ReLU MLP:

  encoding   per level l: a grid of resolution res_l = floor(base * g**l),
             g = (finest / base) ** (1 / (L - 1)), over the box [lo, hi];
             the 8 corners of the cell around x read a table of T rows of F
             features -- directly (x + r (y + r z), r = res_l + 1) while
             r**3 <= T, else through the spatial hash
             (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod T -- and are
             blended with smoothstep weights S(f) = f^2 (3 - 2 f) per axis
             (continuous first derivatives, so the forces of the field are
             continuous).  e(x): L * F features; J(x) = de/dx.
  MLP        z1 = W1 e + b1, a1 = relu(z1); z2 = W2 a1 + b2, a2 = relu(z2);
             u_f = s_f (w3_f . a2 + b3_f) for each output field f, s_f a fixed
             per-field output scale (the RMS of its labels).  The engine's
             fields are the smooth far parts of its range-separated forces:
             the far potential of each gas site type and, with the induced
             dipole, the three components of the far electric field.
  forces     F_f = -du_f/dx = -s_f J^T W1^T (m1 * W2^T (m2 * w3_f)), m = z > 0.
  loss       per sample, sum over fields of
               lam_u (u_f - U*_f)^2 / (U*_f^2 + u0_f^2) + |F_f - F*_f|^2 / (|F*_f|^2 + f0_f^2)
             (relative errors with per-field floors), averaged over the batch.  Its
             parameter gradients pass twice through the network (the force
             is itself a gradient): `loss_and_grad`.
  inference  `infer_bf16`: the arithmetic of the tensor-core path -- table
             and W1/W2 in bfloat16, the MMA inputs (features, hidden
             activations, back-propagated vectors) rounded to bfloat16,
             FP32-exact products summed in FP64 here.

Weights are stored [out][in] (row-major), as on the GPU.
"""
import numpy as np

PRIMES = (1, 2654435761, 805459861)


def bf16(a):
    """Round to bfloat16 (nearest even) and back to float64."""
    a = np.asarray(a, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


class HashGrid:
    def __init__(self, lo, hi, levels=16, log2_table=18, features=2, base=16, finest=2048, seed=0,
                 init=1e-4):
        self.lo = np.asarray(lo, dtype=np.float64)
        self.hi = np.asarray(hi, dtype=np.float64)
        self.L, self.T, self.F = levels, 1 << log2_table, features
        growth = np.exp((np.log(finest) - np.log(base)) / max(1, levels - 1))
        self.res = np.floor(base * growth ** np.arange(levels)).astype(np.int64)
        rng = np.random.default_rng(seed)
        self.table = rng.uniform(-init, init, size=(levels, self.T, features))

    def dense(self, level):
        r = int(self.res[level]) + 1
        return r ** 3 <= self.T

    def _index(self, level, c):
        """Table rows of integer corners c (n, 3) on a level."""
        r = self.res[level] + 1
        if self.dense(level):
            return c[:, 0] + r * (c[:, 1] + r * c[:, 2])
        h = (c[:, 0].astype(np.uint64) * np.uint64(PRIMES[0])) ^ \
            (c[:, 1].astype(np.uint64) * np.uint64(PRIMES[1])) ^ \
            (c[:, 2].astype(np.uint64) * np.uint64(PRIMES[2]))
        return ((h & np.uint64(0xFFFFFFFF)) % np.uint64(self.T)).astype(np.int64)

    def corners(self, x, level):
        """Per corner: rows (n, 8), weights (n, 8), weight gradients (n, 8, 3)."""
        scale = self.res[level] / (self.hi - self.lo)          # grid units per A
        p = np.clip((x - self.lo) * scale, 0.0, self.res[level])
        c0 = np.minimum(np.floor(p).astype(np.int64), self.res[level] - 1)
        f = p - c0
        S = f * f * (3.0 - 2.0 * f)
        dS = 6.0 * f * (1.0 - f) * scale
        rows, wts, dws = [], [], []
        for corner in range(8):
            o = np.array([(corner >> k) & 1 for k in range(3)])
            w3 = np.where(o == 1, S, 1.0 - S)
            d3 = np.where(o == 1, dS, -dS)
            rows.append(self._index(level, c0 + o))
            wts.append(w3.prod(axis=1))
            dws.append(np.stack([d3[:, 0] * w3[:, 1] * w3[:, 2], w3[:, 0] * d3[:, 1] * w3[:, 2],
                                 w3[:, 0] * w3[:, 1] * d3[:, 2]], axis=1))
        return np.stack(rows, 1), np.stack(wts, 1), np.stack(dws, 1)

    def encode(self, x, table=None):
        """x (n, 3) -> e (n, L*F), J (n, L*F, 3), per-level corner caches."""
        t = self.table if table is None else table
        x = np.atleast_2d(np.asarray(x, dtype=np.float64))
        n = x.shape[0]
        e = np.zeros((n, self.L * self.F))
        J = np.zeros((n, self.L * self.F, 3))
        cache = []
        for l in range(self.L):
            rows, w, dw = self.corners(x, l)
            val = t[l][rows]                                   # (n, 8, F)
            e[:, l * self.F:(l + 1) * self.F] = np.einsum("nc,ncf->nf", w, val)
            J[:, l * self.F:(l + 1) * self.F, :] = np.einsum("nca,ncf->nfa", dw, val)
            cache.append((rows, w, dw))
        return e, J, cache


class Field:
    """Hash-grid encoding + MLP with one potential output per field."""

    def __init__(self, lo, hi, hidden=64, outputs=2, scale=1.0, seed=0, **grid):
        """scale: one output scale for every field, or a sequence of nf."""
        self.grid = HashGrid(lo, hi, seed=seed, **grid)
        rng = np.random.default_rng(seed + 1)
        E = self.grid.L * self.grid.F
        self.W1 = rng.normal(0, np.sqrt(2.0 / E), size=(hidden, E))
        self.b1 = np.zeros(hidden)
        self.W2 = rng.normal(0, np.sqrt(2.0 / hidden), size=(hidden, hidden))
        self.b2 = np.zeros(hidden)
        self.W3 = rng.normal(0, np.sqrt(1.0 / hidden), size=(outputs, hidden))
        self.b3 = np.zeros(outputs)
        self.s = np.broadcast_to(np.asarray(scale, dtype=np.float64), (outputs,)).copy()

    # parameters as a flat MLP vector in the GPU's order: W1, b1, W2, b2, W3, b3
    def mlp_vector(self):
        return np.concatenate([self.W1.ravel(), self.b1, self.W2.ravel(), self.b2, self.W3.ravel(), self.b3])

    def set_mlp_vector(self, v):
        H, E = self.W1.shape
        nf = self.W3.shape[0]
        k = 0
        for name, shape in (("W1", (H, E)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (nf, H)),
                            ("b3", (nf,))):
            m = int(np.prod(shape))
            setattr(self, name, np.array(v[k:k + m], dtype=np.float64).reshape(shape))
            k += m

    def forward(self, x):
        """u (n, nf), F (n, nf, 3) and the intermediate state."""
        e, J, cache = self.grid.encode(x)
        z1 = e @ self.W1.T + self.b1
        m1 = z1 > 0
        a1 = np.where(m1, z1, 0.0)
        z2 = a1 @ self.W2.T + self.b2
        m2 = z2 > 0
        a2 = np.where(m2, z2, 0.0)
        u = self.s * (a2 @ self.W3.T + self.b3)
        g2 = m2[:, None, :] * self.W3[None, :, :]              # (n, nf, H)
        g1 = m1[:, None, :] * (g2 @ self.W2)                   # (n, nf, H): W2^T g2
        g0 = g1 @ self.W1                                      # (n, nf, E): W1^T g1
        F = -self.s[None, :, None] * np.einsum("nfe,nea->nfa", g0, J)
        st = dict(e=e, J=J, cache=cache, z1=z1, m1=m1, a1=a1, z2=z2, m2=m2, a2=a2, g2=g2, g1=g1, g0=g0)
        return u, F, st

    def loss_and_grad(self, x, U, Fs, lam_u=0.1, u0=0.05, f0=0.05):
        """Mean loss over the batch and its gradients: (loss, dtable, dmlp vector).
        U (n, nf), Fs (n, nf, 3) are the labels; u0, f0: floors (scalars or per field)."""
        n = x.shape[0]
        u, F, st = self.forward(x)
        u0 = np.asarray(u0, dtype=np.float64)
        f0 = np.asarray(f0, dtype=np.float64)
        wu = lam_u / (U * U + u0 * u0)                         # (n, nf)
        wf = 1.0 / ((Fs * Fs).sum(-1) + f0 * f0)               # (n, nf)
        du = u - U
        dF = F - Fs
        loss = float((wu * du * du + wf * (dF * dF).sum(-1)).sum() / n)
        s = self.s
        e, J, m1, a1, m2, a2, g2, g1, g0 = (st[k] for k in ("e", "J", "m1", "a1", "m2", "a2", "g2", "g1", "g0"))
        du_ = 2.0 * wu * du / n                                # dL/du (n, nf)
        eF = 2.0 * wf[..., None] * dF / n                      # dL/dF (n, nf, 3)
        # ---- potential path
        sd = du_ * s[None, :]
        dW3 = sd.T @ a2
        db3 = sd.sum(0)
        da2 = sd @ self.W3                                     # (n, H)
        dz2 = m2 * da2
        dW2 = dz2.T @ a1
        db2 = dz2.sum(0)
        dz1 = m1 * (dz2 @ self.W2)
        dW1 = dz1.T @ e
        db1 = dz1.sum(0)
        de = dz1 @ self.W1                                     # (n, E)
        # ---- force path: F_f = -s_f J^T g0_f
        r0 = -s[None, :, None] * np.einsum("nea,nfa->nfe", J, eF)  # dL/dg0 (n, nf, E)
        dJ = -np.einsum("nfe,nfa->nea", g0 * s[None, :, None], eF)  # dL/dJ (n, E, 3)
        dW1 += np.einsum("nfh,nfe->he", g1, r0)                # g0 = W1^T g1
        r1 = r0 @ self.W1.T                                    # dL/dg1 (n, nf, H)
        h = m1[:, None, :] * r1                                # through g1 = m1 * (W2^T g2)
        dW2 += np.einsum("nfo,nfi->oi", g2, h)
        r2 = h @ self.W2.T                                     # dL/dg2 (n, nf, H)
        dW3 += np.einsum("nh,nfh->fh", m2, r2)                 # g2 = m2 * w3_f
        # ---- table: e = sum_c w_c T[c], J = sum_c dw_c T[c]
        dt = np.zeros_like(self.grid.table)
        Fd = self.grid.F
        for l, (rows, w, dw) in enumerate(st["cache"]):
            ge = de[:, l * Fd:(l + 1) * Fd]                    # (n, F)
            gJ = dJ[:, l * Fd:(l + 1) * Fd, :]                 # (n, F, 3)
            contrib = w[:, :, None] * ge[:, None, :] + np.einsum("nca,nfa->ncf", dw, gJ)
            np.add.at(dt[l], rows.ravel(), contrib.reshape(-1, Fd))
        dmlp = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
        return loss, dt, dmlp

    def infer_bf16(self, x):
        """u (n, nf), F (n, nf, 3) in the tensor-core inference arithmetic."""
        e, J, _ = self.grid.encode(x, table=bf16(self.grid.table))
        W1, W2 = bf16(self.W1), bf16(self.W2)
        W3 = self.W3.astype(np.float32).astype(np.float64)
        A1 = bf16(e)
        z1 = A1 @ W1.T + self.b1
        m1 = z1 > 0
        A2 = bf16(np.where(m1, z1, 0.0))
        z2 = A2 @ W2.T + self.b2
        m2 = z2 > 0
        a2 = np.where(m2, z2, 0.0)
        u = self.s * (a2 @ W3.T + self.b3)
        G2 = bf16(m2[:, None, :] * W3[None, :, :])
        G1 = bf16(m1[:, None, :] * (G2 @ W2))
        g0 = G1 @ W1
        F = -self.s[None, :, None] * np.einsum("nfe,nea->nfa", g0, J)
        return u, F


def switch(r, r_in, r_out):
    """The range-separation weight of a pair at distance r: 1 below r_in, 0
    above r_out, the quintic smootherstep 1 - x^3 (10 - 15 x + 6 x^2) between
    (x = (r - r_in) / (r_out - r_in)), and its derivative d/dr."""
    x = np.clip((np.asarray(r, dtype=np.float64) - r_in) / (r_out - r_in), 0.0, 1.0)
    S = 1.0 - x ** 3 * (10.0 - 15.0 * x + 6.0 * x * x)
    dS = -30.0 * x * x * (1.0 - x) ** 2 / (r_out - r_in)
    return S, dS


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.99, eps=1e-15):
    """One Adam update in place (bias-corrected), as the GPU's optimiser kernel."""
    m *= b1
    m += (1 - b1) * g
    v *= b2
    v += (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    p -= lr * mh / (np.sqrt(vh) + eps)


KCOUL = 332.06348078020324


def field_layout(gas, coul_on, dip_on):
    """The engine's fields for a gas (ccs_gas numbering): a list of
    (kind, lj, q, comp) -- kind 0 the far potential of a site type with LJ
    parameter set lj (0 none, 1 primary, 2 carbon) and charge q, kind 1
    component comp of the far electric field -- and the field of each site
    and the dipole's site."""
    if gas == 2:    # N2: N, N, central charge
        fields = [(0, 1, -0.4825 if coul_on else 0.0, 0), (0, 0, 0.965 if coul_on else 0.0, 0)]
        site_field, dip = [0, 0, 1], (2 if dip_on else -1)
    elif gas == 3:  # CO2: O, C, O
        fields = [(0, 1, -0.3256 if coul_on else 0.0, 0), (0, 2, 0.6512 if coul_on else 0.0, 0)]
        site_field, dip = [0, 1, 0], (1 if dip_on else -1)
    else:
        fields = [(0, 1, 0.0, 0)]
        site_field, dip = [0], (0 if dip_on else -1)
    if dip >= 0:
        fields += [(1, 0, 0.0, a) for a in range(3)]
    return fields, site_field, dip


def far_fields(pts, xyz, q, ab, abc, fields, lj_cutoff, coul_cutoff, r_in, r_out, coul_on):
    """Far parts of the range-separated pair terms at points (n, 3): for each
    field its value and minus its gradient, (n, nf, 4).  Far weight 1 - S(r)
    (switch); LJ shifted at lj_cutoff (Force.cpp:83-102), Coulomb and the
    dipole's field in the shifted-force form within coul_cutoff
    (Force.cpp:671-683, 393-426).  ab / abc: (natoms, 2) pair coefficients
    A = 4 eps sig^12, B = 4 eps sig^6 of the primary and carbon sets."""
    pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
    out = np.zeros((len(pts), len(fields), 4))
    rl, rc = lj_cutoff, coul_cutoff
    rc6i, rc3i = 1.0 / rl ** 6, 1.0 / rc ** 3
    for i, p in enumerate(pts):
        d = p[None, :] - xyz
        r2 = (d * d).sum(1)
        r = np.sqrt(r2)
        S, dS = switch(r, r_in, r_out)
        wf, dsr = 1.0 - S, dS / r
        in_lj, in_c = r2 < rl * rl, r2 < rc * rc
        ir2 = 1.0 / r2
        ir6 = ir2 ** 3
        for f, (kind, lj, qs, comp) in enumerate(fields):
            if kind == 0:
                u = np.zeros_like(r)
                fs = np.zeros_like(r)
                if lj:
                    A, B = (ab if lj == 1 else abc).T
                    u += np.where(in_lj, ir6 * (A * ir6 - B) - (A * rc6i * rc6i - B * rc6i), 0.0)
                    fs += np.where(in_lj, ir6 * (12 * A * ir6 - 6 * B) * ir2, 0.0)
                if qs != 0.0 and coul_on:
                    kq = KCOUL * qs * q
                    u += np.where(in_c, kq * (1 / r - 1.5 / rc + 0.5 * r2 * rc3i), 0.0)
                    fs += np.where(in_c, kq * (1 / r ** 3 - rc3i), 0.0)
                fsc = wf * fs + u * dsr
                out[i, f, 0] = (wf * u).sum()
                out[i, f, 1:] = (fsc[:, None] * d).sum(0)
            else:
                sq = np.where(in_c, q * (1 / r ** 3 - rc3i), 0.0)
                tq = np.where(in_c, -3 * q / r ** 5, 0.0)
                da = d[:, comp]
                out[i, f, 0] = (wf * sq * da).sum()
                t2 = wf * tq * da - sq * da * dsr
                g = (t2[:, None] * d).sum(0)
                g[comp] += (wf * sq).sum()
                out[i, f, 1:] = -g
    return out
