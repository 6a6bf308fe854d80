"""TEST INFRASTRUCTURE ONLY (the checker, never the product).

A numpy restatement of the learned field the engine's fifth configuration
calls for: a multiresolution hash-grid encoding of the probe position (the
published Instant-NGP encoding: per level a grid of resolution
base * growth**l, the 8 corners of the cell around the point looked up
directly on coarse levels and through the spatial hash
(x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod T on fine ones, features
interpolated trilinearly) feeding a ReLU MLP whose outputs are the site
potentials.  Forces are minus the gradient of the potential with respect to
the position, through the MLP and the interpolation weights.

It gives the CUDA training and inference kernels their reference: the
forward pass, the parameter gradients of a squared loss (hash-table
gradients scatter-added), and the position gradient, all in FP64.  No
reference file restates this: the reference has no learned field.
"""
import numpy as np

PRIMES = (1, 2654435761, 805459861)


class HashGrid:
    def __init__(self, lo, hi, levels=16, log2_table=18, features=2, base=16, finest=2048, seed=0):
        self.lo = np.asarray(lo, dtype=np.float64)
        self.hi = np.asarray(hi, dtype=np.float64)
        self.L, self.T, self.F = levels, 1 << log2_table, features
        growth = np.exp((np.log(finest) - np.log(base)) / max(1, levels - 1))
        self.res = np.floor(base * growth ** np.arange(levels)).astype(np.int64)
        rng = np.random.default_rng(seed)
        self.table = rng.uniform(-1e-4, 1e-4, size=(levels, self.T, features))

    def _index(self, level, c):
        """Table rows of integer corners c (n, 3) on a level: direct on coarse levels."""
        r = self.res[level] + 1
        if r ** 3 <= self.T:
            return (c[:, 0] + r * (c[:, 1] + r * c[:, 2])) % self.T
        h = (c[:, 0].astype(np.uint64) * np.uint64(PRIMES[0])) ^ \
            (c[:, 1].astype(np.uint64) * np.uint64(PRIMES[1])) ^ \
            (c[:, 2].astype(np.uint64) * np.uint64(PRIMES[2]))
        return (h % np.uint64(self.T)).astype(np.int64)

    def _cells(self, x, level):
        u = (x - self.lo) / (self.hi - self.lo)          # unit cube
        p = np.clip(u, 0.0, 1.0) * self.res[level]
        c0 = np.minimum(np.floor(p).astype(np.int64), self.res[level] - 1)
        return p - c0, c0, self.res[level] / (self.hi - self.lo)  # fraction, corner, d(p)/d(x)

    def encode(self, x, want_grad=False):
        """x (n, 3) -> features (n, L*F); with want_grad also d(features)/dx (n, L*F, 3)
        and the corner rows and weights for the backward pass."""
        x = np.atleast_2d(np.asarray(x, dtype=np.float64))
        n = x.shape[0]
        out = np.zeros((n, self.L * self.F))
        dout = np.zeros((n, self.L * self.F, 3)) if want_grad else None
        cache = []
        for l in range(self.L):
            f, c0, dpdx = self._cells(x, l)
            rows, weights = [], []
            for corner in range(8):
                o = np.array([(corner >> k) & 1 for k in range(3)])
                w3 = np.where(o == 1, f, 1.0 - f)          # per-axis weights (n, 3)
                w = w3.prod(axis=1)
                idx = self._index(l, c0 + o)
                val = self.table[l, idx]                  # (n, F)
                out[:, l * self.F:(l + 1) * self.F] += w[:, None] * val
                if want_grad:
                    for a in range(3):
                        dw = np.where(o[a] == 1, 1.0, -1.0) * np.prod(np.delete(w3, a, axis=1), axis=1)
                        dout[:, l * self.F:(l + 1) * self.F, a] += (dw * dpdx[a])[:, None] * val
                rows.append(idx)
                weights.append(w)
            cache.append((np.stack(rows, 1), np.stack(weights, 1)))
        return out, dout, cache


class Field:
    """Hash-grid encoding + MLP (ReLU hidden layers, linear output)."""

    def __init__(self, lo, hi, hidden=(64, 64), outputs=1, seed=0, **grid):
        self.grid = HashGrid(lo, hi, seed=seed, **grid)
        rng = np.random.default_rng(seed + 1)
        dims = [self.grid.L * self.grid.F, *hidden, outputs]
        self.W = [rng.normal(0, np.sqrt(2.0 / a), size=(a, b)) for a, b in zip(dims[:-1], dims[1:])]
        self.b = [np.zeros(b) for b in dims[1:]]

    def forward(self, x):
        h, dh, cache = self.grid.encode(x, want_grad=True)
        acts, pre = [h], []
        for k, (W, b) in enumerate(zip(self.W, self.b)):
            z = acts[-1] @ W + b
            pre.append(z)
            acts.append(np.maximum(z, 0.0) if k < len(self.W) - 1 else z)
        self._state = (dh, cache, acts, pre)
        return acts[-1]

    def backward(self, dy):
        """Gradients of sum(dy * y) for the weights, biases and hash table."""
        dh, cache, acts, pre = self._state
        gW, gb = [None] * len(self.W), [None] * len(self.b)
        g = dy
        for k in range(len(self.W) - 1, -1, -1):
            if k < len(self.W) - 1:
                g = g * (pre[k] > 0)
            gW[k] = acts[k].T @ g
            gb[k] = g.sum(axis=0)
            g = g @ self.W[k].T
        gt = np.zeros_like(self.grid.table)
        F = self.grid.F
        for l, (rows, weights) in enumerate(cache):
            gl = g[:, l * F:(l + 1) * F]
            for corner in range(8):
                np.add.at(gt[l], rows[:, corner], weights[:, corner][:, None] * gl)
        return gW, gb, gt, g

    def position_grad(self, x):
        """d y / d x (n, outputs, 3): the force is minus this for a potential output."""
        y = self.forward(x)
        dh, cache, acts, pre = self._state
        out = np.zeros((y.shape[0], y.shape[1], 3))
        for j in range(y.shape[1]):
            g = np.zeros_like(y)
            g[:, j] = 1.0
            for k in range(len(self.W) - 1, -1, -1):
                if k < len(self.W) - 1:
                    g = g * (pre[k] > 0)
                g = g @ self.W[k].T
            out[:, j, :] = np.einsum("nf,nfa->na", g, dh)
        return out
