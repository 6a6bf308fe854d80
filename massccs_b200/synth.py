"""Seeded synthetic targets for the benchmark configurations.

No public benchmark suite is involved; these generators stand in for the
configurations the engine is measured on (sizes and distributions as stated):

  c60_he     60 C on a truncated icosahedron (C-C 1.40 A, centred), neutral,
             uff.ff carbon parameters, He, all cutoff/long-range/dipole flags
             on (force type 4), 3e5 trajectories.
  globule_n2 1231 atoms uniform in a sphere of radius Rg*sqrt(5/3) = 14.85 A
             (Rg 11.5 A) with a 1.0 A minimum pair distance, elements
             C .32 / H .50 / N .08 / O .09 / S .01, charges N(0, 0.3 e)
             shifted to a net +4 e, positions rounded to float32, default N2
             force field, N2, force type 6, 3e5 trajectories.
  shell      5e5 atoms uniform in the shell 100 A < r < 130 A with a 1.2 A
             minimum spacing, same element mix, charges N(0, 0.3 e) shifted to
             a net +40 e; He or N2; 1e6 trajectories.
  globule    N atoms, radius 1.3 N^(1/3) sqrt(5/3) A, net charge Q: the
             batched-ion and learned-field configurations.
  batch      256 globules, N log-uniform in [500, 50000], net charge a
             uniform integer in [0, 30] e, He, 2e4 trajectories each; the
             minimum distance is enforced by thinning a uniform sample with
             a k-d tree (fast_globule_atoms), not by sequential addition.
  field_globule  the learned-field configuration: 20,000 atoms (radius
             1.3 N^(1/3) sqrt(5/3) = 45.5 A, 1.0 A minimum spacing by k-d
             tree thinning), same element mix, charges N(0, 0.3 e) shifted
             to a net +12 e, default force field; N2 or CO2 (force type 6),
             1e6 trajectories.

Every generator writes `target.xyz` (5 columns: symbol x y z q), `uff.ff`
when used and `input.json` into a directory and returns the json path.
"""
import json
import os

import numpy as np

ELEMENTS = np.array(["C", "H", "N", "O", "S"])
FRACTIONS = np.array([0.32, 0.50, 0.08, 0.09, 0.01])

UFF_FF = """7
Symbol  mass (amu)  epislon (kcal/mol)  sigma(Angstroms)
C\t12.011\t0.10500\t3.43085
O\t15.9994\t0.06000\t3.11815
N\t14.0067\t0.06900\t3.26069
H\t1.008\t0.04400\t2.57113
S\t32.06\t0.27400\t3.59478
Na\t22.9897\t0.03000\t2.65755
K\t39.0983\t0.03500\t3.39611
"""

FLAGS = {  # force type -> (Short-range cutoff, Long-range forces, Long-range cutoff, polarizability)
    ("atom", 4): ("yes", "yes", "yes", "yes"),
    ("atom", 2): ("yes", "no", "yes", "no"),
    ("mol", 6): ("yes", "yes", "yes", "yes"),
    ("mol", 4): ("yes", "yes", "yes", "no"),
}


def truncated_icosahedron(edge=1.40):
    """The 60 vertices: even permutations of (0, +-1, +-3phi), (+-1, +-(2+phi), +-2phi),
    (+-phi, +-2, +-phi^3), which have edge length 2; scaled to `edge`."""
    phi = (1 + 5 ** 0.5) / 2
    base = [(0.0, 1.0, 3 * phi), (1.0, 2 + phi, 2 * phi), (phi, 2.0, phi ** 3)]
    pts = set()
    for b in base:
        for perm in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):  # even permutations
            v = [b[perm[0]], b[perm[1]], b[perm[2]]]
            for sx in (1, -1):
                for sy in (1, -1):
                    for sz in (1, -1):
                        w = (sx * v[0], sy * v[1], sz * v[2])
                        pts.add(tuple(round(c, 12) + 0.0 for c in w))
    p = np.array(sorted(pts)) * (edge / 2.0)
    assert p.shape == (60, 3)
    return p - p.mean(axis=0)


def _rsa(n, sample, dmin, rng, box_lo, box_hi, max_tries=200):
    """Random sequential addition with a minimum pair distance (cell grid)."""
    h = dmin
    dims = np.maximum(1, np.ceil((box_hi - box_lo) / h).astype(int))
    grid = {}
    out = np.empty((n, 3))
    k = 0
    tries = 0
    d2 = dmin * dmin
    while k < n:
        cand = sample(4096)
        for c in cand:
            tries += 1
            if tries > max_tries * n:
                raise RuntimeError("packing failed: lower the density or the minimum distance")
            ci = tuple(((c - box_lo) // h).astype(int))
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for j in grid.get((ci[0] + dx, ci[1] + dy, ci[2] + dz), ()):
                            e = out[j] - c
                            if e @ e < d2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                out[k] = c
                grid.setdefault(ci, []).append(k)
                k += 1
                if k == n:
                    break
    return out


def _charges(n, net, rng, sd=0.3):
    q = rng.normal(0.0, sd, n)
    return q + (net - q.sum()) / n


def _elements(n, rng):
    return ELEMENTS[rng.choice(len(ELEMENTS), size=n, p=FRACTIONS)]


def write_xyz(path, sym, xyz, q, float32=False):
    if float32:
        xyz = xyz.astype(np.float32).astype(np.float64)
    with open(path, "w") as f:
        f.write(f"{len(sym)}\nsynthetic target (massccs_b200.synth)\n")
        for s, (x, y, z), c in zip(sym, xyz, q):
            f.write(f"{s} {x:.9g} {y:.9g} {z:.9g} {c:.9g}\n")


def write_input(d, target, gas, ft, nprobe, niter, seed=2104, ff=None, extra=None, name="input.json"):
    kind = "mol" if gas in ("N2", "CO2") else "atom"
    fl = FLAGS[(kind, ft)]
    cfg = {"targetFileName": target, "numberProbe": int(nprobe), "nIter": int(niter), "seed": seed,
           "dt": 10.0, "Temp": 298.0, "skin": 0.01, "GasBuffer": gas, "Equipotential": "no",
           "Short-range cutoff": fl[0], "LJ-cutoff": 12.0, "Long-range forces": fl[1],
           "Long-range cutoff": fl[2], "Coul-cutoff": 25.0, "polarizability": fl[3]}
    if ff:
        cfg["force-field"] = ff
    if extra:
        cfg.update(extra)
    p = os.path.join(d, name)
    with open(p, "w") as f:
        json.dump(cfg, f, indent=1)
    return p


def c60_he(d, nprobe=30000, niter=10, seed=2104, **extra):
    os.makedirs(d, exist_ok=True)
    xyz = truncated_icosahedron(1.40)
    write_xyz(os.path.join(d, "target.xyz"), ["C"] * 60, xyz, np.zeros(60))
    with open(os.path.join(d, "uff.ff"), "w") as f:
        f.write(UFF_FF)
    return write_input(d, "target.xyz", "He", 4, nprobe, niter, seed, ff="uff.ff", extra=extra or None)


def globule_atoms(n, radius, net, rng, dmin=1.0):
    def sample(m):
        v = rng.normal(size=(m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        return v * radius * rng.random((m, 1)) ** (1 / 3)
    lo, hi = np.full(3, -radius - 1), np.full(3, radius + 1)
    xyz = _rsa(n, sample, dmin, rng, lo, hi)
    return _elements(n, rng), xyz, _charges(n, net, rng)


def globule_n2(d, nprobe=30000, niter=10, seed=2104, natoms=1231, rg=11.5, net=4.0, gen_seed=1231, **extra):
    os.makedirs(d, exist_ok=True)
    rng = np.random.default_rng(gen_seed)
    sym, xyz, q = globule_atoms(natoms, rg * (5 / 3) ** 0.5, net, rng)
    write_xyz(os.path.join(d, "target.xyz"), sym, xyz, q, float32=True)
    return write_input(d, "target.xyz", "N2", 6, nprobe, niter, seed, extra=extra or None)


def globule(d, natoms, net, gas="He", ft=None, nprobe=2000, niter=10, seed=2104, gen_seed=0, **extra):
    os.makedirs(d, exist_ok=True)
    rng = np.random.default_rng(gen_seed)
    radius = 1.3 * natoms ** (1 / 3) * (5 / 3) ** 0.5
    sym, xyz, q = globule_atoms(natoms, radius, net, rng)
    write_xyz(os.path.join(d, "target.xyz"), sym, xyz, q)
    ft = ft or (6 if gas in ("N2", "CO2") else 4)
    return write_input(d, "target.xyz", gas, ft, nprobe, niter, seed, extra=extra or None)


def fast_globule_atoms(n, radius, net, rng, dmin=1.0):
    """n atoms uniform in a sphere with no pair closer than dmin: draw 1.3 n
    points, drop the later point of every close pair (k-d tree), keep the
    first n survivors (redrawing if too few survive)."""
    from scipy.spatial import cKDTree
    m = int(1.3 * n) + 16
    while True:
        v = rng.normal(size=(m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        pts = v * radius * rng.random((m, 1)) ** (1 / 3)
        pairs = cKDTree(pts).query_pairs(dmin, output_type="ndarray")
        keep = np.ones(m, dtype=bool)
        keep[pairs.max(axis=1)] = False
        # a point dropped for one pair may leave its partner in another close pair: thin again
        idx = np.flatnonzero(keep)
        sub = pts[idx]
        pairs = cKDTree(sub).query_pairs(dmin, output_type="ndarray")
        if len(pairs):
            k2 = np.ones(len(idx), dtype=bool)
            k2[pairs.max(axis=1)] = False
            idx = idx[k2]
        if len(idx) >= n:
            xyz = pts[idx[:n]]
            return _elements(n, rng), xyz, _charges(n, net, rng)
        m = int(m * 1.3)


def batch(d, nions=256, ntraj=20000, nmin=500, nmax=50000, qmax=30, seed=2104, gen_seed=256):
    """The batched-ion workload: one directory (and input.json) per ion; returns the json paths."""
    rng = np.random.default_rng(gen_seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nions)).astype(int)
    charges = rng.integers(0, qmax + 1, nions)
    paths = []
    for i, (n, q) in enumerate(zip(sizes, charges)):
        di = os.path.join(d, f"ion{i:03d}")
        os.makedirs(di, exist_ok=True)
        radius = 1.3 * n ** (1 / 3) * (5 / 3) ** 0.5
        sym, xyz, qq = fast_globule_atoms(int(n), radius, float(q), rng)
        write_xyz(os.path.join(di, "target.xyz"), sym, xyz, qq)
        paths.append(write_input(di, "target.xyz", "He", 4, ntraj, 1, seed + i))
    return paths


def shell(d, natoms=500000, r_in=100.0, r_out=130.0, net=40.0, gas="He", nprobe=100000, niter=10, seed=2104,
          gen_seed=500000, **extra):
    os.makedirs(d, exist_ok=True)
    rng = np.random.default_rng(gen_seed)

    def sample(m):
        v = rng.normal(size=(m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        r = (r_in ** 3 + (r_out ** 3 - r_in ** 3) * rng.random((m, 1))) ** (1 / 3)
        return v * r
    lo, hi = np.full(3, -r_out - 1), np.full(3, r_out + 1)
    xyz = _rsa(natoms, sample, 1.2, rng, lo, hi)
    write_xyz(os.path.join(d, "target.xyz"), _elements(natoms, rng), xyz, _charges(natoms, net, rng))
    ft = 6 if gas in ("N2", "CO2") else 4
    return write_input(d, "target.xyz", gas, ft, nprobe, niter, seed, extra=extra or None)


def field_globule(d, gas="N2", natoms=20000, net=12.0, nprobe=100000, niter=10, seed=2104, gen_seed=20000,
                  **extra):
    """The learned-field workload: a 20,000-atom globule at +12 e with the N2
    or CO2 probe, all force terms on (force type 6)."""
    os.makedirs(d, exist_ok=True)
    rng = np.random.default_rng(gen_seed)
    radius = 1.3 * natoms ** (1 / 3) * (5 / 3) ** 0.5
    sym, xyz, q = fast_globule_atoms(natoms, radius, net, rng)
    write_xyz(os.path.join(d, "target.xyz"), sym, xyz, q)
    return write_input(d, "target.xyz", gas, 6, nprobe, niter, seed, extra=extra or None)
