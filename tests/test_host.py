"""The product's host set-up (libmassccs_host.so) against the oracle (CPU).

The host re-implements the reference's Input / GasBuffer / MoleculeTarget /
ellipsoid / pre-draw / reduction in C++; every one of them must reproduce the
oracle's restatement exactly (bit-exact scalars and arrays), because the GPU
engine's parity is only meaningful on identical inputs.
"""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, input_dict, workdir, write_input

CASES = [("c60.xyz", "He", 4, None), ("c60.xyz", "Ar", 4, None), ("c60.xyz", "N2", 6, None),
         ("c60.xyz", "CO2", 6, None), ("c60.xyz", "co2", 2, None), ("c60.xyz", "He", 1, None),
         ("04_1ubq_charge_4e_min.pqr", "He", 4, None), ("04_1ubq_charge_4e_min.pqr", "N2", 4, None),
         ("c60.xyz", "He", 2, "uff.ff"), ("04_1ubq_charge_4e_min.pqr", "CO2", 4, "uff.ff")]


@pytest.fixture(scope="module")
def host():
    from massccs_b200 import build, host
    build.build()
    return host


def _sorted_target(t):
    keys = ("x", "y", "z", "q", "m", "eps", "sig")
    arr = np.stack([t[k] for k in keys], 1)
    return arr[np.lexsort(arr[:, :3].T[::-1])]


@pytest.mark.parametrize("target,gas,ft,ff", CASES)
def test_setup_matches_oracle(oracle, host, target, gas, ft, ff):
    d = workdir()
    p = write_input(d, input_dict(target, gas, ft, nprobe=50, niter=2, ff=ff))
    S = host.System(p)
    O = oracle.OracleSystem(p)
    hi, oi = S.info, O.params
    for k in ("gas_flag", "force_type", "natoms", "gas_natoms", "nprobe", "niter", "seed", "Nx", "Ny", "Nz"):
        assert hi[k] == oi[k], k
    for k in ("dt", "temperature", "skin", "lj_cutoff", "coul_cutoff", "alpha", "mu", "target_mass",
              "target_charge", "gas_mass", "gas_inertia", "d_bond", "a", "b", "c", "bmax", "lx", "ly", "lz",
              "max_x", "max_y", "max_z", "radius"):
        assert hi[k] == oi[k], (k, hi[k], oi[k])
    # the oracle keeps the reference's cell order; compare as sorted sets, bit-exact
    np.testing.assert_array_equal(_sorted_target(S.target()), _sorted_target(O.target()))
    if gas == "CO2":
        ts, to = S.target(), O.target()
        np.testing.assert_array_equal(np.sort(ts["eps_c"]), np.sort(to["eps_c"]))
        np.testing.assert_array_equal(np.sort(ts["sig_c"]), np.sort(to["sig_c"]))


@pytest.mark.parametrize("gas", ["He", "N2"])
def test_bulk_predraw_matches_oracle_on_a_long_odd_run(oracle, host, gas):
    """The host draws the mt19937 words in blocks of 624 and converts them in
    parallel; the rows must equal the oracle's one-by-one draws bit for bit
    over many blocks and a count that ends inside a block."""
    d = workdir()
    p = write_input(d, input_dict("c60.xyz", gas, 4, nprobe=100003, niter=1))
    S, O = host.System(p), oracle.OracleSystem(p)
    np.testing.assert_array_equal(S.predraw(100003), O.predraw(100003))


@pytest.mark.parametrize("gas", ["He", "N2"])
def test_predraw_matches_oracle(oracle, host, gas):
    d = workdir()
    p = write_input(d, input_dict("c60.xyz", gas, 4, nprobe=300, niter=3))
    S, O = host.System(p), oracle.OracleSystem(p)
    np.testing.assert_array_equal(S.predraw(), O.predraw(900))


def test_reduction_matches_oracle(oracle, host):
    rng = np.random.default_rng(0)
    status = rng.choice([0, 1, 1, 1, 2], size=5000).astype(np.int8)
    omc = np.where(status == 1, rng.random(5000) * 2, 0.0)
    a = host.reduce(10, 500, status, omc, 53.6)
    b = oracle.reduce(10, 500, status, omc, 53.6)
    np.testing.assert_array_equal(a["omega"], b["omega"])
    np.testing.assert_array_equal(a["nfree"], b["nfree"])
    assert a["ccs"] == b["ccs"] and a["err"] == b["err"]


def test_input_errors_are_reported(host):
    d = workdir()
    p = os.path.join(d, "bad.json")
    json.dump({"numberProbe": 10}, open(p, "w"))
    with pytest.raises(Exception, match="targetFileName"):
        host.System(p)
    p2 = write_input(d, dict(input_dict("c60.xyz"), GasBuffer="Xe"), name="bad2.json")
    with pytest.raises(Exception, match="gas buffer"):
        host.System(p2)
    p3 = write_input(d, input_dict("missing.xyz"), name="bad3.json")
    with pytest.raises(Exception):
        host.System(p3)


def test_synthetic_targets(host):
    from massccs_b200 import synth
    d = workdir(())
    S = host.System(synth.c60_he(os.path.join(d, "c60"), nprobe=10, niter=1))
    t = S.target()
    xyz = np.stack([t["x"], t["y"], t["z"]], 1)
    dist = np.linalg.norm(xyz[:, None] - xyz[None], axis=2)
    np.fill_diagonal(dist, 9)
    assert S.info["natoms"] == 60 and abs(dist.min() - 1.40) < 1e-6
    assert ((np.abs(dist - 1.40) < 1e-6).sum() // 2) == 90  # the 90 edges of a truncated icosahedron
    G = host.System(synth.globule_n2(os.path.join(d, "glob"), nprobe=10, niter=1))
    assert G.info["natoms"] == 1231 and abs(G.info["target_charge"] - 4.0) < 1e-5
    assert G.info["force_type"] == 6 and G.info["gas_flag"] == 2


def test_batch_workload_generator(host):
    """The batched-ion workload: log-uniform sizes in range, integer net
    charges in [0, 30] e, the 1.0 A minimum distance, seeded (same files twice)."""
    from scipy.spatial import cKDTree
    from massccs_b200 import synth
    d = workdir(())
    paths = synth.batch(os.path.join(d, "b1"), nions=6, ntraj=10, nmin=500, nmax=5000)
    again = synth.batch(os.path.join(d, "b2"), nions=6, ntraj=10, nmin=500, nmax=5000)
    for p, q in zip(paths, again):
        S = host.System(p)
        assert 500 <= S.info["natoms"] <= 5000 and S.info["gas_flag"] == 1
        Q = S.info["target_charge"]
        assert abs(Q - round(Q)) < 1e-6 and 0 <= round(Q) <= 30
        t = S.target()
        xyz = np.stack([t["x"], t["y"], t["z"]], 1)
        assert not cKDTree(xyz).query_pairs(1.0 - 1e-9)
        a = open(os.path.join(os.path.dirname(p), "target.xyz")).read()
        assert a == open(os.path.join(os.path.dirname(q), "target.xyz")).read()


def test_number_forms_read_as_stream_extraction(oracle, host):
    """The whole-file reader (from_chars on plain numbers, stream extraction
    for anything else) reads signs, exponents, bare fractions, CRLF line ends
    and tabs exactly as the oracle's reader does."""
    d = workdir()
    lines = ["C +1.25 -0.5e1 .75 0.125", "C\t1.5E+01 -2 3. -0.25", "H 0.5 +2.5E-1 -1e0 +0.0625",
             "O -3.75 4 0.0 0.0625", "N 2.5 -1.25 +3.5 0.0"]
    with open(os.path.join(d, "forms.xyz"), "w", newline="") as f:
        f.write("5\r\ncomment\r\n" + "\r\n".join(lines) + "\r\n")
    with open(os.path.join(d, "forms_lf.xyz"), "w") as f:
        f.write("5\ncomment\n" + "\n".join(lines) + "\n")
    for name in ("forms.xyz", "forms_lf.xyz"):
        p = write_input(d, input_dict(name, "He", 4, nprobe=10, niter=1), name=name + ".json")
        S, O = host.System(p), oracle.OracleSystem(p)
        np.testing.assert_array_equal(_sorted_target(S.target()), _sorted_target(O.target()))
        assert S.info["target_charge"] == O.params["target_charge"]


REF_BIN = os.path.join(os.path.dirname(GOLDEN), os.pardir, "oracle", "_ref", "massccs")


@pytest.mark.parametrize("target,gas,ft", [("c60.xyz", "He", 4), ("c60.xyz", "He", 2), ("c60.xyz", "N2", 6),
                                            ("c60.xyz", "N2", 4), ("c60.xyz", "CO2", 4),
                                            ("04_1ubq_charge_4e_min.pqr", "He", 4)])
def test_equipotential_ellipsoid_matches_reference_binary(host, target, gas, ft):
    """"Equipotential": "yes" (Equipotential.cpp): the host's axes against the
    reference binary's report, which prints them to 6 significant digits."""
    import re
    import subprocess
    if not os.access(REF_BIN, os.X_OK):
        pytest.skip("reference binary not built here")
    d = workdir()
    cfg = dict(input_dict(target, gas, ft, nprobe=2, niter=1), Equipotential="yes", nthreads=4)
    p = write_input(d, cfg)
    out = subprocess.run([os.path.abspath(REF_BIN), "input.json"], cwd=d, capture_output=True, text=True,
                         timeout=600).stdout
    ref = [float(v) for v in re.search(r"^ellipsoid axis length: (\S+)\s+(\S+)\s+(\S+)", out, re.M).groups()]
    S = host.System(p)
    for k, r in zip("abc", ref):
        assert abs(S.info[k] - r) <= 6e-6 * r, (k, S.info[k], r)
    assert S.info["bmax"] == max(S.info["a"], S.info["b"], S.info["c"])


def test_setup_device_key(host):
    """input.json's "setup_device" extension key: cpu, gpu or auto (the CPU
    path needs no GPU; anything else is an input error)."""
    d = workdir()
    cfg = dict(input_dict("c60.xyz"), Equipotential="yes", setup_device="cpu")
    S = host.System(write_input(d, cfg, name="a.json"))
    assert S.info["bmax"] > 0
    with pytest.raises(Exception, match="setup_device"):
        host.System(write_input(d, dict(input_dict("c60.xyz"), setup_device="tpu"), name="b.json"))


def test_devices_key(host):
    """input.json's "devices" extension key: a count (GPUs 0..N-1) or a list."""
    d = workdir()
    assert host.System(write_input(d, input_dict("c60.xyz"), name="a.json")).devices() == []
    assert host.System(write_input(d, dict(input_dict("c60.xyz"), devices=3), name="b.json")).devices() == [0, 1, 2]
    assert host.System(write_input(d, dict(input_dict("c60.xyz"), devices="0,2,2"), name="c.json")).devices() == [0, 2, 2]
    with pytest.raises(Exception, match="devices"):
        host.System(write_input(d, dict(input_dict("c60.xyz"), devices="0,x"), name="e.json"))
