"""The FP64 oracle against the reference's own outputs (CPU only).

Pins oracle/ccs_oracle.c:
  - std::mt19937 known answer (the C++ standard's 10000th output for seed 5489);
  - the reference's shipped logs (ccs_He.log, ccs_Ar.log, ccs.out exact at the
    printed 6 digits; ccs_N2.log 9/10 iterations, the tenth is a chaotic
    trajectory that differs even between builds of the reference);
  - the reference binary, built from its sources, on small runs of every gas
    and every force type whose arithmetic is defined (tests/golden/reference_runs.json).
"""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, input_dict, oracle_system, workdir, write_input


def test_mt19937_known_answer(oracle):
    assert int(oracle.mt19937(5489, 10000)[-1]) == 4123659995


def test_predraw_rows_follow_the_reference_order(oracle):
    s = oracle_system(oracle, gas="N2", ft=6, nprobe=16)
    raw = oracle.mt19937(s.params["seed"], 16 * 9).astype(np.float64) / 4294967295.0
    rnd = s.predraw(16)
    # System.cpp:185-196: 9 draws per trajectory, j ascending; row 0 is sqrt(bmax^2 u)
    np.testing.assert_array_equal(rnd[1], raw[1::9])
    np.testing.assert_array_equal(rnd[8], raw[8::9])
    np.testing.assert_array_equal(rnd[0], np.sqrt(s.params["bmax"] ** 2 * raw[0::9]))


def _replay(oracle, rep, quirks=1):
    d = workdir()
    p = write_input(d, rep["input"])
    s = oracle.OracleSystem(p)
    P = s.params
    n = P["nprobe"] * P["niter"]
    out = s.run(s.predraw(n), quirks=quirks)
    red = oracle.reduce(P["niter"], P["nprobe"], out["status"], out["one_minus_cos"], P["bmax"])
    return red


@pytest.mark.parametrize("name", ["ccs_He.log", "ccs_Ar.log", "ccs.out"])
def test_shipped_logs_replay_exactly(oracle, name):
    rep = json.load(open(os.path.join(GOLDEN, "shipped_logs.json")))[name]
    red = _replay(oracle, rep)
    assert ["%g" % w for w in red["omega"]] == [it["omega"] for it in rep["iterations"]]
    assert [int(v) for v in red["nfree"]] == [it["Nfree"] for it in rep["iterations"]]
    assert [int(v) for v in red["nlost"]] == [it["Nlost"] for it in rep["iterations"]]
    assert "%g" % red["ccs"] == rep["ccs"]
    assert "%g" % red["err"] == rep["err"]


def test_shipped_n2_log_replays_to_chaos_noise(oracle):
    rep = json.load(open(os.path.join(GOLDEN, "shipped_logs.json")))["ccs_N2.log"]
    red = _replay(oracle, rep)
    match = sum("%g" % w == it["omega"] for w, it in zip(red["omega"], rep["iterations"]))
    assert match >= 9
    assert abs(red["ccs"] - float(rep["ccs"])) / float(rep["ccs"]) < 1e-4


def test_reference_binary_runs(oracle):
    runs = json.load(open(os.path.join(GOLDEN, "reference_runs.json")))
    total = exact = 0
    for rep in runs:
        red = _replay(oracle, rep)
        it = rep["iterations"]
        # counts are exact on every configuration
        assert [int(v) for v in red["nfree"]] == [i["Nfree"] for i in it], rep["input"]
        assert [int(v) for v in red["nscatter"]] == [i["Nscatter"] for i in it], rep["input"]
        m = sum("%g" % w == i["omega"] for w, i in zip(red["omega"], it))
        total += len(it)
        exact += m
        assert m >= len(it) - 1, rep["input"]
        assert abs(red["ccs"] - float(rep["ccs"])) / float(rep["ccs"]) < 2e-3, rep["input"]
    assert exact >= total - 2


def test_co2_quirk_switch_changes_only_the_reference_velocity(oracle):
    s = oracle_system(oracle, gas="CO2", ft=4, nprobe=64)
    rnd = s.predraw(64)
    a = s.run(rnd, quirks=1)
    b = s.run(rnd, quirks=0)
    np.testing.assert_array_equal(a["status"], b["status"])
    np.testing.assert_array_equal(a["steps"], b["steps"])
    assert not np.allclose(a["one_minus_cos"], b["one_minus_cos"])


def test_site_force_out_of_grid_is_zero(oracle):
    s = oracle_system(oracle, gas="He", ft=4)
    P = s.params
    f, U, vis = s.site_force(0, np.array([P["lx"] * 3, 0.0, 0.0]))
    assert np.all(f == 0) and U == 0 and vis == 0


def test_site_force_matches_finite_difference(oracle):
    """-dU/dx of the oracle's energy equals its force inside the cutoffs."""
    s = oracle_system(oracle, target="04_1ubq_charge_4e_min.pqr", gas="N2", ft=6)
    t = s.target()
    rng = np.random.default_rng(3)
    for k in range(20):
        a = rng.integers(0, len(t["x"]))
        p = np.array([t["x"][a], t["y"][a], t["z"][a]]) + rng.normal(size=3) * 2.0 + 2.0
        for site in (0, 2):
            f, U, _ = s.site_force(site, p)
            h = 1e-5
            for d in range(3):
                e = np.zeros(3)
                e[d] = h
                Up = s.site_force(site, p + e)[1]
                Um = s.site_force(site, p - e)[1]
                fd = -(Up - Um) / (2 * h)
                assert abs(fd - f[d]) <= 1e-4 * max(1.0, abs(f[d])), (site, d, fd, f[d])
