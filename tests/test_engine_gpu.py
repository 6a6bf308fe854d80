"""Parity of the CUDA engine with the FP64 oracle, through the C-ABI (GPU).

Bars (stated here, used below):
  FP64 engine mode: per-pair force sums to 1e-9 relative; setup identical hit
    flags and positions to 1e-12; per trajectory the same status and
    1-cos(chi) to 1e-7 on >= 97 % of trajectories (the rest are chaotic
    orbits, which differ even between two builds of the reference).
  FP32 engine mode (the production mode): forces to 1e-4 relative plus
    1e-4 kcal/mol/A, energies to 1e-5 relative plus 2e-4 kcal/mol (FP32
    accumulation of ~1e3 Coulomb terms); status agreement >= 97 %; paired CCS
    within 0.5 % of the oracle's on identical initial conditions, or within 4
    paired standard errors on samples too small for a single chaotic orbit to
    stay below 0.5 % (the 0.5 % bar at 1e5 trajectories: test_cli_gpu.py).
"""
import numpy as np
import pytest

from helpers import engine_for, oracle_system, rel

pytestmark = pytest.mark.gpu


def _points(sys_, n, rng, near=True):
    t = sys_.target()
    a = rng.integers(0, len(t["x"]), n)
    base = np.stack([t["x"][a], t["y"][a], t["z"][a]], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = rng.uniform(2.6, 30.0, size=(n, 1)) if near else rng.uniform(20, 60, size=(n, 1))
    return base + d * r


def _coulomb_abs_sum(sys_, site, pts):
    """Sum over atoms of |k q_site q_i / r_i| at each point (the magnitude of
    the terms an all-pairs Coulomb energy adds up)."""
    q_site = {1: 0.0, 4: 0.0, 5: 0.0, 2: (-0.4825, -0.4825, 0.965)[site], 3: (-0.3256, 0.6512, -0.3256)[site]}
    qs = q_site[sys_.params["gas_flag"]]
    t = sys_.target()
    xyz = np.stack([t["x"], t["y"], t["z"]], 1)
    r = np.linalg.norm(pts[:, None, :] - xyz[None, :, :], axis=2)
    return 332.06348078020324 * abs(qs) * (np.abs(t["q"])[None, :] / r).sum(1)


CASES = [("c60.xyz", "He", 4), ("c60.xyz", "He", 2), ("c60.xyz", "He", 1), ("c60.xyz", "Ar", 4),
         ("04_1ubq_charge_4e_min.pqr", "He", 4), ("04_1ubq_charge_4e_min.pqr", "N2", 6),
         ("04_1ubq_charge_4e_min.pqr", "N2", 4), ("04_1ubq_charge_4e_min.pqr", "N2", 3),
         ("04_1ubq_charge_4e_min.pqr", "CO2", 6), ("c60.xyz", "CO2", 4), ("c60.xyz", "co2", 2),
         # all-pairs routines (force types 1/3/5: no cutoffs, no shifts; Force.cpp:117-300, 495-574,
         # 836-897, 1169-1219, 1352-1415, 1637-1725)
         ("c60.xyz", "He", 3), ("04_1ubq_charge_4e_min.pqr", "He", 3), ("04_1ubq_charge_4e_min.pqr", "N2", 5),
         ("c60.xyz", "N2", 1), ("04_1ubq_charge_4e_min.pqr", "CO2", 5), ("c60.xyz", "CO2", 3),
         ("c60.xyz", "CO2", 1)]


@pytest.mark.parametrize("target,gas,ft", CASES)
@pytest.mark.parametrize("prec", [1, 0])
def test_site_forces_match_oracle(oracle, target, gas, ft, prec):
    s = oracle_system(oracle, target=target, gas=gas, ft=ft)
    eng = engine_for(s, precision=prec)
    rng = np.random.default_rng(7)
    pts = np.concatenate([_points(s, 300, rng), _points(s, 50, rng, near=False)])
    nsite = 3 if gas in ("N2", "CO2") else 1
    for site in range(nsite):
        f, U, _ = eng.eval_site_forces(site, pts)
        fo = np.empty_like(f)
        Uo = np.empty_like(U)
        for i, p in enumerate(pts):
            fo[i], Uo[i], _ = s.site_force(site, p)
        fn = np.linalg.norm(f - fo, axis=1)
        if prec == 1:
            assert (fn / (np.linalg.norm(fo, axis=1) + 1e-3)).max() < 1e-9, site
            assert (np.abs(U - Uo) / (np.abs(Uo) + 1e-3)).max() < 1e-9, site
        else:
            # positions a thermal probe can reach (|U| below 100 kcal/mol; probes carry ~1)
            reach = np.abs(Uo) < 100.0
            assert reach.sum() > 100
            # all-pairs types sum every atom's unshifted Coulomb term: FP32 rounding
            # scales with the sum of their magnitudes (64 units of 2^-24 of it)
            floor = 2e-4 + (64 * 2.0 ** -24 * _coulomb_abs_sum(s, site, pts) if ft in (1, 3, 5)
                            else np.zeros(len(pts)))
            assert np.all(fn[reach] <= 1e-4 * np.linalg.norm(fo[reach], axis=1) + 1e-4), (site, fn[reach].max())
            assert np.all(np.abs(U - Uo)[reach] <= 1e-5 * np.abs(Uo[reach]) + floor[reach]), \
                (site, (np.abs(U - Uo) - 1e-5 * np.abs(Uo) - floor)[reach].max())
            # inside atoms the r^-12 wall amplifies FP32 rounding of the separation: relative bar
            assert np.all(np.abs(U - Uo) <= 1e-4 * np.abs(Uo) + floor), (site, (np.abs(U - Uo) / np.abs(Uo)).max())


@pytest.mark.parametrize("gas", ["He", "N2", "CO2"])
def test_setup_matches_oracle(oracle, gas):
    s = oracle_system(oracle, gas=gas, ft=4)
    eng = engine_for(s, precision=1)
    rnd = s.predraw(4000)
    hit, pos, vel = eng.eval_setup(rnd)
    ns = 3 if gas in ("N2", "CO2") else 1
    for j in range(0, 4000, 7):
        h, p, v, _, _ = s.setup_one(rnd[:, j])
        assert h == hit[j]
        if h:
            np.testing.assert_allclose(pos[j, :ns], p[:ns], rtol=1e-12, atol=1e-10)
            np.testing.assert_allclose(vel[j, :ns], v[:ns], rtol=1e-11, atol=1e-15)


def _paired(oracle, target, gas, ft, n, prec, quirks=0, **kw):
    s = oracle_system(oracle, target=target, gas=gas, ft=ft, nprobe=n)
    rnd = s.predraw(n)
    ref = s.run(rnd, quirks=quirks)
    eng = engine_for(s, precision=prec, quirks=quirks, **kw)
    out = eng.run(rnd)
    return s, ref, out


TRAJ = [("c60.xyz", "He", 4, 3000), ("c60.xyz", "Ar", 4, 2000),
        ("04_1ubq_charge_4e_min.pqr", "He", 4, 1500), ("c60.xyz", "N2", 6, 1000),
        ("04_1ubq_charge_4e_min.pqr", "N2", 6, 600), ("c60.xyz", "CO2", 4, 800),
        ("c60.xyz", "He", 3, 1500), ("c60.xyz", "N2", 5, 400), ("c60.xyz", "CO2", 5, 300)]


@pytest.mark.parametrize("target,gas,ft,n", TRAJ)
def test_trajectories_fp64_match_oracle(oracle, target, gas, ft, n):
    s, ref, out = _paired(oracle, target, gas, ft, n, prec=1)
    same = out["status"] == ref["status"]
    assert same.mean() >= 0.97
    close = same & (np.abs(out["one_minus_cos"] - ref["one_minus_cos"]) <= 1e-7)
    assert close.mean() >= 0.97, close.mean()
    st = out["stats"]
    assert st["nfree"] + st["nscatter"] + st["nlost"] + st["ncapped"] == n


@pytest.mark.parametrize("target,gas,ft,n", TRAJ)
@pytest.mark.parametrize("lanes", [0, 1, 32])
def test_trajectories_fp32_paired_ccs(oracle, target, gas, ft, n, lanes):
    s, ref, out = _paired(oracle, target, gas, ft, n, prec=0, lanes_per_traj=lanes)
    assert (out["status"] == ref["status"]).mean() >= 0.97
    _paired_ccs_ok(s.params["bmax"], ref, out)


def _paired_ccs_ok(bmax, ref, out):
    """Paired comparison of the CCS estimator on identical initial conditions."""
    a = np.pi * np.where(ref["status"] == 1, ref["one_minus_cos"], 0.0) * bmax ** 2
    b = np.pi * np.where(out["status"] == 1, out["one_minus_cos"], 0.0) * bmax ** 2
    ok = (ref["status"] <= 1) & (out["status"] <= 1)
    d = (b - a)[ok]
    w_ref = a[ok].mean()
    se = d.std(ddof=1) / np.sqrt(len(d))
    assert abs(d.mean()) <= max(0.005 * w_ref, 4 * se), (d.mean(), se, w_ref)


# A low park threshold sends most trajectories through both passes (lane
# pass, then the warp pass after 64 steps): the hand-over must not change a
# result, whatever the warp pass's threads per trajectory.
PASSES = [("c60.xyz", "He", 4, 1500), ("04_1ubq_charge_4e_min.pqr", "N2", 6, 300), ("c60.xyz", "CO2", 4, 400)]


@pytest.mark.parametrize("target,gas,ft,n", PASSES)
@pytest.mark.parametrize("resume_block", [0, 32, 64])
def test_trajectories_fp64_through_both_passes(oracle, target, gas, ft, n, resume_block):
    s, ref, out = _paired(oracle, target, gas, ft, n, prec=1, park_steps=64, resume_block=resume_block)
    assert out["stats"]["parked"] > n // 4
    same = out["status"] == ref["status"]
    assert same.mean() >= 0.97
    close = same & (np.abs(out["one_minus_cos"] - ref["one_minus_cos"]) <= 1e-7)
    assert close.mean() >= 0.97, close.mean()
    assert (out["steps"] == ref["steps"]).mean() >= 0.97


@pytest.mark.parametrize("target,gas,ft,n", PASSES)
@pytest.mark.parametrize("resume_block", [32, 128])
def test_trajectories_fp32_through_both_passes(oracle, target, gas, ft, n, resume_block):
    s, ref, out = _paired(oracle, target, gas, ft, n, prec=0, park_steps=64, resume_block=resume_block)
    assert out["stats"]["parked"] > n // 4
    assert (out["status"] == ref["status"]).mean() >= 0.97
    _paired_ccs_ok(s.params["bmax"], ref, out)


def test_watchdog_expiry_is_an_error_and_the_context_survives(oracle):
    """A device wall-time budget far below the run's length: every CTA drains
    at its next check, the call returns CCS_ERR_TIMEOUT, and the same context
    runs normally afterwards (no fault, no hang: the deadline is polled)."""
    from massccs_b200 import engine as E
    s = oracle_system(oracle, target="04_1ubq_charge_4e_min.pqr", gas="N2", ft=6, nprobe=3000)
    rnd = s.predraw(3000)
    eng = engine_for(s, precision=0, lanes_per_traj=32, watchdog_s=1e-3)
    with pytest.raises(E.CcsError, match="watchdog"):
        eng.run(rnd)
    eng.set_params(E.params_from_system(s.params, precision=0, lanes_per_traj=32))
    t = s.target()
    eng.set_target(t["x"], t["y"], t["z"], t["q"], t["eps"], t["sig"])
    out = eng.run(rnd[:, :400])
    assert out["stats"]["ncapped"] == 0
    assert (out["status"] <= 1).mean() > 0.9


def test_co2_reference_velocity_quirk_matches_oracle(oracle):
    """CCS_QUIRK_CO2_VCM reproduces the reference's CO2 initial-velocity slip
    (System.cpp:1012): FP64 engine and oracle agree with the quirk on, and the
    quirk changes the scattering angles (it is not a no-op)."""
    s, ref, out = _paired(oracle, "c60.xyz", "CO2", 4, 400, prec=1, quirks=1)
    same = out["status"] == ref["status"]
    close = same & (np.abs(out["one_minus_cos"] - ref["one_minus_cos"]) <= 1e-7)
    assert close.mean() >= 0.97, close.mean()
    plain = engine_for(s, precision=1, quirks=0).run(s.predraw(400))
    sc = (plain["status"] == 1) & (out["status"] == 1)
    assert np.abs(plain["one_minus_cos"][sc] - out["one_minus_cos"][sc]).max() > 1e-3


@pytest.mark.parametrize("prec", [1, 0])
def test_speculative_tries_change_no_result(oracle, prec):
    """A trajectory's tries run at once (speculatively) once it has failed two
    in the warp pass; that changes the order of work, never a result: status,
    1-cos(chi) and steps equal those of the sequential tries bit for bit."""
    # few parked trajectories (speculation only runs when the warp pass is short of work)
    s = oracle_system(oracle, target="c60.xyz", gas="He", ft=4, nprobe=20000)
    rnd = s.predraw(20000)
    seq = engine_for(s, precision=prec, lanes_per_traj=32, park_steps=1024, spec_tries=-1).run(rnd)
    spec = engine_for(s, precision=prec, lanes_per_traj=32, park_steps=1024, spec_tries=2).run(rnd)
    assert spec["stats"]["speculated"] > 0 and seq["stats"]["speculated"] == 0
    assert np.array_equal(seq["status"], spec["status"])
    assert np.array_equal(seq["steps"], spec["steps"])
    assert np.array_equal(seq["one_minus_cos"], spec["one_minus_cos"])
    for k in ("nfree", "nscatter", "nlost", "ncapped", "steps"):
        assert seq["stats"][k] == spec["stats"][k], k
