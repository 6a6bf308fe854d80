"""Parity on the benchmark workloads themselves (GPU, through the C-ABI).

The throughput figures are quoted on seeded synthetic targets
(massccs_b200/synth.py): the 60-atom cage with He (c60_he), the 1231-atom
+4 e globule with N2 (globule_n2) and the 20,000-atom +12 e globule of the
learned-field configuration with N2 and CO2 (field_globule).  These tests run
the engine against the FP64 oracle on samples of exactly those workloads, on
identical initial conditions (the reference's mt19937 pre-draw).

Bars (stated here, used below):
  FP64 engine mode: the same status and 1-cos(chi) within 1e-7 on >= 97 % of
    trajectories (>= 90 % on the 20,000-atom N2 sample of 96 trajectories and
    >= 85 % on the CO2 sample of 48, where one chaotic orbit is 1-2 % of the
    sample: a rotating CO2 in the field of a +12 e ion makes many
    multi-collision orbits, on which any change of summation order grows;
    measured 87.5-92 %).
  FP32 engine mode (production), per trajectory, on the trajectories that
    scatter in both runs (|delta(1-cos chi)| against the oracle's FP64):
      c60_he      <= 1e-6 on >= 99 % and <= 1e-4 on >= 99.9 % (one collision
                  with a 60-atom cage: rounding stays at the FP32 level);
      globule_n2  <= 1e-5 on >= 85 % and <= 1e-3 on >= 90 % (measured: 90.0 %
                  and 95.4 %; the rest are multi-collision orbits of the
                  rotating N2 whose outcome any rounding change alters);
    status agreement >= 97 %; and the paired CCS within 0.5 % of the oracle's,
    or 4 paired standard errors where the sample is too small for 0.5 %.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# |delta(1 - cos chi)| bars per workload: (tight, share), (loose, share)
FP32_BARS = {"c60_he": ((1e-6, 0.99), (1e-4, 0.999)), "globule_n2": ((1e-5, 0.85), (1e-3, 0.90))}


def _workload(kind, d, n):
    from massccs_b200 import synth
    if kind == "c60_he":
        return synth.c60_he(d, nprobe=n, niter=1)
    if kind == "globule_n2":
        return synth.globule_n2(d, nprobe=n, niter=1)
    gas = kind.split("_")[-1].upper()
    return synth.field_globule(d, gas=gas, nprobe=n, niter=1)


_CACHE = {}


def _oracle_run(oracle, kind, n, tmp):
    """Oracle results on the workload's first n trajectories (cached per session)."""
    key = (kind, n)
    if key not in _CACHE:
        from massccs_b200 import host
        p = _workload(kind, os.path.join(tmp, f"{kind}_{n}"), n)
        S = host.System(p)
        rnd = S.predraw(n)
        ref = oracle.OracleSystem(p).run(rnd)
        _CACHE[key] = (S, rnd, ref)
    return _CACHE[key]


def _paired_ccs_ok(bmax, ref, out):
    a = np.pi * np.where(ref["status"] == 1, ref["one_minus_cos"], 0.0) * bmax ** 2
    b = np.pi * np.where(out["status"] == 1, out["one_minus_cos"], 0.0) * bmax ** 2
    ok = (ref["status"] <= 1) & (out["status"] <= 1)
    d = (b - a)[ok]
    w = a[ok].mean()
    se = d.std(ddof=1) / np.sqrt(len(d))
    assert abs(d.mean()) <= max(0.005 * w, 4 * se), (d.mean(), se, w)


FP64_CASES = [("c60_he", 4000, 0.97), ("globule_n2", 600, 0.97), ("field_n2", 96, 0.90), ("field_co2", 48, 0.85)]


@pytest.mark.parametrize("kind,n,bar", FP64_CASES)
def test_workload_fp64_matches_oracle(oracle, tmp_path_factory, kind, n, bar):
    S, rnd, ref = _oracle_run(oracle, kind, n, str(tmp_path_factory.getbasetemp()))
    eng = S.engine(precision=1)
    out = eng.run(rnd)
    eng.close()
    same = out["status"] == ref["status"]
    assert same.mean() >= bar, same.mean()
    close = same & (np.abs(out["one_minus_cos"] - ref["one_minus_cos"]) <= 1e-7)
    assert close.mean() >= bar, close.mean()
    st = out["stats"]
    assert st["nfree"] + st["nscatter"] + st["nlost"] + st["ncapped"] == n


FP32_CASES = [("c60_he", 4000), ("globule_n2", 600)]


@pytest.mark.parametrize("kind,n", FP32_CASES)
def test_workload_fp32_per_trajectory_bar(oracle, tmp_path_factory, kind, n):
    S, rnd, ref = _oracle_run(oracle, kind, n, str(tmp_path_factory.getbasetemp()))
    eng = S.engine(precision=0)
    out = eng.run(rnd)
    eng.close()
    assert (out["status"] == ref["status"]).mean() >= 0.97
    both = (out["status"] == 1) & (ref["status"] == 1)
    d = np.abs(out["one_minus_cos"] - ref["one_minus_cos"])[both]
    assert both.sum() >= 0.5 * n
    for tol, share in FP32_BARS[kind]:
        assert (d <= tol).mean() >= share, (tol, (d <= tol).mean(), np.quantile(d, [0.5, 0.9, 0.95, 0.99]))
    _paired_ccs_ok(S.info["bmax"], ref, out)


@pytest.mark.parametrize("gas", ["n2", "co2"])
def test_field_globule_fp32_paired_with_fp64(tmp_path, gas):
    """The 20,000-atom workload at a size the oracle cannot cover in a test:
    the FP32 engine paired with the (oracle-pinned) FP64 engine mode on the
    same 2000 initial conditions."""
    from massccs_b200 import host
    n = 2000
    S = host.System(_workload(f"field_{gas}", str(tmp_path), n))
    rnd = S.predraw(n)
    e64 = S.engine(precision=1)
    r64 = e64.run(rnd)
    e64.close()
    e32 = S.engine(precision=0)
    r32 = e32.run(rnd)
    e32.close()
    assert (r32["status"] == r64["status"]).mean() >= 0.95
    _paired_ccs_ok(S.info["bmax"], r64, r32)
