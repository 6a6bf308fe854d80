"""Batched ions (GPU): ccs_run_batch runs many ions of uneven size in one
launch of each pass.  Every ion's trajectories must come out as they do from
that ion's own ccs_run on the same initial conditions.

Bars: FP64 mode, per trajectory the same status and 1-cos(chi) to 1e-7 on
>= 97 %; FP32 mode, status agreement >= 97 % and paired CCS within 0.5 % or 4
paired standard errors (the batch kernels read each ion's parameters from
device memory, and a chaotic orbit may round differently).
"""
import ctypes
import os

import numpy as np
import pytest

from helpers import input_dict, workdir, write_input

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ions(tmp_path_factory):
    from massccs_b200 import host, synth
    d = workdir()
    out = [host.System(write_input(d, input_dict("c60.xyz", "He", 4, nprobe=600, niter=1), name="c60.json")),
           host.System(write_input(d, input_dict("04_1ubq_charge_4e_min.pqr", "He", 4, nprobe=400, niter=1),
                                   name="ubq.json"))]
    base = str(tmp_path_factory.mktemp("globules"))
    for k, (natoms, q) in enumerate([(500, 3), (2500, 12), (900, 0)]):
        out.append(host.System(synth.globule(os.path.join(base, f"g{k}"), natoms, q, gas="He", nprobe=500,
                                             niter=1, gen_seed=k)))
    return out


def _bmax_ccs(status, omc, bmax):
    return np.pi * np.where(status == 1, omc, 0.0) * bmax ** 2


@pytest.mark.parametrize("precision", [1, 0])
def test_batch_matches_separate_runs(ions, precision):
    from massccs_b200 import engine as E
    engs = [S.engine(precision=precision, lanes_per_traj=32) for S in ions]
    rnds = [S.predraw() for S in ions]
    sep = [e.run(r) for e, r in zip(engs, rnds)]
    bat, st = E.run_batch(engs, rnds)
    assert st["ntraj"] == sum(r.shape[1] for r in rnds)
    assert st["nfree"] + st["nscatter"] + st["nlost"] + st["ncapped"] == st["ntraj"]
    for S, a, b in zip(ions, sep, bat):
        same = a["status"] == b["status"]
        assert same.mean() >= 0.97
        if precision == 1:
            close = same & (np.abs(a["one_minus_cos"] - b["one_minus_cos"]) <= 1e-7)
            assert close.mean() >= 0.97, close.mean()
        else:
            bmax = S.info["bmax"]
            ok = (a["status"] <= 1) & (b["status"] <= 1)
            d = (_bmax_ccs(b["status"], b["one_minus_cos"], bmax) - _bmax_ccs(a["status"], a["one_minus_cos"], bmax))[ok]
            ref = _bmax_ccs(a["status"], a["one_minus_cos"], bmax)[ok].mean()
            assert abs(d.mean()) <= max(0.005 * ref, 4 * d.std(ddof=1) / np.sqrt(len(d)))
    for e in engs:
        e.close()


def test_batch_autotuned_and_parked(ions):
    from massccs_b200 import engine as E
    engs = [S.engine(park_steps=64) if i == 0 else S.engine() for i, S in enumerate(ions)]
    rnds = [S.predraw() for S in ions]
    bat, st = E.run_batch(engs, rnds)
    assert st["lanes_per_traj"] in (8, 16, 32)
    assert st["parked"] > 0
    for b in bat:
        assert set(np.unique(b["status"])) <= {0, 1, 2}
        assert (b["steps"][b["status"] == 1] > 0).all()
    for e in engs:
        e.close()


def test_batch_rejects_mixed_gases(ions):
    from massccs_b200 import engine as E
    from massccs_b200 import host
    d = workdir()
    n2 = host.System(write_input(d, input_dict("c60.xyz", "N2", 6, nprobe=10, niter=1), name="n2.json"))
    engs = [ions[0].engine(), n2.engine()]
    with pytest.raises(E.CcsError, match="mixed"):
        E.run_batch(engs, [ions[0].predraw(10), n2.predraw(10)])
    for e in engs:
        e.close()
