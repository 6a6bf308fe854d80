"""One job split over several GPUs (mh_run_devices), through the host C-ABI
(GPU).  This machine offers one GPU, so the split runs as several contexts
on that GPU (a GPU number may repeat): the slices, threads, gather and the
fixed-order reduction are the multi-GPU code path itself, and with the lanes
per force evaluation fixed the CCS must equal the one-context run's bit for
bit (every trajectory keeps its random numbers)."""
import os

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,split", [("c60_he", 2), ("globule_n2", 3)])
def test_split_run_equals_single_run(tmp_path, kind, split):
    from massccs_b200 import host, synth
    gen = getattr(synth, kind)
    S = host.System(gen(os.path.join(tmp_path, kind), nprobe=2000, niter=5))
    one = S.run(0, lanes_per_traj=32)
    many = S.run_devices([0] * split, lanes_per_traj=32)
    assert one[0] == many[0] and one[1] == many[1], (one, many)
    tuned = S.run_devices([0] * split)  # lanes tuned once and shared: a valid run
    assert abs(tuned[0] - one[0]) <= 0.02 * one[0]
