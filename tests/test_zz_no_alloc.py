"""ccs_run_device_noalloc against ccs_run_device (GPU).

The no-allocation entry point serves callers that cannot allocate device
memory while they run (a host whose allocator owns the device heap, a service
with a fixed memory budget, code where an allocation would synchronise the
device): it keeps the run's scratch in the library's static device array.  It
runs the same kernels on the same inputs as the allocating entry point, so it
must return the same results bit for bit, and keep doing so on back-to-back
calls (the array keeps the previous call's contents, so everything that must
start at zero is cleared by each call).

This file sorts last so that a stopping run has executed every other test
first; it also passes on its own in a fresh process, where its first call is
the one that looks up the array's device address.
"""
import ctypes
import os

import pytest

pytestmark = pytest.mark.gpu

STAT_KEYS = ("nfree", "nscatter", "nlost", "ncapped", "steps", "visits", "parked")


def _system(kind, tmp, nprobe=None):
    from massccs_b200 import host, synth
    if kind == "c60_he":
        p = synth.c60_he(os.path.join(tmp, kind), nprobe=nprobe or 20000, niter=1)
    else:
        p = synth.globule_n2(os.path.join(tmp, kind), nprobe=nprobe or 3000, niter=1)
    return host.System(p)


class _Run:
    """Device buffers of one run (outputs pre-filled with values no run writes)."""

    def __init__(self, n, dev):
        import torch
        self.status = torch.full((n,), -1, dtype=torch.int8, device=dev)
        self.omc = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
        self.steps = torch.zeros(n, dtype=torch.int32, device=dev)
        self.visits = torch.zeros(n, dtype=torch.int32, device=dev)

    def ptrs(self):
        return (self.status.data_ptr(), self.omc.data_ptr(), self.steps.data_ptr(), self.visits.data_ptr())

    def same(self, o):
        import torch
        return (torch.equal(self.status, o.status) and torch.equal(self.omc, o.omc)
                and torch.equal(self.steps, o.steps) and torch.equal(self.visits, o.visits))


def _reference(eng, n, d_rnd, stream, dev):
    ref = _Run(n, dev)
    st, om, sp, vi = ref.ptrs()
    eng.run_device(n, d_rnd.data_ptr(), n, st, om, sp, vi, stream.cuda_stream)
    return ref, eng.sync_stats()


@pytest.mark.parametrize("kind,park", [("c60_he", 256), ("globule_n2", 512)])
@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_run_device_twice(tmp_path, kind, park, precision):
    """Two calls in a row, the first returning its statistics, the second
    without (stats == NULL, read back by ccs_sync_stats): both equal the
    allocating run bit for bit (status, 1-cos chi, steps, visits, counters)."""
    import torch
    S = _system(kind, str(tmp_path))
    n = S.info["nprobe"] * S.info["niter"]
    eng = S.engine(precision=precision, lanes_per_traj=32, park_steps=park)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    d_rnd = torch.from_numpy(S.predraw(n)).to(dev)
    ref, ref_stats = _reference(eng, n, d_rnd, stream, dev)
    assert ref_stats["parked"] > 0  # the park buffer in the scratch is exercised
    for call in range(2):
        out = _Run(n, dev)
        st, om, sp, vi = out.ptrs()
        stats = eng.run_device_noalloc(n, d_rnd.data_ptr(), n, st, om, sp, vi, stream.cuda_stream,
                                       want_stats=(call == 0))
        if stats is None:
            stats = eng.sync_stats()
        torch.cuda.synchronize()
        assert out.same(ref), call
        for key in STAT_KEYS:
            assert stats[key] == ref_stats[key], (call, key)
    eng.close()


def test_noalloc_parks_beyond_65536(tmp_path):
    """131,072 trajectories with a 16-step park threshold: almost all park
    (more than 65,536), so the park region of the array is used at the
    capacity ccs_run_device gives that size (every trajectory), and the
    results stay identical.  (A run whose trajectories outnumber the park
    slots keeps the excess in the lane pass, and which ones find the buffer
    full depends on timing, so such runs agree only to FP32 rounding.)"""
    import torch
    S = _system("c60_he", str(tmp_path), nprobe=131072)
    n = 131072
    eng = S.engine(precision=0, lanes_per_traj=32, park_steps=16)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    d_rnd = torch.from_numpy(S.predraw(n)).to(dev)
    ref, ref_stats = _reference(eng, n, d_rnd, stream, dev)
    assert ref_stats["parked"] > 65536
    out = _Run(n, dev)
    st, om, sp, vi = out.ptrs()
    stats = eng.run_device_noalloc(n, d_rnd.data_ptr(), n, st, om, sp, vi, stream.cuda_stream)
    torch.cuda.synchronize()
    assert out.same(ref)
    for key in STAT_KEYS:
        assert stats[key] == ref_stats[key], key
    eng.close()


def test_noalloc_watchdog_is_reported_without_stats(tmp_path):
    """A 1 ms watchdog: the call with stats == NULL returns at once, the
    following ccs_sync_stats reports the expiry (CCS_ERR_TIMEOUT), and the
    next call with a normal budget runs to completion on the same context."""
    import torch
    from massccs_b200 import engine as E
    S = _system("globule_n2", str(tmp_path))
    n = 3000
    eng = S.engine(precision=0, lanes_per_traj=32, watchdog_s=1e-3)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    d_rnd = torch.from_numpy(S.predraw(n)).to(dev)
    out = _Run(n, dev)
    st, om, sp, vi = out.ptrs()
    assert eng.run_device_noalloc(n, d_rnd.data_ptr(), n, st, om, None, None, stream.cuda_stream,
                                  want_stats=False) is None
    with pytest.raises(E.CcsError, match="watchdog"):
        eng.sync_stats()
    eng.close()
    eng = S.engine(precision=0, lanes_per_traj=32)
    stats = eng.run_device_noalloc(n, d_rnd.data_ptr(), n, st, om, None, None, stream.cuda_stream)
    assert stats["ncapped"] == 0
    assert stats["nfree"] + stats["nscatter"] + stats["nlost"] == n
    eng.close()


def test_noalloc_rejects_oversized_runs(tmp_path):
    from massccs_b200 import engine as E
    S = _system("c60_he", str(tmp_path))
    eng = S.engine()
    L = E.load_library()
    fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.ccs_run_device_noalloc(eng._h, (1 << 18) + 1, fake, (1 << 18) + 1, fake, fake, None, None, None, None)
    assert rc == -1  # CCS_ERR_INVALID
    assert b"262144" in L.ccs_last_error(eng._h)
    eng.close()
