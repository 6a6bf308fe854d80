"""ccs_run_device_noalloc against ccs_run_device (GPU).

The no-allocation entry point serves callers that cannot allocate device
memory while they run (a host whose allocator owns the device heap, a service
with a fixed memory budget, code where an allocation would synchronise the
device): it keeps the run's scratch in the library's static device array.  It
must return what the allocating entry point returns for the same inputs, and
keep doing so on back-to-back calls (the array keeps the previous call's
contents, so everything that must start at zero is cleared by each call).

This file sorts last so that a stopping run has executed every other test
first; it also passes on its own in a fresh process, where its first call is
the one that looks up the array's device address.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(kind, tmp):
    from massccs_b200 import host, synth
    if kind == "c60_he":
        p = synth.c60_he(os.path.join(tmp, kind), nprobe=20000, niter=1)
    else:
        p = synth.globule_n2(os.path.join(tmp, kind), nprobe=3000, niter=1)
    return host.System(p)


@pytest.mark.parametrize("kind,park", [("c60_he", 256), ("globule_n2", 512)])
@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_run_device_twice(tmp_path, kind, park, precision):
    import torch
    S = _system(kind, str(tmp_path))
    n = S.info["nprobe"] * S.info["niter"]
    eng = S.engine(precision=precision, lanes_per_traj=32, park_steps=park)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    d_rnd = torch.from_numpy(S.predraw(n)).to(dev)

    def buffers():
        return (torch.full((n,), -1, dtype=torch.int8, device=dev),
                torch.full((n,), -1.0, dtype=torch.float64, device=dev),
                torch.zeros(n, dtype=torch.int32, device=dev))

    st_a, om_a, sp_a = buffers()
    eng.run_device(n, d_rnd.data_ptr(), n, st_a.data_ptr(), om_a.data_ptr(), sp_a.data_ptr(), 0,
                   stream.cuda_stream)
    ref_stats = eng.sync_stats()
    assert ref_stats["parked"] > 0  # the park buffer in the scratch is exercised
    for call in range(2):
        st_b, om_b, sp_b = buffers()
        stats = eng.run_device_noalloc(n, d_rnd.data_ptr(), n, st_b.data_ptr(), om_b.data_ptr(), sp_b.data_ptr(),
                                       0, stream.cuda_stream)
        torch.cuda.synchronize()
        assert torch.equal(st_a, st_b), call
        assert torch.equal(sp_a, sp_b), call
        assert float((om_a - om_b).abs().max()) <= 1e-7, call
        for key in ("nfree", "nscatter", "nlost", "ncapped", "steps", "parked"):
            assert stats[key] == ref_stats[key], (call, key)
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
