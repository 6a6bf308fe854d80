"""Sharding of one run over ranks (CPU, gloo, world sizes 2 and 3).

Each rank runs only its contiguous range of trajectories (here through the
oracle, on its own columns of the pre-draw); the gathered results and the
fixed-order reduction must equal the single-process run exactly, for even
and uneven splits.
"""
import os
import socket

import numpy as np
import pytest

from helpers import input_dict, workdir, write_input


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, json_path, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from oracle import pyoracle
        from massccs_b200 import shard
        s = pyoracle.OracleSystem(json_path)
        info = s.params
        n = info["nprobe"] * info["niter"]
        rnd = np.ascontiguousarray(shard.local_rnd(s.predraw(n), rank, world))
        res = s.run(rnd, nthreads=1)
        red = shard.sharded_ccs(res["status"], res["one_minus_cos"], info["niter"], info["nprobe"], info["bmax"])
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), omega=red["omega"], ccs=red["ccs"], err=red["err"],
                 nfree=red["nfree"], nscatter=red["nscatter"], nlost=red["nlost"])
    finally:
        dist.destroy_process_group()


def _host_worker(rank, world, port, json_path, out_dir):
    """The product's host C-ABI on a rank: mh_open, mh_predraw of the whole
    job, this rank's slice (trajectories through the oracle, no GPU here),
    then the gather and mh_reduce."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from oracle import pyoracle
        from massccs_b200 import host, shard
        S = host.System(json_path)
        n = S.info["nprobe"] * S.info["niter"]
        rnd = np.ascontiguousarray(shard.local_rnd(S.predraw(n), rank, world))
        res = pyoracle.OracleSystem(json_path).run(rnd, nthreads=1)
        red = shard.sharded_ccs(res["status"], res["one_minus_cos"], S.info["niter"], S.info["nprobe"],
                                S.info["bmax"])
        np.savez(os.path.join(out_dir, f"host{rank}.npz"), omega=red["omega"], ccs=red["ccs"], err=red["err"])
    finally:
        dist.destroy_process_group()


def test_sharded_host_api_equals_single_process(oracle, tmp_path):
    """Ranks driving the product's host library (pre-draw and reduction in
    C++) give the single-process CCS bit for bit (N2, uneven split)."""
    import torch.multiprocessing as mp
    from massccs_b200 import host
    d = workdir()
    p = write_input(d, input_dict("c60.xyz", "N2", 6, nprobe=25, niter=4))
    S = host.System(p)
    n = 100
    full = oracle.OracleSystem(p).run(S.predraw(n), nthreads=1)
    ref = host.reduce(4, 25, full["status"], full["one_minus_cos"], S.info["bmax"])
    mp.start_processes(_host_worker, args=(3, _free_port(), p, str(tmp_path)), nprocs=3, join=True,
                       start_method="spawn")
    for r in range(3):
        got = np.load(tmp_path / f"host{r}.npz")
        np.testing.assert_array_equal(got["omega"], ref["omega"])
        assert float(got["ccs"]) == ref["ccs"] and float(got["err"]) == ref["err"]


def test_shard_range_covers_every_trajectory():
    from massccs_b200 import shard
    for n in (0, 1, 7, 300, 300001):
        for w in (1, 2, 3, 8):
            spans = [shard.shard_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - s for s, e in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shard_range(10, 2, 2)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_run_equals_single_process(oracle, world, tmp_path):
    import torch.multiprocessing as mp
    d = workdir()
    p = write_input(d, input_dict("c60.xyz", "He", 4, nprobe=40, niter=5))
    s = oracle.OracleSystem(p)
    n = 200
    full = s.run(s.predraw(n), nthreads=1)
    ref = oracle.reduce(5, 40, full["status"], full["one_minus_cos"], s.params["bmax"])
    mp.start_processes(_worker, args=(world, _free_port(), p, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npz")
        np.testing.assert_array_equal(got["omega"], ref["omega"])
        np.testing.assert_array_equal(got["nfree"], ref["nfree"])
        assert float(got["ccs"]) == ref["ccs"] and float(got["err"]) == ref["err"]


def _lost_rank_worker(rank, world, port, out_dir):
    import datetime
    import time
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=3))
    from massccs_b200 import shard
    if rank == 1:  # this rank fails before the gather: it never joins the collective
        time.sleep(1.0)
        open(os.path.join(out_dir, "rank1_left"), "w").close()
        os._exit(0)
    s, e = shard.shard_range(20, rank, world)
    t0 = time.time()
    try:
        shard.sharded_ccs(np.ones(e - s, dtype=np.int8), np.zeros(e - s), 2, 10, 10.0)
        result = "completed"
    except Exception as exc:  # the surviving rank learns of the loss from the timeout
        result = f"error after {time.time() - t0:.1f} s: {type(exc).__name__}"
    open(os.path.join(out_dir, "rank0"), "w").write(result)
    os._exit(0)


def test_lost_rank_ends_the_gather_with_an_error(tmp_path):
    """A rank that leaves before the final gather: the other rank's collective
    ends with an error within the process group's timeout instead of waiting
    forever (failure made on the host, CPU ranks)."""
    import torch.multiprocessing as mp
    mp.start_processes(_lost_rank_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    assert (tmp_path / "rank1_left").exists()
    result = (tmp_path / "rank0").read_text()
    assert result.startswith("error after"), result
    assert float(result.split()[2]) < 60
