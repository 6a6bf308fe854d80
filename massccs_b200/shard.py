"""Trajectory sharding over ranks (one process per GPU).

Trajectories are independent and the reference draws their random numbers
in global trajectory order j (src/System.cpp:184-197), so a run splits into
contiguous j-ranges with no exchange while the trajectories run. The ranks
meet once, at the end: the per-trajectory status and 1-cos(chi) arrays are
gathered to every rank in global order and reduced there with the
reference's fixed-order per-iteration sums (src/System.cpp:287-321), so the
CCS is bit-identical for any number of ranks.

The process group is the caller's (`nccl` on GPUs, `gloo` on CPU); the only
collective is one all-gather of 9 bytes per trajectory.
"""
import numpy as np


def shard_range(ntraj, rank, world):
    """Contiguous [start, stop) of global trajectory indices for `rank`; the
    first ntraj % world ranks take one more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(int(ntraj), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def local_rnd(rnd, rank, world):
    """This rank's columns of the 9-row pre-draw (a view, rows keep their stride)."""
    s, e = shard_range(rnd.shape[1], rank, world)
    return rnd[:, s:e]


def gather_results(status, one_minus_cos, ntraj, group=None):
    """All-gather every rank's (status, 1-cos chi) shard into global order.

    status: int8[local], one_minus_cos: float64[local] for this rank's
    shard_range. Returns (int8[ntraj], float64[ntraj]) on every rank.
    """
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    s, e = shard_range(ntraj, rank, world)
    if len(status) != e - s or len(one_minus_cos) != e - s:
        raise ValueError(f"rank {rank}: expected {e - s} results, got {len(status)}")
    width = -(-int(ntraj) // world)  # the largest shard
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    st = torch.full((width,), -1, dtype=torch.int8, device=dev)
    om = torch.zeros(width, dtype=torch.float64, device=dev)
    st[: e - s] = torch.as_tensor(np.ascontiguousarray(status, dtype=np.int8), device=dev)
    om[: e - s] = torch.as_tensor(np.ascontiguousarray(one_minus_cos, dtype=np.float64), device=dev)
    sts = [torch.empty_like(st) for _ in range(world)]
    oms = [torch.empty_like(om) for _ in range(world)]
    dist.all_gather(sts, st, group=group)
    dist.all_gather(oms, om, group=group)
    out_s = np.empty(ntraj, dtype=np.int8)
    out_o = np.empty(ntraj, dtype=np.float64)
    for r in range(world):
        a, b = shard_range(ntraj, r, world)
        out_s[a:b] = sts[r][: b - a].cpu().numpy()
        out_o[a:b] = oms[r][: b - a].cpu().numpy()
    return out_s, out_o


def sharded_ccs(status, one_minus_cos, niter, nprobe, bmax, group=None):
    """Gather the shards and apply the reference's reduction; returns the
    same dict as massccs_b200.host.reduce on every rank."""
    from . import host
    ntraj = int(niter) * int(nprobe)
    st, om = gather_results(status, one_minus_cos, ntraj, group)
    return host.reduce(niter, nprobe, st, om, bmax)
