"""Multi-GPU plumbing of the field path: one process per GPU, the mesh
replicated on every GPU, the observation points split between the ranks.

Observation points are independent (get_field.h:49 parallelises over them), so
the ranks share no data: there is no collective on the data path. The process
group (NCCL between GPUs, gloo for CPU-only runs) carries only the barrier
around timed regions and the max-over-ranks of their times.
"""
import datetime
import os

import numpy as np


def env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(ws, local, backend=None, timeout_s=300):
    """Joins the process group when ws > 1: NCCL when a GPU is visible (the
    rank's device made current first), gloo otherwise. Returns the backend."""
    if ws <= 1:
        return None
    import torch
    import torch.distributed as dist

    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return backend


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(ws, v, local=0):
    """The largest of every rank's v (the job's time is its slowest rank's)."""
    if ws <= 1:
        return v
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", local) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(n, ws, rank):
    """[lo, hi) of n items for `rank`: contiguous blocks whose sizes differ by
    at most one (a fixed point set split between ranks: strong scaling)."""
    base, extra = divmod(n, ws)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def rank_points(cells, rank, n_far=18000, n_near=2000):
    """The headline workload's point set of one rank (weak scaling: every rank
    evaluates its own set of the same distribution against the replicated
    mesh). Rank 0 has the single-GPU set (seed 1); rank r > 0 draws with seed
    1000 + r: n_far points on 2-5 m shells, n_near points 0.02-0.1 m above
    random cells."""
    from . import workloads as W

    if rank == 0:
        return W.config2(n_far, n_near)["pts"]
    rng = np.random.default_rng(1000 + rank)
    return np.concatenate([W.shell_points(n_far, 2.0, 5.0, rng), W.near_points(cells, n_near, 0.02, 0.1, rng)])
