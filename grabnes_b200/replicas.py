"""Replicas of a recursion job over GPUs: one process per GPU, launched by torchrun.

The recursion has no exchange step: every rank holds the whole Hamiltonian and runs its own random-phase
vectors (its own seed range), so the units of work are shared out with no collective during the
recursion.  The only exchange is at the end of a job, where the ranks' averaged densities of states are
combined (one all-reduce), and for timing, where a job's duration is the maximum over ranks.  The same
helpers run over NCCL on GPUs and over gloo on CPU (tests).
"""
import datetime
import os

import numpy as np

SEED_STRIDE = 1000


def world():
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=300):
    """Join the process group when there is more than one rank; returns (ws, rank, local)."""
    ws, rank, local = world()
    if ws > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return ws, rank, local


def shard_units(n_units, rank, ws):
    """The units of a sweep that rank runs: unit u on rank u % ws (the drop-in driver's rule for its
    (field, Haldane phase) units, GRABNES_RANK / GRABNES_NRANKS)."""
    return [u for u in range(n_units) if u % ws == rank]


def seed_of(base, rank):
    """Seed of a rank's random-phase vectors: disjoint streams per rank (the reference seeds by SeedValue)."""
    return base + SEED_STRIDE * rank


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x, ws):
    """The largest value of x over all ranks (device time of a job: the slowest rank)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def mean_over_ranks(arr, ws):
    """Element-wise mean of a float64 array over the ranks (the combined DOS of all replicas)."""
    a = np.ascontiguousarray(arr, np.float64)
    if ws == 1:
        return a.copy()
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(a.copy()).to(_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy() / ws


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def finish(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
