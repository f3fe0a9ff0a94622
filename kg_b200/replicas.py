"""Independent solves on several GPUs: one process per GPU, no exchange step.

The reference decomposes one solve into r-slabs over MPI ranks
(MoL/lines_method_lib.f90:475-505, mpi/mpi_lib.f90); here a solve lives whole
on one GPU, and several GPUs run independent solves ("replicas", or the
requests of a serving queue split between processes).  The only collective is
the max over ranks of a timing, which is measurement plumbing.  These helpers
hold that host logic so it is testable on the CPU with the gloo backend.
"""
from __future__ import annotations

import datetime
import os


def rank_env():
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)"""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world, backend="nccl", timeout_s=120):
    """join the process group when world > 1 (a short timeout, so a rank that
    never joins ends the others' first collective with an error)"""
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def finish(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value, world, device="cpu"):
    """the largest value over all ranks (every rank gets it)"""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(base, rank):
    """each replica solves its own seeded initial data"""
    return int(base) + int(rank)


def job_rate(units_per_rank, world, ms):
    """whole-job throughput: every rank processed units_per_rank in at most ms"""
    return world * units_per_rank / (ms / 1e3)


def dispatch(items, world, rank):
    """this rank's share of a request list (round robin; disjoint, covering)"""
    return list(items)[rank::world]
