"""Replica plumbing for running the filter path on several GPUs of a node.

Frames and streams are independent, so N GPUs run N replicas with no
collective on the data path: each rank filters its own share of the work,
and the only cross-rank traffic is control (a barrier around the timed
region and one max-reduction of each rank's elapsed time).  The same code
runs over NCCL on GPUs and over gloo on CPU (the tests use the latter).
"""
import datetime
import os

import torch
import torch.distributed as dist


def env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend, timeout_s=120):
    """Join the process group when WORLD_SIZE > 1 (a short timeout, so a
    rank that never arrives ends the others' collectives with an error)."""
    rank, world, _ = env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, init_method="env://", timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world


def finish():
    if dist.is_initialized():
        dist.destroy_process_group()


def barrier():
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value, device="cpu"):
    """The largest `value` over all ranks (timings: the job takes as long as
    its slowest replica)."""
    if not (dist.is_initialized() and dist.get_world_size() > 1):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items, rank, world):
    """This rank's share of independent work items (round robin, so mixed
    sizes spread evenly)."""
    return items[rank::world]


def aggregate(units, ms, device="cpu"):
    """Whole-job totals of one timed region: (units summed over the ranks,
    the largest elapsed milliseconds of any rank, the number of ranks that
    reported).  Every rank contributes what it actually processed, so the
    job's rate is units / (ms / 1e3) whatever the number of ranks."""
    if not (dist.is_initialized() and dist.get_world_size() > 1):
        return float(units), float(ms), 1
    t = torch.tensor([float(units), 1.0], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    m = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(t[0].item()), float(m[0].item()), int(round(t[1].item()))


def check_world(requested):
    """The number of processes must be the number of GPUs asked for: one
    process per GPU, started by torchrun.  A single process asked for N > 1
    GPUs is an error (it would otherwise report one GPU's work as N's)."""
    _, world, _ = env()
    if world != requested:
        raise SystemExit(f"--gpus {requested} needs {requested} processes (one per GPU, e.g. "
                         f"python -m torch.distributed.run --nproc-per-node {requested} bench.py --gpus {requested}); "
                         f"WORLD_SIZE is {world}")
