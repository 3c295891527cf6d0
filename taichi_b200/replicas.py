"""Replica plumbing for multi-GPU runs of the multiply.

The multiply does not shard (one matrix, one GPU), so N GPUs run N
independent replicas, one process per GPU, launched by torchrun.  The only
cross-process steps are a barrier around the timed region and the maximum of
the ranks' device times (the slowest replica bounds the whole job).  No data
moves between GPUs.

`backend` is "nccl" for GPU runs and "gloo" for the CPU tests of this module.
"""
import datetime
import os


def env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=120):
    """Joins the process group when there is more than one rank (GPU backends
    bind the rank's device first).  Returns (rank, world_size, local_rank)."""
    rank, world, local_rank = env()
    if world > 1:
        import torch
        if backend == "nccl":
            torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local_rank


def barrier(world):
    if world > 1:
        import torch
        torch.distributed.barrier()


def max_over_ranks(value, world, device=None):
    """The largest of the ranks' `value` (every rank gets it)."""
    if world <= 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def finish(world):
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
