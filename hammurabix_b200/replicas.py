"""Multi-process plumbing of the benchmark: one process per GPU.  In
replica mode each rank runs an independent copy of the workload (no
exchange); the pixel-sharded pass (sharded.py) uses the same process group
for its per-shell Faraday-depth all-reduce (integrator.cc:78-86).

Timing follows the contract of the benchmark: every rank brackets its timed
region with a barrier, the job time is the maximum over ranks, and the
throughput is the work of all ranks over that time (weak scaling).
"""
import datetime
import os


def env():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=600, device=None):
    """Join the process group when WORLD_SIZE > 1; returns (ws, rank, local).
    A short timeout makes a rank that never arrives fail the others' next
    collective instead of hanging them."""
    ws, rank, local = env()
    if ws > 1:
        import torch.distributed as dist
        kw = {}
        if device is not None:
            kw["device_id"] = device
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws, device="cpu"):
    """The maximum of a per-rank float over all ranks."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def throughput(units_per_rank, ws, seconds):
    """Whole-job throughput: every rank processed units_per_rank in at most
    `seconds` (the max over ranks)."""
    return ws * units_per_rank / seconds


def finish(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
