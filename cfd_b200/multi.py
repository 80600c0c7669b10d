"""Multi-GPU plumbing of the benchmark: the pressure path does not shard (one system per GPU),
so N ranks run independent replicas with no collective on the data path. The only
communication is the timing summary: the slowest rank's device time defines the job time."""
from __future__ import annotations


def replica_summary(local_ms: float, steps: int, world: int):
    """Returns (max_ms_over_ranks, total solves/s over all ranks). Uses torch.distributed
    (NCCL on GPUs, gloo on CPU) when more than one rank is running."""
    ms = float(local_ms)
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = dist.get_backend()
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, world * steps / (ms / 1e3)
