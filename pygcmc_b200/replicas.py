"""Multi-GPU layout: replicas only.

A single GCMC system does not shard usefully (one MC step is at most 1024
trial poses against a few MB of state), so N processes -- one per GPU,
launched by torchrun -- each advance their own independent replica(s) and
exchange nothing on the data path.  The only collectives are host-side
bookkeeping: a barrier around timed regions and a max over ranks of the
measured time (the job's time is the slowest rank's).  These helpers work for
the ``nccl`` backend (GPU tensors) and for ``gloo`` (CPU tensors, used by the
tests).
"""
import datetime
import os


def env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 300):
    """Initialise the process group when running under torchrun (world size > 1)."""
    ws, _, _ = env()
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws


def finalize():
    ws, _, _ = env()
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


def replica_seed(base: int, rank: int, stride: int = 1) -> int:
    """Seed of rank `rank`'s replica: independent chains per rank."""
    return int(base) + stride * int(rank)


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float, ws: int) -> float:
    """The maximum of a per-rank scalar (e.g. the timed region's milliseconds)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, ws: int) -> float:
    """The sum of a per-rank scalar (e.g. MC steps done)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
