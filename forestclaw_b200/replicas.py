"""Multi-GPU layout of the benchmark: independent replicas.

The patch update shards by Morton ranges with a ghost-patch exchange per ghost
update in the reference (MPI); this package runs one independent solve per
GPU (weak scaling), so the only cross-rank operations are the barrier around
the timed region and two reductions of the measurement: the slowest rank's
device time and the total number of cell updates.
"""
from __future__ import annotations


def aggregate(ms_local: float, cells_local: int, dist=None):
    """(max over ranks of ms_local, sum over ranks of cells_local).  `dist` is
    torch.distributed (initialised) or None for one process."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms_local), int(cells_local)
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=dev)
    c = torch.tensor([int(cells_local)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(c.item())


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s replica (different synthetic data per rank)."""
    return base + 1000 * rank
