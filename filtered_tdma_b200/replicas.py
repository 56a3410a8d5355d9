"""Multi-GPU use of the solver: one process per GPU, systems sharded by rank.

The systems of a batch are independent, so a batch splits over GPUs by system
with no communication on the data path (the reference's multi-rank split of one
system's rows is not needed on B200, which holds every shape of the reference).
Each rank solves its own contiguous [n_row x n_sys_local] batch; the only
collective is the max-over-ranks reduction of a timing, for reporting.

The split is the reference's block split (libs/pascal_tdma/cpu/para_range.cpp:4-10),
rounded to multiples of `align` systems so that every rank's row stride keeps
the 16-byte alignment the TMA paths need (align = 2 for FP64, 4 for FP32).
"""
from __future__ import annotations


def local_systems(n_sys: int, rank: int, world: int, align: int = 2) -> tuple[int, int]:
    """(first system, number of systems) owned by `rank` of `world`."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    units = (n_sys + align - 1) // align
    base, rem = divmod(units, world)
    first_u = rank * base + min(rank, rem)
    count_u = base + (1 if rank < rem else 0)
    first = min(first_u * align, n_sys)
    last = min((first_u + count_u) * align, n_sys)
    return first, last - first


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (the value
    itself without one).  Works on gloo (CPU tensors) and nccl (device tensors)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(rows_per_rank: int, world: int, max_ms: float) -> float:
    """Rows per second of the whole job: every rank's rows over the slowest rank's time."""
    return world * rows_per_rank / (max_ms * 1e-3)
