"""Row-block sharding of one GEMM across GPUs (one process per GPU).

C = alpha*A*B + beta*C splits into row blocks with no reduction: rank r owns
rows [r0, r1) of C, needs the same rows of A and all of B, and runs an
ordinary single-GPU GEMM on them.  Nothing crosses NVLink on the data path;
only optional collection steps (all-gather of C blocks, the scalar all-reduce
of the adjoint's d(alpha)/d(beta)) use torch.distributed, with NCCL on GPUs
and gloo on CPUs.
"""
from __future__ import annotations


def partition_rows(m: int, world: int, align: int = 128):
    """[(r0, r1)] per rank: contiguous, balanced row blocks whose boundaries
    fall on multiples of `align` (the GEMM tile height) where possible."""
    if world < 1:
        raise ValueError("world must be >= 1")
    units = (m + align - 1) // align
    out, start = [], 0
    for r in range(world):
        n_units = units // world + (1 if r < units % world else 0)
        end = min(m, start + n_units * align)
        out.append((start, end))
        start = end
    return out


def block_seed(base: int, r0: int) -> int:
    """Seed of the row block of a sharded input that starts at global row r0:
    the blocks of one global matrix get distinct, reproducible streams."""
    return (base * 1_000_003 + r0) % (2 ** 63)


def local_block(rank: int, world: int, m: int, align: int = 128):
    return partition_rows(m, world, align)[rank]


def gather_rows(local, m: int, world: int, align: int = 128):
    """All-gather row blocks (torch tensors, rows x cols) into the full m x cols
    matrix on every rank.  Blocks may differ in height, so they are padded to
    the largest block for the collective."""
    import torch
    import torch.distributed as dist
    parts = partition_rows(m, world, align)
    hmax = max(r1 - r0 for r0, r1 in parts)
    cols = local.shape[1]
    pad = torch.zeros((hmax, cols), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad)
    return torch.cat([b[:r1 - r0] for b, (r0, r1) in zip(bufs, parts)], dim=0)


def allreduce_sum(value: float, device="cpu") -> float:
    """Sum one scalar over ranks (the adjoint's d(alpha) / d(beta) when dA is
    sharded by rows)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
