"""World-size-2 checks of the sharded (row-block) GEMM host logic on CPU with gloo.

Each rank computes its row block of C (the CPU oracle stands in for the
per-GPU GEMM), the blocks are all-gathered, and every rank compares the
assembled C and the all-reduced d(alpha) with the unsharded computation.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, m, n, k, errq):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        from jlc_b200 import shard
        from oracle import oracle as O
        A = O.uniform((m, k), 1)
        B = O.uniform((k, n), 2)
        C = O.uniform((m, n), 3)
        r0, r1 = shard.local_block(rank, world, m, align=16)
        local = O.gemm_fmachain(A[r0:r1], B, C[r0:r1], 1.5, 0.5)
        full = shard.gather_rows(torch.from_numpy(local), m, world, align=16).numpy()
        want = O.gemm_fmachain(A, B, C, 1.5, 0.5)
        assert np.array_equal(full, want), "gathered row blocks differ from the unsharded GEMM"
        # adjoint: d(alpha) = <A, dC B^T> splits over row blocks of A and dC
        dC = O.uniform((m, n), 4)
        G = dC[r0:r1] @ B.T
        da = shard.allreduce_sum(float(np.sum(A[r0:r1] * G)))
        da_full = float(np.sum(A * (dC @ B.T)))
        assert abs(da - da_full) <= 1e-9 * max(1.0, abs(da_full))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # surfaced to the parent
        errq.put(f"rank {rank}: {e!r}")
        raise


def _bench_worker(rank, world, port, rows_per_rank, n, k, errq):
    """The benchmark's sharded product: rank r holds rows partition_rows(...)[r]
    of one global A (seeded per block by shard.block_seed) and the same B; the
    gathered row blocks equal the product of the whole A, built from the same
    block seeds on one rank."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        from jlc_b200 import shard
        from oracle import oracle as O
        gm = world * rows_per_rank
        parts = shard.partition_rows(gm, world, align=16)
        r0, r1 = parts[rank]
        assert r1 - r0 == rows_per_rank
        block = lambda a0, a1: O.uniform((a1 - a0, k), shard.block_seed(20260604, a0) % (2 ** 31))
        B = O.uniform((k, n), 20260605)
        local = O.gemm_fmachain(block(r0, r1), B, np.zeros((r1 - r0, n)), 1.0, 0.0)
        full = shard.gather_rows(torch.from_numpy(local), gm, world, align=16).numpy()
        A_global = np.concatenate([block(a0, a1) for (a0, a1) in parts], axis=0)
        want = O.gemm_fmachain(A_global, B, np.zeros((gm, n)), 1.0, 0.0)
        assert np.array_equal(full, want), "row blocks of the sharded product differ from the whole product"
        # distinct blocks: no two ranks multiply the same rows
        firsts = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(firsts, torch.tensor([float(local[0, 0])], dtype=torch.float64))
        assert len({float(x) for x in firsts}) == world
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # surfaced to the parent
        errq.put(f"rank {rank}: {e!r}")
        raise


def test_bench_sharded_product_world2_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, world, port, 48, 40, 36, errq)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    errors = []
    while not errq.empty():
        errors.append(errq.get())
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a gloo rank did not finish")
    assert not errors, errors
    assert all(p.exitcode == 0 for p in procs)


def test_block_seed_distinct_and_stable():
    from jlc_b200 import shard
    seeds = {shard.block_seed(20260604, r0) for r0 in range(0, 8 * 8192, 8192)}
    assert len(seeds) == 8
    assert shard.block_seed(20260604, 0) == shard.block_seed(20260604, 0)


def test_partition_rows_covers_and_aligns():
    from jlc_b200 import shard
    for m, world in [(8192, 2), (8192, 8), (1000, 3), (5, 4), (0, 2)]:
        parts = shard.partition_rows(m, world, align=128)
        assert len(parts) == world
        assert parts[0][0] == 0 and parts[-1][1] == m
        for (a0, a1), (b0, b1) in zip(parts, parts[1:]):
            assert a1 == b0
        for (r0, r1) in parts:
            if r1 > r0:  # non-empty blocks start on a tile boundary
                assert r0 % 128 == 0


def test_row_block_gemm_world2_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, 90, 70, 50, errq)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    errors = []
    while not errq.empty():
        errors.append(errq.get())
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a gloo rank did not finish")
    assert not errors, errors
    assert all(p.exitcode == 0 for p in procs)
