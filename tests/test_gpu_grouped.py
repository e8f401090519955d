"""GPU parity of grouped launches (many uneven GEMMs in one persistent launch).

Mirrors the reference's batched use: the TINY/SMALL dispatch shapes
(GemmDispatch.java:76-106) and blocked-factorisation updates issued as many
independent gemm calls.  Every problem's result must sit inside the FP64
componentwise bound of the double-double oracle.
"""
import os

import numpy as np
import pytest

from parity import assert_fp64_bound

pytestmark = pytest.mark.gpu


def make_batch(oracle, shapes, seed, layouts=None, alphas=None, betas=None):
    """Allocates every operand in one device arena; returns (problems, host copies, arena)."""
    import torch
    rng = np.random.default_rng(seed)
    host, sizes = [], []
    for idx, (m, n, k) in enumerate(shapes):
        la, lb = layouts[idx] if layouts else (int(rng.integers(0, 2)), int(rng.integers(0, 2)))
        alpha = alphas[idx] if alphas else float(rng.uniform(-2, 2))
        beta = betas[idx] if betas else float(rng.uniform(-2, 2))
        A = oracle.uniform((m, k), seed * 1000 + 3 * idx)
        B = oracle.uniform((k, n), seed * 1000 + 3 * idx + 1)
        C = oracle.uniform((m, n), seed * 1000 + 3 * idx + 2)
        host.append((m, n, k, la, lb, alpha, beta, A, B, C))
        sizes.append(m * k + k * n + m * n)
    arena = torch.zeros(int(sum(sizes)) + 8, dtype=torch.float64, device="cuda")
    probs, off = [], 0
    base = arena.data_ptr()
    for (m, n, k, la, lb, alpha, beta, A, B, C) in host:
        a_store = A if la == 0 else np.ascontiguousarray(A.T)
        b_store = B if lb == 0 else np.ascontiguousarray(B.T)
        pa = off
        arena[pa:pa + m * k] = torch.from_numpy(a_store.ravel())
        pb = pa + m * k
        arena[pb:pb + k * n] = torch.from_numpy(b_store.ravel())
        pc = pb + k * n
        arena[pc:pc + m * n] = torch.from_numpy(C.ravel())
        off = pc + m * n
        probs.append(dict(m=m, n=n, k=k, layout_a=la, layout_b=lb,
                          lda=max(1, a_store.shape[1]), ldb=max(1, b_store.shape[1]), ldc=max(1, n),
                          alpha=alpha, beta=beta, a=base + 8 * pa, b=base + 8 * pb, c=base + 8 * pc))
    return probs, host, arena


def check_batch(oracle, probs, host, arena, label):
    flat = arena.cpu().numpy()
    worst = 0.0
    for p, (m, n, k, la, lb, alpha, beta, A, B, C) in zip(probs, host):
        if m == 0 or n == 0:
            continue
        off = (p["c"] - arena.data_ptr()) // 8
        got = flat[off:off + m * n].reshape(m, n)
        worst = max(worst, assert_fp64_bound(f"{label} {m}x{n}x{k}", np.ascontiguousarray(got), A, B, C,
                                             alpha, beta))
    return worst


def mixed_shapes(rng, count):
    shapes = []
    for i in range(count):
        r = rng.random()
        if r < 0.3:
            s = int(rng.integers(2, 5))
            shapes.append((s, s, s))
        elif r < 0.5:
            shapes.append(tuple(int(x) for x in rng.integers(1, 49, size=3)))
        else:
            shapes.append(tuple(int(x) for x in np.exp(rng.uniform(np.log(8), np.log(300), size=3)).round()))
    return shapes


def test_grouped_mixed_batch(ctx, oracle):
    rng = np.random.default_rng(3)
    shapes = mixed_shapes(rng, 300) + [(0, 5, 3), (5, 0, 3), (7, 9, 0), (1, 1, 1), (1, 200, 70), (200, 1, 70)]
    alphas = [float(x) for x in rng.uniform(-2, 2, size=len(shapes))]
    alphas[10] = 0.0  # alpha == 0: A and B are not read
    probs, host, arena = make_batch(oracle, shapes, 5, alphas=alphas)
    rep = ctx.dgemm_grouped_device(probs)
    assert rep["kernel"] == 4
    check_batch(oracle, probs, host, arena, "grouped")


def test_grouped_small_tile_build_many_items(ctx, oracle):
    """Many small problems (max(m, n) <= 48): several items per warp, odd
    leading dimensions (8-byte copies) beside even ones, edge tiles trimmed to
    16 rows and to 8-column blocks, and a few long products whose k-blocks
    wrap the slot ring many times."""
    rng = np.random.default_rng(17)
    shapes = [tuple(int(x) for x in rng.integers(1, 49, size=3)) for _ in range(1400)]
    shapes += [(32, 32, 2000), (48, 17, 1029), (5, 40, 777), (40, 40, 16), (33, 1, 100)]
    probs, host, arena = make_batch(oracle, shapes, 19)
    plan = ctx.grouped_plan(probs)
    assert plan.info()["work_items"] > 1400
    plan.run()
    ctx.synchronize()
    check_batch(oracle, probs, host, arena, "small-tile build")
    plan.close()


def test_grouped_long_k_both_ring_depths(ctx, oracle, tmp_path):
    """Problems of several tiles each with k long enough that one item's
    k-blocks wrap the slot ring, beta 0 / 1 / other and alpha == 1 (the
    unscaled path), run with both ring depths: the autotuner records its
    choice in the cache, the cache is rewritten to the other depth and a plan
    made without tuning reads it back."""
    import torch
    shapes = [(130, 70, 3000), (64, 64, 16), (200, 90, 257), (49, 300, 1), (100, 100, 100)] + \
             [(20, 30, 40)] * 50
    betas = [0.0, 1.0, -0.5, 0.0, 2.0] + [0.0] * 50
    cache = tmp_path / "tune.txt"
    os.environ["JLCGPU_TUNE_CACHE"] = str(cache)
    try:
        probs, host, arena = make_batch(oracle, shapes, 23, alphas=[1.0] * len(shapes), betas=betas)
        saved = arena.clone()
        plan = ctx.grouped_plan(probs, autotune=True)
        plan.run()
        ctx.synchronize()
        check_batch(oracle, probs, host, arena, "tuned depth")
        plan.close()
        key, depth = cache.read_text().split()
        other = "3" if depth == "2" else "2"
        cache.write_text(f"{key} {other}\n")
        arena.copy_(saved)
        torch.cuda.synchronize()
        plan = ctx.grouped_plan(probs)
        plan.run()
        ctx.synchronize()
        check_batch(oracle, probs, host, arena, f"depth {other}")
        plan.close()
    finally:
        os.environ.pop("JLCGPU_TUNE_CACHE", None)


def test_grouped_plan_graph_replay_sees_new_data(ctx, oracle):
    import torch
    rng = np.random.default_rng(7)
    shapes = mixed_shapes(rng, 120)
    probs, host, arena = make_batch(oracle, shapes, 9, betas=[0.0] * len(shapes))
    plan = ctx.grouped_plan(probs, graph=True)
    info = plan.info()
    assert info["work_items"] > 0 and info["flops"] > 0
    plan.run()
    ctx.synchronize()
    check_batch(oracle, probs, host, arena, "graph run 1")
    # new A data written in place; the same plan (same pointers) replays
    host2 = []
    for p, (m, n, k, la, lb, alpha, beta, A, B, C) in zip(probs, host):
        A2 = -2.0 * A
        a_store = A2 if la == 0 else np.ascontiguousarray(A2.T)
        off = (p["a"] - arena.data_ptr()) // 8
        arena[off:off + m * k] = torch.from_numpy(a_store.ravel())
        host2.append((m, n, k, la, lb, alpha, beta, A2, B, C))
    torch.cuda.synchronize()
    plan.run()
    ctx.synchronize()
    check_batch(oracle, probs, host2, arena, "graph run 2")
    plan.close()


def test_grouped_autotune_writes_cache(ctx, oracle, tmp_path):
    cache = tmp_path / "tune.txt"
    os.environ["JLCGPU_TUNE_CACHE"] = str(cache)
    try:
        rng = np.random.default_rng(11)
        shapes = [tuple(int(x) for x in rng.integers(20, 48, size=3)) for _ in range(40)] + \
                 [tuple(int(x) for x in rng.integers(60, 260, size=3)) for _ in range(40)]
        probs, host, arena = make_batch(oracle, shapes, 13)
        plan = ctx.grouped_plan(probs, autotune=True)
        info = plan.info()
        # problems above 32 rows and columns run as 64 x 64 CTA tiles
        assert info["tile_small"] == 32 and info["tile_large"] == 64
        text = cache.read_text()
        assert "grouped-fp64|stages|k" in text
        assert text.split()[-1] in ("2", "3")
        plan.run()
        ctx.synchronize()
        check_batch(oracle, probs, host, arena, "autotuned")
        plan.close()
    finally:
        os.environ.pop("JLCGPU_TUNE_CACHE", None)


def test_grouped_cta_tiles_many_items(ctx, oracle):
    """Problems above 32 rows and 32 columns run as 64 x 64 items of four
    32 x 32 quadrants on CTAs of two copy warps and four DMMA warps; the rest
    (at most 32 rows or columns) on warp tiles beside them.  Thousands of items (more than the
    persistent grid holds, so every CTA's record queue and slot ring wrap many
    times), all four operand layouts, odd and even leading dimensions (8- and
    16-byte copies), ragged edges in every quadrant, alpha == 0, k == 0 and
    k == 1, and a few long products; the same batch on the warp tiles alone
    (JLCGPU_GROUPED_CTA=0) as well.  Both inside the FP64 bound."""
    import torch
    rng = np.random.default_rng(41)
    shapes = [(int(rng.integers(33, 200)), int(rng.integers(33, 200)), int(rng.integers(1, 300)))
              for _ in range(700)]
    shapes += [(33, 33, 1), (64, 64, 16), (65, 97, 0), (200, 40, 2500), (40, 200, 1777), (129, 129, 129)]
    # at most 32 rows or at most 32 columns (warp tiles), 1 included
    shapes += [(int(rng.integers(1, 33)), int(rng.integers(33, 400)), int(rng.integers(1, 300))) for _ in range(150)]
    shapes += [(int(rng.integers(33, 400)), int(rng.integers(1, 33)), int(rng.integers(1, 300))) for _ in range(150)]
    shapes += [(1, 513, 40), (513, 1, 40), (32, 129, 1000), (129, 32, 1000)]
    layouts = [(i % 2, (i // 2) % 2) for i in range(len(shapes))]
    alphas = [float(x) for x in rng.uniform(-2, 2, size=len(shapes))]
    alphas[5] = 0.0
    betas = [float(x) for x in rng.uniform(-2, 2, size=len(shapes))]
    betas[7] = 0.0
    probs, host, arena = make_batch(oracle, shapes, 37, layouts=layouts, alphas=alphas, betas=betas)
    saved = arena.clone()
    plan = ctx.grouped_plan(probs, graph=True)
    info = plan.info()
    assert info["tile_large"] == 64 and info["work_items"] > 2000
    plan.run()
    ctx.synchronize()
    check_batch(oracle, probs, host, arena, "CTA tiles")
    # graph replay (the counters are reset inside the graph) on the first
    # run's results as C
    flat = arena.cpu().numpy()
    host2 = []
    for p, (m, n, k, la, lb, alpha, beta, A, B, C) in zip(probs, host):
        o = (p["c"] - arena.data_ptr()) // 8
        host2.append((m, n, k, la, lb, alpha, beta, A, B, flat[o:o + m * n].reshape(m, n).copy()))
    plan.run()
    ctx.synchronize()
    check_batch(oracle, probs, host2, arena, "CTA tiles, graph replay")
    plan.close()
    arena.copy_(saved)
    torch.cuda.synchronize()
    os.environ["JLCGPU_GROUPED_CTA"] = "0"
    try:
        plan = ctx.grouped_plan(probs)
    finally:
        os.environ.pop("JLCGPU_GROUPED_CTA", None)
    assert plan.info()["tile_large"] == 32
    plan.run()
    ctx.synchronize()
    check_batch(oracle, probs, host, arena, "warp tiles")
    plan.close()


def test_grouped_rejects_bad_problem(ctx):
    from jlc_b200 import IllegalArgumentException
    bad = [dict(m=4, n=4, k=4, layout_a=0, layout_b=0, lda=2, ldb=4, ldc=4, alpha=1.0, beta=0.0, a=8, b=8, c=8)]
    with pytest.raises(IllegalArgumentException):
        ctx.dgemm_grouped_device(bad)


def _per_problem_ozaki(ctx, probs, arena_before, base_ptr):
    """Each problem through the per-call Ozaki residue route on a copy of the
    arena as it was before the grouped run (problem pointers point into the
    arena at base_ptr); returns that copy after all of them."""
    import torch
    from jlc_b200 import JLC_PREC_OZAKI_CRT
    ref = arena_before.clone()
    shift = ref.data_ptr() - base_ptr
    for p in probs:
        if p["m"] == 0 or p["n"] == 0:
            continue
        ctx.dgemm_device(p["layout_a"], p["layout_b"], p["m"], p["n"], p["k"], p["alpha"], p["a"] + shift,
                         p["lda"], p["b"] + shift, p["ldb"], p["beta"], p["c"] + shift, p["ldc"],
                         precision=JLC_PREC_OZAKI_CRT)
    ctx.synchronize()
    torch.cuda.synchronize()
    return ref


def _on_residues(p):
    """Problems both routes compute with the residue scheme: the others (alpha
    == 0, k == 0, matrix-vector shapes, k < 32 where no modulus count reaches
    the FP64 bound) run FP64 kernels with different summation orders."""
    return p["alpha"] != 0.0 and p["k"] >= 32 and p["m"] > 1 and p["n"] > 1


def _assert_matches_per_call(probs, arena, want):
    """Bitwise per residue-scheme problem (the rest are held to the FP64 bound
    by check_batch)."""
    got, ref = arena.cpu().numpy(), want.cpu().numpy()
    exact = 0
    for p in probs:
        m, n = p["m"], p["n"]
        if m == 0 or n == 0 or not _on_residues(p):
            continue
        o = (p["c"] - arena.data_ptr()) // 8
        np.testing.assert_array_equal(got[o:o + m * n], ref[o:o + m * n], err_msg=f"{m}x{n}x{p['k']}")
        exact += 1
    assert exact > 0


def test_grouped_ozaki_matches_per_call_route(ctx, oracle):
    """Ozaki precision in a grouped launch: the residue scheme per problem,
    bitwise equal to calling the residue route problem by problem (same
    moduli, scales and exact reconstruction), and inside the FP64 bound."""
    from jlc_b200 import JLC_PREC_OZAKI_CRT
    rng = np.random.default_rng(21)
    shapes = mixed_shapes(rng, 160) + [(1, 1, 1), (1, 150, 70), (150, 1, 70), (33, 65, 129), (64, 64, 600),
                                       (0, 4, 4), (5, 6, 0)]
    alphas = [float(x) for x in rng.uniform(-2, 2, size=len(shapes))]
    betas = [float(x) for x in rng.uniform(-2, 2, size=len(shapes))]
    alphas[3], betas[4], alphas[5] = 1.0, 0.0, 0.0
    probs, host, arena = make_batch(oracle, shapes, 23, alphas=alphas, betas=betas)
    before = arena.clone()
    plan = ctx.grouped_plan(probs, precision=JLC_PREC_OZAKI_CRT, residue=True)
    info = plan.info()
    assert info["int8_problems"] == sum(1 for p in probs if p["m"] and p["n"] and _on_residues(p))
    plan.run()
    ctx.synchronize()
    plan.close()
    want = _per_problem_ozaki(ctx, probs, before, arena.data_ptr())
    _assert_matches_per_call(probs, arena, want)
    check_batch(oracle, probs, host, arena, "grouped ozaki")


def test_grouped_ozaki_long_k_and_graph_replay(ctx, oracle):
    """k beyond one INT32 run (the accumulators fold to residues every 16352
    k) and a captured plan replayed on new data."""
    import torch
    from jlc_b200 import JLC_PREC_OZAKI
    shapes = [(40, 36, 20000), (17, 70, 33000), (96, 96, 300), (3, 3, 3)]
    probs, host, arena = make_batch(oracle, shapes, 29, betas=[0.0, 0.5, -1.0, 0.0])
    before = arena.clone()
    plan = ctx.grouped_plan(probs, precision=JLC_PREC_OZAKI, graph=True, residue=True)
    assert plan.info()["tile_small"] == 32
    plan.run()
    ctx.synchronize()
    want = _per_problem_ozaki(ctx, probs, before, arena.data_ptr())
    _assert_matches_per_call(probs, arena, want)
    check_batch(oracle, probs, host, arena, "grouped ozaki long k")
    # new B data in place, C restored: the replay recomputes every exponent
    host2 = []
    for p, (m, n, k, la, lb, alpha, beta, A, B, C) in zip(probs, host):
        B2 = 0.001 * B
        b_store = B2 if lb == 0 else np.ascontiguousarray(B2.T)
        off = (p["b"] - arena.data_ptr()) // 8
        arena[off:off + k * n] = torch.from_numpy(b_store.ravel())
        offc = (p["c"] - arena.data_ptr()) // 8
        arena[offc:offc + m * n] = torch.from_numpy(C.ravel())
        host2.append((m, n, k, la, lb, alpha, beta, A, B2, C))
    torch.cuda.synchronize()
    before2 = arena.clone()
    plan.run()
    ctx.synchronize()
    want2 = _per_problem_ozaki(ctx, probs, before2, arena.data_ptr())
    _assert_matches_per_call(probs, arena, want2)
    check_batch(oracle, probs, host2, arena, "grouped ozaki replay")
    plan.close()


def test_grouped_ozaki_nonfinite_problem_takes_fp64(ctx, oracle):
    """A problem whose operands hold Inf/NaN runs the FP64 tile (IEEE
    propagation as on the native route); the others stay on the residues."""
    import torch
    from jlc_b200 import JLC_PREC_OZAKI_CRT
    shapes = [(20, 30, 40), (50, 20, 70), (8, 8, 48)]
    probs, host, arena = make_batch(oracle, shapes, 31, betas=[0.0, 0.0, 0.0])
    p1 = probs[1]
    A1 = host[1][7].copy()
    A1[3, 5] = np.nan
    A1[10, 0] = np.inf
    a_store = A1 if p1["layout_a"] == 0 else np.ascontiguousarray(A1.T)
    off = (p1["a"] - arena.data_ptr()) // 8
    arena[off:off + 50 * 70] = torch.from_numpy(a_store.ravel())
    torch.cuda.synchronize()
    before = arena.clone()
    plan = ctx.grouped_plan(probs, precision=JLC_PREC_OZAKI_CRT, residue=True)
    plan.run()
    ctx.synchronize()
    plan.close()
    got = arena.cpu().numpy()
    want = _per_problem_ozaki(ctx, probs, before, arena.data_ptr()).cpu().numpy()
    flat_host = [(p, h) for p, h in zip(probs, host)]
    for i, (p, h) in enumerate(flat_host):
        m, n = p["m"], p["n"]
        oc = (p["c"] - arena.data_ptr()) // 8
        g, w = got[oc:oc + m * n], want[oc:oc + m * n]
        if i == 1:
            np.testing.assert_array_equal(np.isnan(g), np.isnan(w))
            np.testing.assert_array_equal(np.isinf(g), np.isinf(w))
            fin = np.isfinite(w)
            np.testing.assert_allclose(g[fin], w[fin], rtol=0, atol=1e-12)
        else:
            np.testing.assert_array_equal(g, w)


def test_grouped_ozaki_default_runs_fp64_tiles(ctx, oracle):
    """Without the residue opt-in, Ozaki precision runs every problem on the
    FP64 tiles (no per-problem certificate exists in a grouped launch): the
    results are bitwise the native plan's and the routes say so."""
    from jlc_b200 import JLC_PREC_NATIVE, JLC_PREC_OZAKI_CRT
    rng = np.random.default_rng(41)
    shapes = mixed_shapes(rng, 120) + [(64, 64, 600), (40, 36, 2500)]
    probs, host, arena = make_batch(oracle, shapes, 43)
    before = arena.clone()
    plan = ctx.grouped_plan(probs, precision=JLC_PREC_OZAKI_CRT)
    info = plan.info()
    nonempty = sum(1 for p in probs if p["m"] and p["n"])
    assert info["int8_problems"] == 0 and info["fp64_problems"] == nonempty
    plan.run()
    ctx.synchronize()
    plan.close()
    got = arena.clone()
    arena.copy_(before)
    rep = ctx.dgemm_grouped_device(probs, precision=JLC_PREC_NATIVE)
    assert rep["precision"] == JLC_PREC_NATIVE
    np.testing.assert_array_equal(got.cpu().numpy(), arena.cpu().numpy())
    check_batch(oracle, probs, host, arena, "grouped ozaki default")
    arena.copy_(before)
    rep = ctx.dgemm_grouped_device(probs, precision=JLC_PREC_OZAKI_CRT)
    assert rep["precision"] == JLC_PREC_NATIVE  # the precision actually used
