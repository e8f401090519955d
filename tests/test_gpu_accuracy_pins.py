"""Pins of the accuracy evidence to the CPU double-double oracle.

  * jlc_check_fp64_bound_device, the device double-double check that the
    benchmark uses for its 8192^3 / 16384^3 accuracy figures, returns the
    oracle's max |err|/bound and max |err| on the same sampled entries, and
    counts entries pushed over the bound on the host.
  * The automatic slice / modulus count at the headline depth (k = 8192 and
    k = 16384) meets the FP64 bound against the oracle on every entry.
  * The real 20,000-problem batch generator (its first 2,000 problems, dims up
    to 512) meets the bound through the grouped launch, native and Ozaki.
"""
import os
import sys

import numpy as np
import pytest

from parity import assert_fp64_bound

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _device_check(ctx, la, lb, m, n, k, alpha, dA, lda, dB, ldb, beta, dCin, dCout, rows, cols):
    return ctx.check_fp64_bound_device(la, lb, m, n, k, alpha, dA.data_ptr(), lda, dB.data_ptr(), ldb, beta,
                                       dCin.data_ptr() if dCin is not None else None, n, dCout.data_ptr(), n,
                                       rows, cols)


@pytest.mark.parametrize("la,lb,precision", [(0, 0, 0), (1, 0, 0), (0, 1, 3), (1, 1, 1)])
def test_device_checker_matches_oracle(ctx, oracle, la, lb, precision):
    import torch
    m, n, k = 520, 384, 640
    alpha, beta = 1.5, 0.5
    A = oracle.uniform((m, k), 1201)
    B = oracle.uniform((k, n), 1202)
    C = oracle.uniform((m, n), 1203)
    a_store = A if la == 0 else np.ascontiguousarray(A.T)
    b_store = B if lb == 0 else np.ascontiguousarray(B.T)
    dA, dB, dCin = _dev(a_store), _dev(b_store), _dev(C)
    dC = dCin.clone()
    ctx.dgemm_device(la, lb, m, n, k, alpha, dA.data_ptr(), a_store.shape[1], dB.data_ptr(), b_store.shape[1],
                     beta, dC.data_ptr(), n, precision=precision)
    ctx.synchronize()
    out = dC.cpu().numpy()
    rows, cols = oracle.sample_entries(m, n, 2000, 1204)
    ref, bound = oracle.gemm_dd(A, B, C, alpha, beta, rows=rows, cols=cols)

    # the result as computed
    got = _device_check(ctx, la, lb, m, n, k, alpha, dA, a_store.shape[1], dB, b_store.shape[1], beta, dCin, dC,
                        rows, cols)
    err = np.abs(out[rows, cols] - ref)
    want_ratio, want_abs = float(np.max(err / bound)), float(np.max(err))
    assert got["over_bound"] == int(np.sum(err > bound)) == 0
    assert got["max_ratio"] == pytest.approx(want_ratio, rel=1e-6, abs=1e-12)
    assert got["max_abs_err"] == pytest.approx(want_abs, rel=1e-6, abs=1e-18)

    # the same result with entries pushed to 3x and 0.5x their bound on the host
    pert = out.copy()
    over_idx = np.arange(0, rows.size, 7)
    half_idx = np.setdiff1d(np.arange(3, rows.size, 11), over_idx)
    sign = np.where(np.arange(rows.size) % 2 == 0, 1.0, -1.0)
    pert[rows[half_idx], cols[half_idx]] = ref[half_idx] + 0.5 * sign[half_idx] * bound[half_idx]
    # written last: an entry sampled twice keeps its 3x value
    pert[rows[over_idx], cols[over_idx]] = ref[over_idx] + 3.0 * sign[over_idx] * bound[over_idx]
    dP = torch.from_numpy(pert).cuda()
    got = _device_check(ctx, la, lb, m, n, k, alpha, dA, a_store.shape[1], dB, b_store.shape[1], beta, dCin, dP,
                        rows, cols)
    err = np.abs(pert[rows, cols] - ref)
    assert got["over_bound"] == int(np.sum(err > bound)) > 0
    assert got["max_ratio"] == pytest.approx(float(np.max(err / bound)), rel=1e-6)
    # ref + 3 bound is itself rounded: 3 up to u |ref| / (3 bound) <= 1 / (12 k)
    assert got["max_ratio"] == pytest.approx(3.0, rel=1e-3)
    assert got["max_abs_err"] == pytest.approx(float(np.max(err)), rel=1e-6)


@pytest.mark.parametrize("mode", ["slices", "crt"])
@pytest.mark.parametrize("m,n,k", [(256, 256, 8192), (128, 128, 16384)])
def test_automatic_count_at_headline_depth(ctx, oracle, mode, m, n, k):
    A = oracle.uniform((m, k), 1301)
    B = oracle.uniform((k, n), 1302)
    dA, dB = _dev(A), _dev(B)
    dC = _dev(np.zeros((m, n)))
    entry = ctx.ozaki_device if mode == "slices" else ctx.ozaki_crt_device
    rep = entry(0, 0, m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), n, 0.0, dC.data_ptr(), n, 0)
    ctx.synchronize()
    want = oracle.auto_slices(k) if mode == "slices" else oracle.auto_moduli(k)
    assert rep["kernel"] == 3 and rep["slices"] == want, rep
    ratio = assert_fp64_bound(f"auto {mode} {m}x{n}x{k}", dC.cpu().numpy(), A, B, None, 1.0, 0.0)
    assert ratio <= rep["est_err_ratio"] <= 1.0


@pytest.mark.parametrize("precision,residue", [(0, False), (3, False), (3, True)])
def test_c4_generator_first_2000(ctx, oracle, precision, residue):
    """The benchmark's batch generator (30 % tiny M=N=K in {2,3,4}, the rest
    log-uniform on [8, 512], alpha and beta uniform on [-2, 2]): its first
    2,000 problems through one grouped launch, 24 sampled entries per problem
    (all entries of the tiny ones) against the oracle."""
    import torch
    import bench
    shapes, ab = bench.c4_shapes(count=2000)
    even = lambda x: (x + 1) // 2 * 2  # each matrix starts 16-byte aligned
    host, offs, total = [], [], 0
    for idx, ((m, n, k), (alpha, beta)) in enumerate(zip(shapes, ab)):
        A = oracle.uniform((m, k), 140000 + 3 * idx)
        B = oracle.uniform((k, n), 140000 + 3 * idx + 1)
        C = oracle.uniform((m, n), 140000 + 3 * idx + 2)
        host.append((m, n, k, alpha, beta, A, B, C))
        pa = total
        pb = pa + even(m * k)
        pc = pb + even(k * n)
        total = pc + even(m * n)
        offs.append((pa, pb, pc))
    flat = np.zeros(total)
    for (m, n, k, alpha, beta, A, B, C), (pa, pb, pc) in zip(host, offs):
        flat[pa:pa + m * k] = A.ravel()
        flat[pb:pb + k * n] = B.ravel()
        flat[pc:pc + m * n] = C.ravel()
    arena = torch.from_numpy(flat).cuda()
    base = arena.data_ptr()
    probs = [dict(m=m, n=n, k=k, layout_a=0, layout_b=0, lda=k, ldb=n, ldc=n, alpha=alpha, beta=beta,
                  a=base + 8 * pa, b=base + 8 * pb, c=base + 8 * pc)
             for (m, n, k, alpha, beta, A, B, C), (pa, pb, pc) in zip(host, offs)]
    plan = ctx.grouped_plan(probs, precision=precision, residue=residue)
    plan.run()
    ctx.synchronize()
    plan.close()
    res = arena.cpu().numpy()
    rng = np.random.default_rng(1401)
    for (m, n, k, alpha, beta, A, B, C), (pa, pb, pc) in zip(host, offs):
        got = res[pc:pc + m * n].reshape(m, n)
        if m * n <= 24:
            rows, cols = np.divmod(np.arange(m * n, dtype=np.int64), n)
        else:
            rows = rng.integers(0, m, 24, dtype=np.int64)
            cols = rng.integers(0, n, 24, dtype=np.int64)
        ref, bound = oracle.gemm_dd(A, B, C, alpha, beta, rows=rows, cols=cols)
        ratio, _ = oracle.max_err_ratio(got[rows, cols], ref, bound)
        assert ratio <= 1.0, f"C4 problem {m}x{n}x{k} precision {precision} residue {residue}: {ratio:.3g}"
