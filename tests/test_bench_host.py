"""CPU checks of bench.py's host-side pieces: the C4 problem generator, and the
port of the reference's parity-gated backend comparison (report columns,
percentile statistics, artifacts), run with the GPU routes replaced by numpy.
"""
import csv
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402

# header of GemmBackendComparison.writeCsv (GemmBackendComparison.java:510)
REFERENCE_CSV_HEADER = ("timestamp,size,m,k,n,backend,threads,valid,parity_status,oracle_type,reference_backend,"
                        "rel_residual,max_abs_err,warmups,iters,median_ms,mean_ms,stddev_ms,min_ms,p10_ms,p25_ms,"
                        "p75_ms,p90_ms,gflops_median,speedup_vs_baseline,baseline_label,checksum,notes")


def test_harness_columns_are_the_reference_columns():
    assert ",".join(bench.HARNESS_COLUMNS) == REFERENCE_CSV_HEADER


def _reference_percentile(sorted_v, q):
    # TimingStats.percentile (GemmBackendComparison.java:1031-1046), restated
    if len(sorted_v) == 0:
        return float("nan")
    if len(sorted_v) == 1:
        return sorted_v[0]
    position = q * (len(sorted_v) - 1)
    lower, upper = int(np.floor(position)), int(np.ceil(position))
    if lower == upper:
        return sorted_v[lower]
    w = position - lower
    return sorted_v[lower] * (1.0 - w) + sorted_v[upper] * w


@pytest.mark.parametrize("n", [1, 2, 5, 25])
def test_percentiles(n):
    v = sorted(np.random.default_rng(n).uniform(0, 10, n).tolist())
    for q in (0.1, 0.25, 0.5, 0.75, 0.9):
        assert bench._percentile(v, q) == _reference_percentile(v, q)


def test_c4_problem_mix():
    shapes, ab = bench.c4_shapes()
    assert len(shapes) == 20000 and len(ab) == 20000
    tiny = [s for s in shapes if s[0] == s[1] == s[2] and s[0] in (2, 3, 4)]
    assert 0.27 < len(tiny) / len(shapes) < 0.33
    rest = [s for s in shapes if s not in tiny]
    assert all(8 <= x <= 512 for s in rest for x in s)
    assert all(-2.0 <= a <= 2.0 and -2.0 <= b <= 2.0 for a, b in ab)


def test_harness_writes_reference_shaped_reports(tmp_path, monkeypatch):
    """The comparison run end to end with the GPU routes standing in as numpy
    products: parity gate, statistics, speed-up against opt-1t, CSV (stable
    and time-stamped) and JSON artifacts."""
    import torch
    import jlc_b200
    from jlc_b200 import compute

    def fake_gemm(a, b, c, alpha, beta, precision=0):
        c.getRawData()[:] = (alpha * (a.to_numpy() @ b.to_numpy())).ravel()
        return True

    monkeypatch.setattr(jlc_b200, "Context", lambda *a: None)
    monkeypatch.setattr(compute.CudaGemm, "gemm", staticmethod(fake_gemm))
    monkeypatch.setattr(torch.cuda, "set_device", lambda *a: None)
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a: "stand-in")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "harness", "--sizes", "32,48", "--iters", "3",
                                      "--warmups", "1", "--report-dir", str(tmp_path)])
    assert bench.main() == 0
    with open(tmp_path / "gemm-backend-comparison.csv") as f:
        rows = list(csv.reader(f))
    assert ",".join(rows[0]) == REFERENCE_CSV_HEADER
    body = [dict(zip(rows[0], r)) for r in rows[1:]]
    assert len(body) == 2 * len(bench.HARNESS_BACKENDS)
    for r in body:
        if r["backend"].startswith("blas3"):
            assert r["parity_status"] == "SKIPPED"
        else:
            assert r["parity_status"] == "PASS" and r["valid"] == "true"
            assert float(r["median_ms"]) > 0 and float(r["gflops_median"]) > 0
            assert r["baseline_label"] == "opt-1t"
    stamped = [p for p in os.listdir(tmp_path) if p.startswith("gemm-backend-comparison-") and p.endswith(".csv")]
    assert len(stamped) == 1
    with open(tmp_path / "gemm-backend-comparison.json") as f:
        doc = json.load(f)
    assert set(doc) == {"metadata", "artifacts", "rows"} and len(doc["rows"]) == len(body)
