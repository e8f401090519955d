"""Benchmark: 8192^3 DGEMM GFLOP/s at FP64 accuracy, Ozaki-INT8 vs native FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size 8192]

One step = one C = A*B (alpha=1, beta=0, M=N=K=size, FP64, uniform[-1,1)
synthetic inputs from a fixed seed) through libjlcgpu.  `value` is the
FP64-accurate rate of the Ozaki-INT8 route (FP64-equivalent 2*M*N*K/t); the
native FP64 DMMA route is measured in the same run and reported beside it.
Inputs are 3 x 512 MiB, larger than the 126 MB L2, so no flush is needed
between steps.  For N > 1 (torchrun) every rank computes its own row block of
an (N*size) x size product (weak scaling, no data-path collective); the time is
the max over ranks.

--impl reference times the reference's CPU algorithm (the oracle's restatement
of OptimizedBLAS3's PARALLEL_MICRO path, all host threads) on a bounded sample
of the same workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "8192^3 DGEMM GFLOP/s at FP64 accuracy: Ozaki-INT8 vs native FP64, % of peak"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--size", type=int, default=8192)
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of one CPU baseline sample")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", default="dgemm",
                   choices=["dgemm", "grouped", "configs", "harness", "qr", "shape", "hessenberg", "bidiag"],
                   help="dgemm: the 8192^3 headline; grouped: 20,000 uneven problems in one launch; "
                        "configs: one line per C1-C5 shape (rate and accuracy), one GPU")
    p.add_argument("--count", type=int, default=20000, help="grouped workload: number of problems")
    p.add_argument("--mnk", default="16384,1,16384", help="shape workload: m,n,k of one device product")
    p.add_argument("--precision", type=int, default=0, help="shape workload: JLC_PREC_* of the product")
    p.add_argument("--layouts", default="rr",
                   help="shape workload: storage of A and B, r (row-major) or c (column-major) each")
    p.add_argument("--sizes", default="128,256,512", help="harness workload: square sizes")
    p.add_argument("--iters", type=int, default=25, help="harness workload: timed iterations per backend")
    p.add_argument("--warmups", type=int, default=8, help="harness workload: warm-up iterations per backend")
    p.add_argument("--report-dir", default=os.path.join("build", "reports", "gemm"),
                   help="harness workload: where the CSV/JSON reports go")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock, power and clock-event reasons through NVML during the
    timed region (read-only queries)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle",
               0x2: "applications_clocks_setting", 0x10: "sync_boost"}

    def __init__(self, torch_device: int):
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = self._handle(torch_device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # NVML missing: report no clocks rather than guess
            self.nv = None
            self.error = str(e)

    def _handle(self, dev):
        import torch
        nv = self.nv
        props = torch.cuda.get_device_properties(dev)
        try:
            bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
            return nv.nvmlDeviceGetHandleByPciBusId_v2(bus)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[dev]) if vis else dev
            return nv.nvmlDeviceGetHandleByIndex(idx)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                try:
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except Exception:
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.samples.append((sm, pw, rs))
            except Exception:
                pass
            self._stop.wait(0.02)

    def __enter__(self):
        if self.nv is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join()

    def summary(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": []}
        reasons = set()
        for _, _, rs in self.samples:
            for bit, name in self.REASONS.items():
                if rs & bit and name != "gpu_idle":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(s[0] for s in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "power_w_max": max(s[1] for s in self.samples),
                "samples": len(self.samples)}


# ----------------------------------------------------------------------------- helpers
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


def profile_traffic(name):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>.txt,
    line 'dram_bytes_per_launch: <bytes>'), or None."""
    path = os.path.join(ROOT, "profiles", name + ".txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("dram_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1])
                except ValueError:
                    return None
    return None


def cpu_baseline(size, seconds, threads=None):
    """The oracle's restatement of OptimizedBLAS3 PARALLEL_MICRO (packed, tiled,
    threaded; bit-exact with the Java path) on a row sample of the size^3
    product, timed on this host's cores."""
    import numpy as np
    from oracle import oracle as O
    threads = threads or (os.cpu_count() or 1)
    rng = np.random.default_rng(20260604)
    B = rng.uniform(-1.0, 1.0, (size, size))
    probe_rows = 64
    A = rng.uniform(-1.0, 1.0, (probe_rows, size))
    C = np.zeros((probe_rows, size))
    t0 = time.perf_counter()
    O.gemm_packed_parallel(A, B, C, 1.0, 0.0, threads=threads)
    dt = time.perf_counter() - t0
    rate = 2.0 * probe_rows * size * size / max(dt, 1e-9)
    rows = int(max(64, min(size, seconds * rate / (2.0 * size * size))))
    rows = max(64, rows // 64 * 64)
    A = rng.uniform(-1.0, 1.0, (rows, size))
    C = np.zeros((rows, size))
    t0 = time.perf_counter()
    O.gemm_packed_parallel(A, B, C, 1.0, 0.0, threads=threads)
    dt = time.perf_counter() - t0
    gflops = 2.0 * rows * size * size / dt / 1e9
    return {"value": round(gflops, 2), "unit": "GFLOP/s", "cores": threads, "kind": "port",
            "sample": f"rows 0..{rows} of the {size}^3 product ({rows}x{size}x{size}, alpha=1, beta=0) through "
                      f"the C restatement of OptimizedBLAS3 PARALLEL_MICRO (MC/KC/NC=2048/128/128, 6x8 "
                      f"microkernel, bit-exact fma chain), {threads} threads, {dt:.1f} s"}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    size = args.size
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(size, args.cpu_seconds / 2 if i < args.warmup else args.cpu_seconds, threads)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median(x["value"] for x in vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic uniform[-1,1), seed 20260604",
        "config": {"workload": f"DGEMM M=N=K={size}, alpha=1, beta=0, row-major, FP64 (CPU sample)",
                   "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": threads, "kind": "port",
                         "sample": vals[-1]["sample"]},
        "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference path is Java (OptimizedBLAS3); no JDK exists in this image, so its algorithm "
                "is timed through the C restatement in oracle/ on all host threads",
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- our arm
def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import jlc_b200
    from jlc_b200 import JLC_PREC_AUTO, JLC_PREC_NATIVE, JLC_PREC_OZAKI

    world, rank, local = dist_env()
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    size = args.size
    # One product of world*size rows: rank r computes its row block of C from
    # the same rows of A and all of B (no collective on the data path)
    from jlc_b200 import shard
    global_m = world * size
    r0, r1 = shard.partition_rows(global_m, world)[rank]
    M, N, K = r1 - r0, size, size
    flops = 2.0 * M * N * K

    ctx = jlc_b200.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)

    peaks = ctx.measure_peaks()  # burst rates, short probes on a cool GPU
    g = torch.Generator(device="cuda")
    with torch.cuda.stream(stream):
        # rows [r0, r1) of the one global A (seeded by the block's first row)
        # and the same B on every rank
        g.manual_seed(shard.block_seed(20260604, r0))
        A = torch.rand((M, K), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        g.manual_seed(20260605)
        B = torch.rand((K, N), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        Cn = torch.zeros((M, N), dtype=torch.float64, device="cuda")
        Cs = torch.zeros((M, N), dtype=torch.float64, device="cuda")
        Co = torch.zeros((M, N), dtype=torch.float64, device="cuda")
    stream.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    def step(prec, C, report=False):
        return ctx.dgemm_device(0, 0, M, N, K, 1.0, A.data_ptr(), K, B.data_ptr(), N, 0.0, C.data_ptr(), N,
                                precision=prec, report=report)

    def timed(prec, C, clocks=None):
        # the first warm-up call reports (route, count, certified error ratio);
        # the timed calls stay asynchronous
        rep = step(prec, C, report=True)
        for _ in range(args.warmup - 1):
            step(prec, C)
        ctx.synchronize()
        ctx.profile_collect()
        ctx.set_profiling(True)
        launches0 = ctx.launch_count()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step(prec, C)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        launches = ctx.launch_count() - launches0
        recs = ctx.profile_collect()
        ctx.set_profiling(False)
        if world > 1:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        phases = {}
        for name, pms in recs:
            phases.setdefault(name, []).append(pms)
        return ms / args.steps, rep, launches, phases

    # the headline first -- the default policy (JLC_PREC_AUTO), which takes the
    # Ozaki residue scheme at this size, with clocks sampled over its timed
    # region -- then the Ozaki slice scheme and native FP64 beside it (each
    # with its own warm-up), so the headline does not inherit their heat
    with ClockSampler(local) as clk:
        oz_ms, oz_rep, oz_launches, oz_phases = timed(JLC_PREC_AUTO, Co)
    clocks = clk.summary()
    sl_ms, sl_rep, sl_launches, sl_phases = timed(JLC_PREC_OZAKI, Cs)
    nat_ms, nat_rep, nat_launches, nat_phases = timed(JLC_PREC_NATIVE, Cn)
    # the residue GEMM's roofline denominator, probed after the timed regions:
    # the INT8 rate over the second half of a 3 s loop at the power limit
    int8_sustained = ctx.measure_int8_sustained(3.0)

    # accuracy of both results on sampled entries against the device double-double check
    rng = np.random.default_rng(17 + rank)
    rows = np.concatenate([rng.integers(0, M, 4096), [0, M - 1, 127, 128, M - 1]])
    cols = np.concatenate([rng.integers(0, N, 4096), [0, N - 1, 255, 256, 0]])
    acc_oz = ctx.check_fp64_bound_device(0, 0, M, N, K, 1.0, A.data_ptr(), K, B.data_ptr(), N, 0.0, None, N,
                                         Co.data_ptr(), N, rows, cols)
    acc_nat = ctx.check_fp64_bound_device(0, 0, M, N, K, 1.0, A.data_ptr(), K, B.data_ptr(), N, 0.0, None, N,
                                          Cn.data_ptr(), N, rows, cols)
    acc_sl = ctx.check_fp64_bound_device(0, 0, M, N, K, 1.0, A.data_ptr(), K, B.data_ptr(), N, 0.0, None, N,
                                         Cs.data_ptr(), N, rows, cols)

    # end to end through the public host entry (pinned host buffers, copies timed on the device)
    e2e = None
    if not args.no_e2e:
        Ah = A.cpu().pin_memory()
        Bh = B.cpu().pin_memory()
        Ch = torch.zeros((M, N), dtype=torch.float64).pin_memory()
        a_np, b_np, c_np = Ah.numpy(), Bh.numpy(), Ch.numpy()
        for _ in range(max(1, min(args.warmup, 2))):
            ctx.gemm(a_np, b_np, c_np, 1.0, 0.0, precision=JLC_PREC_AUTO)
        dev_ms, wall = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            rep = ctx.gemm(a_np, b_np, c_np, 1.0, 0.0, precision=JLC_PREC_AUTO)
            wall.append((time.perf_counter() - t0) * 1e3)
            dev_ms.append(rep["device_ms"])
        e2e_ms = statistics.mean(dev_ms)
        if world > 1:
            t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": round(world * flops / (e2e_ms * 1e-3) / 1e9, 1), "unit": "GFLOP/s",
               "h2d_bytes_per_step": int(rep["h2d_bytes"]), "d2h_bytes_per_step": int(rep["d2h_bytes"]),
               "ms_per_step": round(e2e_ms, 3), "wall_ms_per_step": round(statistics.mean(wall), 3),
               "path": "jlc_gemm (host pointers, pinned), default policy (Ozaki residue scheme), "
                       "H2D+D2H inside the timed region"}
        # the same calls on pageable buffers (what a caller that copies heap
        # arrays into fresh native memory per call gets)
        import numpy as np
        a_pg, b_pg, c_pg = np.array(a_np), np.array(b_np), np.zeros_like(c_np)
        ctx.gemm(a_pg, b_pg, c_pg, 1.0, 0.0, precision=JLC_PREC_AUTO)
        pg_ms = []
        for _ in range(max(2, min(args.steps, 5))):
            t0 = time.perf_counter()
            ctx.gemm(a_pg, b_pg, c_pg, 1.0, 0.0, precision=JLC_PREC_AUTO)
            pg_ms.append((time.perf_counter() - t0) * 1e3)
        pg = statistics.mean(pg_ms)
        if world > 1:
            t = torch.tensor([pg], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pg = float(t.item())
        e2e["pageable"] = {"value": round(world * flops / (pg * 1e-3) / 1e9, 1), "unit": "GFLOP/s",
                           "ms_per_step": round(pg, 3), "steps": len(pg_ms), "clock": "host wall clock per call",
                           "path": "jlc_gemm on pageable numpy buffers (the library stages the copies through "
                                   "its ring of pinned chunks, filled and drained by host threads), same copies "
                                   "inside the timed region"}
        del a_pg, b_pg, c_pg

    if rank != 0:
        return 0

    nat_gflops = flops / (nat_ms * 1e-3) / 1e9
    oz_gflops = flops / (oz_ms * 1e-3) / 1e9
    sl_gflops = flops / (sl_ms * 1e-3) / 1e9
    P = oz_rep["products"]
    gemm_ms = statistics.mean(oz_phases.get("ozaki_gemm", [float("nan")]))
    split_ms = statistics.mean(oz_phases.get("ozaki_split", [float("nan")]))
    cert_ms = statistics.mean(oz_phases.get("ozaki_cert", [float("nan")]))
    dmma_ms = statistics.mean(nat_phases.get("dmma", [float("nan")]))
    int8_ops_per_launch = 2.0 * M * N * K * P
    achieved_tops = int8_ops_per_launch / (gemm_ms * 1e-3) / 1e12
    mp = measured_peaks()
    traffic = profile_traffic(f"ozaki_crt_gemm_{size}")
    line = {
        "metric": METRIC,
        "value": round(world * oz_gflops, 1),
        "unit": "GFLOP/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(oz_ms, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (INT8 residue products, INT32 accumulation, exact integer CRT reconstruction)",
        "data": "synthetic uniform[-1,1) (torch Philox; one global A seeded per row block, one B), device resident",
        "config": {"workload": f"DGEMM M=N=K={size}, alpha=1, beta=0, row-major A/B/C, FP64-accurate "
                               f"(default policy: Ozaki-INT8 residue scheme, {oz_rep['slices']} moduli)",
                   "global_M": global_m, "N": N, "K": K,
                   "parallelism": f"dp{world} (row blocks of one product, shard.partition_rows; no collective)",
                   "l2": "inputs 1.5 GiB > 126 MB L2, no flush"},
        "gpu_launches": int(oz_launches),
        "clocks": clocks,
        "accuracy": {"ozaki": acc_oz, "ozaki_slices": acc_sl, "native": acc_nat,
                     "check": "device double-double on 4101 sampled entries, bound 2ku|A||B|"},
        "native_fp64": {"value": round(world * nat_gflops, 1), "unit": "GFLOP/s", "ms_per_step": round(nat_ms, 3),
                        "kernel_ms": round(dmma_ms, 3),
                        "frac_of_dmma_peak": round(flops / (dmma_ms * 1e-3) / 1e12 / peaks["fp64_dmma_tflops"], 4),
                        "gpu_launches": int(nat_launches)},
        "ozaki": {"scheme": "residues (CRT)", "moduli": oz_rep["slices"], "products": P,
                  "certified_err_ratio": oz_rep["est_err_ratio"],
                  "split_ms": round(split_ms, 3), "cert_ms": round(cert_ms, 3), "gemm_ms": round(gemm_ms, 3),
                  "speedup_vs_native": round(oz_gflops / nat_gflops, 3)},
        "ozaki_slices": {"value": round(world * sl_gflops, 1), "unit": "GFLOP/s", "ms_per_step": round(sl_ms, 3),
                         "slices": sl_rep["slices"], "products": sl_rep["products"],
                         "split_ms": round(statistics.mean(sl_phases.get("ozaki_split", [float("nan")])), 3),
                         "gemm_ms": round(statistics.mean(sl_phases.get("ozaki_gemm", [float("nan")])), 3),
                         "gpu_launches": int(sl_launches)},
        "peaks_probed": {k: round(v, 2) for k, v in peaks.items()},
        "roofline": {"bound": "tensor", "kernel": "ozaki_gemm_kernel<CRT=true> (tcgen05 kind::i8)",
                     "achieved": round(achieved_tops, 1), "peak": round(int8_sustained, 1),
                     "unit": "TFLOP/s", "frac": round(achieved_tops / int8_sustained, 4),
                     "traffic": traffic,
                     "traffic_source": (f"dram__bytes_read.sum + dram__bytes_write.sum per launch from the committed "
                                        f"ncu capture profiles/ozaki_crt_gemm_{size}.txt, not measured in this run"
                                        if traffic is not None else None),
                     "peak_source": "INT8 dense tcgen05 rate sustained over 3 s of back-to-back probe launches "
                                    "(second half, at the power limit) in this run: the kernel is timed inside "
                                    "a long step under sw_power_cap (MEASURED_PEAKS.json has no INT8 figure)",
                     "peak_burst": round(peaks["int8_tops"], 1),
                     "frac_of_burst": round(achieved_tops / peaks["int8_tops"], 4),
                     "bf16_probe_vs_measured_peaks": (round(peaks["bf16_tflops"] / mp["bf16_tflops"], 3)
                                                      if mp and mp.get("bf16_tflops") else None),
                     "ops_per_launch": int8_ops_per_launch},
        "e2e": e2e,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(size, args.cpu_seconds)
    print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def c4_shapes(count=20000, seed=20260604):
    """20,000 problems: 30 % tiny (M=N=K in {2,3,4}), 70 % with M, N, K
    independently log-uniform on [8, 512]; alpha, beta uniform on [-2, 2]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    shapes, ab = [], []
    for _ in range(count):
        if rng.random() < 0.3:
            s = int(rng.integers(2, 5))
            shapes.append((s, s, s))
        else:
            shapes.append(tuple(int(x) for x in np.exp(rng.uniform(np.log(8), np.log(512), size=3)).round()))
        ab.append((float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2))))
    return shapes, ab


def run_grouped(args):
    """Config: 20,000 uneven FP64 GEMMs in one persistent launch (CUDA graph replay)."""
    import torch
    import jlc_b200
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    ctx = jlc_b200.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    shapes, ab = c4_shapes(count=args.count, seed=20260604 + rank)
    al = lambda x: (x + 1) // 2 * 2  # each matrix starts 16-byte aligned, as separate allocations would
    total = sum(al(m * k) + al(k * n) + al(m * n) for (m, n, k) in shapes)
    g = torch.Generator(device="cuda")
    g.manual_seed(20260604 + rank)
    with torch.cuda.stream(stream):
        arena = torch.rand(total, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    stream.synchronize()
    base, off, probs, bytes_alg = arena.data_ptr(), 0, [], 0
    for (m, n, k), (alpha, beta) in zip(shapes, ab):
        pa = off
        pb = pa + al(m * k)
        pc = pb + al(k * n)
        off = pc + al(m * n)
        probs.append(dict(m=m, n=n, k=k, layout_a=0, layout_b=0, lda=k, ldb=n, ldc=n, alpha=alpha, beta=beta,
                          a=base + 8 * pa, b=base + 8 * pb, c=base + 8 * pc))
        bytes_alg += 8 * (m * k + k * n + 2 * m * n)
    plan = ctx.grouped_plan(probs, graph=True, autotune=True)
    info = plan.info()
    for _ in range(args.warmup):
        plan.run()
    ctx.synchronize()
    launches0 = ctx.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            plan.run()
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    flops = info["flops"]
    plan.close()
    # the same batch at Ozaki precision: by default FP64 tiles (no per-problem
    # certificate in a grouped launch), and the opt-in residue tiles beside it
    from jlc_b200 import JLC_PREC_OZAKI_CRT

    def time_plan(residue):
        pl = ctx.grouped_plan(probs, precision=JLC_PREC_OZAKI_CRT, graph=True, residue=residue)
        inf = pl.info()
        for _ in range(args.warmup):
            pl.run()
        ctx.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            pl.run()
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / args.steps
        pl.close()
        return t, inf

    oz_ms, oz_info = time_plan(False)
    res_ms, res_info = time_plan(True)
    line = {"metric": f"grouped FP64 GEMM GFLOP/s ({args.count:,} uneven problems, one persistent launch)",
            "value": round(flops / (ms * 1e-3) / 1e9, 1), "unit": "GFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "dtype": "f64", "data": "synthetic uniform[-1,1), 30% M=N=K in {2,3,4}, 70% M,N,K log-uniform [8,512]",
            "config": {"workload": f"{args.count} uneven DGEMMs, alpha/beta uniform[-2,2], row-major, 16-byte aligned "
                                   "matrices in one arena, CUDA-graph replay",
                       "work_items": info["work_items"], "tile_small": info["tile_small"],
                       "tile_large": info["tile_large"], "ring_slots_per_warp": info["stages"],
                       "flops_per_step": flops,
                       "algorithmic_bytes_per_step": bytes_alg},
            "achieved_gbs": round(bytes_alg / (ms * 1e-3) / 1e9, 1),
            "gpu_launches": ctx.launch_count() - launches0, "clocks": clk.summary(),
            "ozaki": {"value": round(flops / (oz_ms * 1e-3) / 1e9, 1), "unit": "GFLOP/s",
                      "ms_per_step": round(oz_ms, 4), "int8_problems": oz_info["int8_problems"],
                      "fp64_problems": oz_info["fp64_problems"],
                      "route": "Ozaki precision default: FP64 tiles for every problem (certified by construction)"},
            "ozaki_residue_opt_in": {"value": round(res_info["flops"] / (res_ms * 1e-3) / 1e9, 1),
                                     "unit": "GFLOP/s", "ms_per_step": round(res_ms, 4),
                                     "int8_problems": res_info["int8_problems"],
                                     "fp64_problems": res_info["fp64_problems"],
                                     "scheme": "JLC_GROUPED_RESIDUE: residues (CRT) per problem, 32x32 tiles, "
                                               "INT8 mma.sync; FP64-equivalent rate; not certified per problem"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_configs(args):
    """One JSON line per configuration of the five workload families: C1
    (1024^3, alpha 1.5, beta 0.5), C2 (DMMA square sweep, beta 0 and 1,
    rectangular shapes, matrix-vector, transposed / column-major operand
    layouts), C3 (Ozaki at 4096/8192/16384 on uniform and ill-scaled inputs),
    C5 (adjoint, native and Ozaki).  Each line: device time per call (CUDA
    events, warm), FP64-equivalent GFLOP/s, algorithmic GB/s, and the max
    |err|/bound over sampled entries from the device double-double check."""
    import numpy as np
    import torch
    import jlc_b200
    from jlc_b200 import JLC_COL_MAJOR, JLC_PREC_AUTO, JLC_PREC_NATIVE, JLC_PREC_OZAKI_CRT, JLC_ROW_MAJOR
    torch.cuda.set_device(0)
    ctx = jlc_b200.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    g = torch.Generator(device="cuda")
    g.manual_seed(20260604)
    reps = max(3, min(args.steps, 10))

    def uniform(shape):
        with torch.cuda.stream(stream):
            t = torch.rand(shape, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        return t

    def timed(fn):
        for _ in range(2):
            fn()
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            rep = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps, rep

    def accuracy(la, lb, m, n, k, alpha, A, lda, B, ldb, beta, Cin, C):
        rng = np.random.default_rng(5)
        rows = np.concatenate([rng.integers(0, m, 1024), [0, m - 1]])
        cols = np.concatenate([rng.integers(0, n, 1024), [0, n - 1]])
        if n == 1:
            cols[:] = 0
        return ctx.check_fp64_bound_device(la, lb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta,
                                           Cin.data_ptr() if Cin is not None else None, C.shape[1] if C.dim() > 1
                                           else 1, C.data_ptr(), C.shape[1] if C.dim() > 1 else 1, rows,
                                           cols)["max_ratio"]

    def gemm_case(name, m, n, k, alpha=1.0, beta=0.0, la=JLC_ROW_MAJOR, lb=JLC_ROW_MAJOR, precision=JLC_PREC_NATIVE,
                  scaled=False):
        A = uniform((m, k) if la == JLC_ROW_MAJOR else (k, m))
        B = uniform((k, n) if lb == JLC_ROW_MAJOR else (n, k))
        if scaled:  # 2^e, e uniform in [-20, 20], per row of A and per column of B
            ea = torch.randint(-20, 21, (m,), device="cuda", generator=g).double()
            eb = torch.randint(-20, 21, (n,), device="cuda", generator=g).double()
            A *= torch.pow(2.0, ea)[:, None] if la == JLC_ROW_MAJOR else torch.pow(2.0, ea)[None, :]
            B *= torch.pow(2.0, eb)[None, :] if lb == JLC_ROW_MAJOR else torch.pow(2.0, eb)[:, None]
        C0 = uniform((m, n))
        C = C0.clone()
        lda = A.shape[1]
        ldb = B.shape[1]
        ms, _ = timed(lambda: ctx.dgemm_device(la, lb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb,
                                               beta, C.data_ptr(), n, precision=precision, report=False))
        # accuracy of one fresh call on the original C (its report carries the
        # route and, for the INT8 routes, the certified error ratio)
        C.copy_(C0)
        rep = ctx.dgemm_device(la, lb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta, C.data_ptr(), n,
                               precision=precision)
        ctx.synchronize()
        ratio = accuracy(la, lb, m, n, k, alpha, A, lda, B, ldb, beta, C0 if beta != 0.0 else None, C)
        flops = 2.0 * m * n * k
        nbytes = 8.0 * (m * k + k * n + m * n * (2 if beta != 0.0 else 1))
        line = {"config": name, "m": m, "n": n, "k": k, "alpha": alpha, "beta": beta,
                "layout_a": "col" if la == JLC_COL_MAJOR else "row", "layout_b": "col" if lb == JLC_COL_MAJOR
                else "row", "route": {0: "native", 1: "ozaki-slices", 3: "ozaki-crt"}.get(rep["precision"]),
                "kernel": rep["kernel"], "ms": round(ms, 4), "gflops": round(flops / (ms * 1e-3) / 1e9, 1),
                "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1), "max_err_ratio": ratio}
        if rep["kernel"] == 3:
            line["certified_err_ratio"] = rep["est_err_ratio"]
        if scaled:
            line["inputs"] = "ill-scaled 2^e, e in [-20,20] per row of A / column of B"
        print(json.dumps(line), flush=True)
        del A, B, C, C0
        torch.cuda.empty_cache()

    gemm_case("C1", 1024, 1024, 1024, alpha=1.5, beta=0.5)
    for sz in (2048, 4096, 8192):
        for beta in (0.0, 1.0):
            gemm_case("C2 square", sz, sz, sz, beta=beta)
    gemm_case("C2 rectangular", 8192, 256, 8192)
    gemm_case("C2 rectangular", 8192, 8192, 256)
    gemm_case("C2 matvec", 16384, 1, 16384)
    gemm_case("C2 TransA (A^T B, A stored k x m)", 4096, 4096, 4096, la=JLC_COL_MAJOR)
    gemm_case("C2 ColMajorB", 4096, 4096, 4096, lb=JLC_COL_MAJOR)
    for sz in (4096, 8192, 16384):
        gemm_case("C3 Ozaki uniform", sz, sz, sz, precision=JLC_PREC_AUTO)
        gemm_case("C3 Ozaki ill-scaled", sz, sz, sz, precision=JLC_PREC_OZAKI_CRT, scaled=True)

    # C5: adjoint of C_out = A B + C_in, A 4096x2048, B 2048x4096, N(0,1)
    m, k, n = 4096, 2048, 4096
    for prec, pname in ((JLC_PREC_NATIVE, "native"), (JLC_PREC_OZAKI_CRT, "ozaki-crt")):
        with torch.cuda.stream(stream):
            A = torch.randn((m, k), dtype=torch.float64, device="cuda", generator=g)
            B = torch.randn((k, n), dtype=torch.float64, device="cuda", generator=g)
            Cin = torch.randn((m, n), dtype=torch.float64, device="cuda", generator=g)
            dC = torch.randn((m, n), dtype=torch.float64, device="cuda", generator=g)
            dA = torch.empty((m, k), dtype=torch.float64, device="cuda")
            dB = torch.empty((k, n), dtype=torch.float64, device="cuda")
            sc = torch.zeros(2, dtype=torch.float64, device="cuda")
        ms, _ = timed(lambda: ctx.adjoint_device(m, n, k, 1.0, 1.0, A.data_ptr(), k, B.data_ptr(), n,
                                                 Cin.data_ptr(), n, dC.data_ptr(), n, dA.data_ptr(), k,
                                                 dB.data_ptr(), n, sc.data_ptr(), sc.data_ptr() + 8,
                                                 precision=prec))
        flops = 2.0 * (2.0 * m * n * k) + 2.0 * m * n
        print(json.dumps({"config": "C5 adjoint", "m": m, "n": n, "k": k, "route": pname, "ms": round(ms, 4),
                          "gflops": round(flops / (ms * 1e-3) / 1e9, 1),
                          "outputs": "dA, dB, dalpha, dbeta"}), flush=True)
        del A, B, Cin, dC, dA, dB
        torch.cuda.empty_cache()
    ctx.close()
    return 0


# ----------------------------------------------------------------------------- blocked QR (next row)
def qr_cpu_baseline(n):
    """The oracle's C restatement of HouseholderQR.factorizeBlocked (scalar
    panels of 64 columns, the compact-WY update of each 128-column trailing
    block through the packed PARALLEL_MICRO kernel, the blocks spread over all
    host cores) on an n x n uniform[-1,1) matrix, timed on this host."""
    import numpy as np
    from oracle import oracle as O
    a = np.random.default_rng(20260604).uniform(-1.0, 1.0, (n, n))
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    O.householder_qr_blocked_c(a, cores)
    dt = time.perf_counter() - t0
    return {"value": round((2.0 * n ** 3 - 2.0 * n ** 3 / 3.0) / dt / 1e9, 2), "unit": "GFLOP/s", "cores": cores,
            "kind": "port",
            "sample": f"one {n}x{n} factorisation through the C restatement of factorizeBlocked (scalar panels, "
                      f"packed trailing GEMMs over {cores} threads), {dt:.1f} s"}


def run_qr(args):
    """Device-resident blocked Householder QR of a size x size uniform[-1,1)
    matrix (the reference's HouseholderQR.factorizeBlocked, panels of 64):
    device time of jlc_qr_factor_device per factorisation (the matrix is
    restored, untimed, before each), FLOPs 2mn^2 - 2n^3/3, and the share of the
    time in the panel kernels and the device time of every phase (phase
    records: qr_panel, qr_vt, and dmma for the Gram and trailing-update GEMMs)."""
    import statistics
    import torch
    import jlc_b200
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    ctx = jlc_b200.Context(local)
    n = args.size
    g = torch.Generator(device="cuda")
    g.manual_seed(20260604)
    a0 = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a = torch.empty_like(a0)
    tau = torch.empty(n, dtype=torch.float64, device="cuda")
    flops = 2.0 * n * n * n - 2.0 * n ** 3 / 3.0
    times, panel, phases = [], [], []
    for it in range(args.warmup + args.steps):
        a.copy_(a0)
        torch.cuda.synchronize()
        ctx.set_profiling(it >= args.warmup)
        rep = ctx.qr_factor_device(n, n, a.data_ptr(), n, tau.data_ptr())
        if it >= args.warmup:
            recs = ctx.profile_collect()
            times.append(rep["device_ms"])
            panel.append(sum(ms for name, ms in recs if name == "qr_panel"))
            per = {}
            for name, t in recs:
                per[name] = per.get(name, 0.0) + t
            phases.append(per)
    ctx.set_profiling(False)
    ms = statistics.median(times)
    peaks = ctx.measure_peaks()  # after the timed factorisations
    tflops = flops / (ms * 1e-3) / 1e12
    cpu = None if args.no_cpu_baseline else qr_cpu_baseline(min(n, 2048))
    line = {"metric": f"blocked Householder QR GFLOP/s ({n}x{n}, FP64, device-resident)",
            "value": round(flops / (ms * 1e-3) / 1e9, 1), "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "f64",
            "data": "synthetic uniform[-1,1) (torch Philox, seed 20260604), device resident",
            "config": {"workload": f"QR {n}x{n}, panels of 64, compact-WY trailing update on the DMMA route"},
            "panel_ms": round(statistics.median(panel), 3),
            "panel_share": round(statistics.median(panel) / ms, 3),
            "phase_ms": {name: round(statistics.median(p.get(name, 0.0) for p in phases), 3)
                         for name in sorted({n for p in phases for n in p})},
            "roofline": {"bound": "tensor", "kernel": "whole factorisation (panel kernels + FP64 DMMA GEMMs)",
                         "achieved": round(tflops, 3), "peak": round(peaks["fp64_dmma_tflops"], 2),
                         "unit": "TFLOP/s", "frac": round(tflops / peaks["fp64_dmma_tflops"], 4), "traffic": None,
                         "peak_source": "FP64 DMMA probe (jlc_measure_peaks) in this run; MEASURED_PEAKS.json has "
                                        "no FP64 figure",
                         "note": "the panel kernels, the largest share, are latency-bound (one barrier per "
                                 "column), not tensor-bound"},
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def hess_cpu_baseline(n):
    """The oracle's C restatement of BlockedHessenbergQR.decompose (the
    reference's scalar factorPanelUnblocked on a full working copy per panel
    of 32, the six block-update GEMMs per panel through the packed
    PARALLEL_MICRO kernel over all host cores) on an n x n uniform[-1,1)
    matrix, H and Q formed."""
    import numpy as np
    from oracle import oracle as O
    a = np.random.default_rng(20260604).uniform(-1.0, 1.0, (n, n))
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    O.blocked_hessenberg_c(a, cores)
    dt = time.perf_counter() - t0
    return {"value": round(14.0 / 3.0 * n ** 3 / dt / 1e9, 2), "unit": "GFLOP/s", "cores": cores, "kind": "port",
            "sample": f"one {n}x{n} reduction (H and Q) through the C restatement of BlockedHessenbergQR.decompose "
                      f"(scalar panels, packed block-update GEMMs over {cores} threads), {dt:.1f} s"}


def run_hessenberg(args):
    """Device-resident blocked Hessenberg reduction of a size x size
    uniform[-1,1) matrix with Q formed (BlockedHessenbergQR.decompose): device
    time per reduction (the matrix restored, untimed, before each), FLOPs
    10n^3/3 for H and 4n^3/3 for Q, and the device time of every phase."""
    import statistics
    import torch
    import jlc_b200
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    ctx = jlc_b200.Context(local)
    n = args.size
    g = torch.Generator(device="cuda")
    g.manual_seed(20260604)
    a0 = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a = torch.empty_like(a0)
    q = torch.empty_like(a0)
    flops = 14.0 / 3.0 * n ** 3
    times, phases = [], []
    for it in range(args.warmup + args.steps):
        a.copy_(a0)
        torch.cuda.synchronize()
        ctx.set_profiling(it >= args.warmup)
        rep = ctx.hessenberg_device(n, a.data_ptr(), n, q.data_ptr(), n)
        if it >= args.warmup:
            recs = ctx.profile_collect()
            times.append(rep["device_ms"])
            per = {}
            for name, t in recs:
                per[name] = per.get(name, 0.0) + t
            phases.append(per)
    ctx.set_profiling(False)
    ms = statistics.median(times)
    cpu = None if args.no_cpu_baseline else hess_cpu_baseline(min(n, 1024))
    line = {"metric": f"blocked Hessenberg reduction GFLOP/s ({n}x{n}, FP64, H and Q, device-resident)",
            "value": round(flops / (ms * 1e-3) / 1e9, 1), "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "f64",
            "data": "synthetic uniform[-1,1) (torch Philox, seed 20260604), device resident",
            "config": {"workload": f"Hessenberg {n}x{n} with Q, panels of 32, one GEMV per reflector, block "
                                   "updates on the DMMA route"},
            "phase_ms": {name: round(statistics.median(p.get(name, 0.0) for p in phases), 3)
                         for name in sorted({nm for p in phases for nm in p})},
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def bidiag_cpu_baseline(n):
    """The oracle's restatement of Bidiagonalization.decompose (one column and
    one row reflector per step applied to the whole trailing matrix and to U
    and V, numpy rank-1 updates on the host) on an n x n uniform[-1,1) matrix."""
    import numpy as np
    from oracle import oracle as O
    a = np.random.default_rng(20260604).uniform(-1.0, 1.0, (n, n))
    t0 = time.perf_counter()
    O.bidiagonalize(a)
    dt = time.perf_counter() - t0
    return {"value": round(16.0 / 3.0 * n ** 3 / dt / 1e9, 2), "unit": "GFLOP/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": f"one {n}x{n} reduction (B, U and V) through the numpy restatement of "
                      f"Bidiagonalization.decompose (rank-1 updates per reflector), {dt:.1f} s"}


def run_bidiag(args):
    """Device Golub-Kahan bidiagonalisation of a size x size uniform[-1,1)
    matrix with U and V formed (Bidiagonalization.decompose): device time per
    reduction (the matrix restored, untimed, before each), FLOPs 8n^3/3 for B
    and 4n^3/3 each for U and V, and the device time of the reflector launch."""
    import statistics
    import torch
    import jlc_b200
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    ctx = jlc_b200.Context(local)
    n = args.size
    g = torch.Generator(device="cuda")
    g.manual_seed(20260604)
    a0 = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a = torch.empty_like(a0)
    u = torch.empty_like(a0)
    v = torch.empty_like(a0)
    d = torch.empty(n, dtype=torch.float64, device="cuda")
    e = torch.empty(max(n - 1, 1), dtype=torch.float64, device="cuda")
    flops = 16.0 / 3.0 * n ** 3
    times, phases = [], []
    for it in range(args.warmup + args.steps):
        a.copy_(a0)
        torch.cuda.synchronize()
        ctx.set_profiling(it >= args.warmup)
        rep = ctx.bidiag_device(n, n, a.data_ptr(), n, d.data_ptr(), e.data_ptr(), u.data_ptr(), n, v.data_ptr(), n)
        if it >= args.warmup:
            recs = ctx.profile_collect()
            times.append(rep["device_ms"])
            per = {}
            for name, t in recs:
                per[name] = per.get(name, 0.0) + t
            phases.append(per)
    ctx.set_profiling(False)
    ms = statistics.median(times)
    cpu = None if args.no_cpu_baseline else bidiag_cpu_baseline(min(n, 512))
    line = {"metric": f"Golub-Kahan bidiagonalisation GFLOP/s ({n}x{n}, FP64, B, U and V, device-resident)",
            "value": round(flops / (ms * 1e-3) / 1e9, 1), "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "f64",
            "data": "synthetic uniform[-1,1) (torch Philox, seed 20260604), device resident",
            "config": {"workload": f"bidiagonalisation {n}x{n} with U and V: one cooperative launch for the "
                                   "reflectors, U and V by blocked WY on the DMMA route"},
            "phase_ms": {name: round(statistics.median(p.get(name, 0.0) for p in phases), 3)
                         for name in sorted({nm for p in phases for nm in p})},
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


# ----------------------------------------------------------------------------- harness (report port)
HARNESS_BACKENDS = ["blas3-naive", "blas3-simd-1t", "blas3-parallel", "opt-1t", "opt-parallel", "cuda",
                    "cuda-ozaki"]
HARNESS_COLUMNS = ["timestamp", "size", "m", "k", "n", "backend", "threads", "valid", "parity_status", "oracle_type",
                   "reference_backend", "rel_residual", "max_abs_err", "warmups", "iters", "median_ms", "mean_ms",
                   "stddev_ms", "min_ms", "p10_ms", "p25_ms", "p75_ms", "p90_ms", "gflops_median",
                   "speedup_vs_baseline", "baseline_label", "checksum", "notes"]


def _percentile(sorted_v, q):
    """Linear interpolation between order statistics (GemmBackendComparison.TimingStats)."""
    if not sorted_v:
        return float("nan")
    if len(sorted_v) == 1:
        return sorted_v[0]
    pos = q * (len(sorted_v) - 1)
    lo, hi = int(pos // 1), int(-(-pos // 1))
    if lo == hi:
        return sorted_v[lo]
    w = pos - lo
    return sorted_v[lo] * (1.0 - w) + sorted_v[hi] * w


def run_harness(args):
    """The reference's parity-gated GEMM backend comparison
    (GemmBackendComparison.java:48-400, report columns :509-545), rerun here:
    square sizes with GemmReference.seededMatrix inputs (seed + 31*size + 11 /
    + 29), alpha = 1, beta = 0; every backend's C checked against
    GemmReference.gemm (independent oracle) with the reference's tolerances
    (GemmReference.java:175-181: CPU 1e-9 / rel 1e-12, GPU 1e-8 / rel 1e-10,
    scaled by max|C| and k/16) before it is timed; timing as the reference's:
    warm-ups, then iterations of max(1, 20M/flops) back-to-back calls, median /
    mean / stddev / percentiles per call; speed-up against opt-1t (the naive
    backend is not restated).  Backends: opt-1t and opt-parallel are the C
    restatement of OptimizedBLAS3 (the CPU baseline, run from the oracle);
    cuda is this library's FP64 route and cuda-ozaki its Ozaki residue route,
    both through the CudaGemm mirror on host arrays (copies included, as
    CudaGemm's calls are).  The blas3-* backends are not restated: SKIPPED."""
    import datetime
    import platform
    import numpy as np
    from oracle import oracle as O
    import jlc_b200
    from jlc_b200 import JLC_PREC_NATIVE, JLC_PREC_OZAKI_CRT, Matrix
    from jlc_b200.compute import CudaGemm
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    jlc_b200.Context(local)  # the library loads and the device answers before anything is timed
    threads = os.cpu_count() or 1
    now = datetime.datetime.now(datetime.timezone.utc)
    stamp_iso, stamp = now.strftime("%Y-%m-%dT%H:%M:%SZ"), now.strftime("%Y%m%dT%H%M%SZ")
    sizes = [int(x) for x in args.sizes.split(",") if x.strip()]
    seed = 20260604

    def execute(backend, a, b, size):
        c = np.zeros((size, size))
        if backend in ("opt-1t", "opt-parallel"):
            out, _ = O.opt_gemm(a, b, c, 1.0, 0.0, threads=1 if backend == "opt-1t" else threads)
            return out
        prec = JLC_PREC_NATIVE if backend == "cuda" else JLC_PREC_OZAKI_CRT
        cm = Matrix.wrap(c.ravel(), size, size)
        if not CudaGemm.gemm(Matrix.wrap(a.ravel(), size, size), Matrix.wrap(b.ravel(), size, size), cm, 1.0,
                             0.0, precision=prec):
            return None
        return cm.to_numpy()

    rows = []
    for size in sizes:
        a = O.seeded_matrix(size, size, seed + size * 31 + 11)
        b = O.seeded_matrix(size, size, seed + size * 31 + 29)
        ref = O.gemm_reference(a, b, np.zeros((size, size)), 1.0, 0.0).ravel()
        ref_norm = float(np.sqrt(np.sum(ref * ref)))
        maxref = float(np.max(np.abs(ref))) if ref.size else 0.0
        for backend in HARNESS_BACKENDS:
            gpu = backend.startswith("cuda")
            row = dict.fromkeys(HARNESS_COLUMNS)
            row.update(timestamp=stamp_iso, size=size, m=size, k=size, n=size, backend=backend,
                       threads=threads if backend in ("opt-parallel", "blas3-parallel") else 1,
                       oracle_type="independent", reference_backend="", warmups=args.warmups, iters=args.iters)
            if backend.startswith("blas3"):
                row.update(valid=False, parity_status="SKIPPED",
                           notes="BLAS3Kernels paths are not restated here; OptimizedBLAS3 (opt-*) is.")
                rows.append(row)
                continue
            out = execute(backend, a, b, size)
            if out is None:
                row.update(valid=False, parity_status="SKIPPED", notes="GPU route returned false.")
                rows.append(row)
                continue
            diff = out.ravel() - ref
            rel = 0.0 if ref_norm == 0.0 else float(np.sqrt(np.sum(diff * diff))) / ref_norm
            mae = float(np.max(np.abs(diff))) if diff.size else 0.0
            abs_tol = max(1e-12, (1e-8 if gpu else 1e-9) * max(1.0, maxref) * max(1.0, size / 16.0))
            rel_tol = 1e-10 if gpu else 1e-12
            row.update(rel_residual=rel, max_abs_err=mae)
            if not (mae <= abs_tol and rel <= rel_tol):
                row.update(valid=False, parity_status="FAIL",
                           notes=f"Parity exceeded tolerances relTol={rel_tol:g} absTol={abs_tol:g}.")
                rows.append(row)
                continue
            flops = 2 * size ** 3
            inner = max(1, -(-20_000_000 // flops))
            checksum = 0.0
            weights = np.arange(1, size * size + 1, dtype=np.float64)
            for _ in range(args.warmups):
                for _ in range(inner):
                    checksum += float(np.dot(execute(backend, a, b, size).ravel(), weights))
            per_call = []
            for _ in range(args.iters):
                t0 = time.perf_counter_ns()
                for _ in range(inner):
                    o = execute(backend, a, b, size)
                per_call.append((time.perf_counter_ns() - t0) / inner)
                checksum += float(np.dot(o.ravel(), weights))
            srt = sorted(per_call)
            mean = sum(per_call) / len(per_call)
            var = sum((x - mean) ** 2 for x in per_call) / (len(per_call) - 1) if len(per_call) > 1 else 0.0
            med = _percentile(srt, 0.5)
            row.update(valid=True, parity_status="PASS", median_ms=med / 1e6, mean_ms=mean / 1e6,
                       stddev_ms=var ** 0.5 / 1e6, min_ms=srt[0] / 1e6, p10_ms=_percentile(srt, 0.1) / 1e6,
                       p25_ms=_percentile(srt, 0.25) / 1e6, p75_ms=_percentile(srt, 0.75) / 1e6,
                       p90_ms=_percentile(srt, 0.9) / 1e6, gflops_median=flops / med if med > 0 else None,
                       checksum=checksum,
                       notes={"opt-1t": "C restatement of OptimizedBLAS3, one thread.",
                              "opt-parallel": "C restatement of OptimizedBLAS3 PARALLEL_MICRO, all host threads.",
                              "cuda": "libjlcgpu FP64 route through CudaGemm (host arrays, copies included).",
                              "cuda-ozaki": "libjlcgpu Ozaki residue route through CudaGemm (host arrays, copies "
                                            "included)."}[backend])
            rows.append(row)
        base = next((r for r in rows if r["size"] == size and r["backend"] == "opt-1t" and r["valid"]), None)
        if base and base["median_ms"]:
            for r in rows:
                if r["size"] == size and r["valid"] and r["median_ms"]:
                    r["baseline_label"] = "opt-1t"
                    r["speedup_vs_baseline"] = base["median_ms"] / r["median_ms"]

    def csv_cell(col, v):
        if col in ("timestamp", "backend", "parity_status", "oracle_type", "reference_backend", "baseline_label",
                   "notes"):
            return '"' + ("" if v is None else str(v)).replace('"', '""') + '"'
        if isinstance(v, bool):
            return "true" if v else "false"
        if v is None or (isinstance(v, float) and (v != v or v in (float("inf"), float("-inf")))):
            return ""
        return repr(v) if isinstance(v, float) else str(v)

    os.makedirs(args.report_dir, exist_ok=True)
    stable = os.path.join(args.report_dir, "gemm-backend-comparison.csv")
    stamped = os.path.join(args.report_dir, f"gemm-backend-comparison-{stamp}.csv")
    js = os.path.join(args.report_dir, "gemm-backend-comparison.json")
    lines = [",".join(HARNESS_COLUMNS)] + [",".join(csv_cell(c, r[c]) for c in HARNESS_COLUMNS) for r in rows]
    for path in (stable, stamped):
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")
    meta = {"timestamp_utc": stamp_iso, "os": platform.platform(), "available_processors": threads,
            "cpu_model": platform.processor(), "gpu": torch.cuda.get_device_name(local),
            "library": "libjlcgpu", "warmups": args.warmups, "iterations": args.iters, "seed": seed}
    with open(js, "w") as f:
        json.dump({"metadata": meta, "artifacts": {"stable_csv": os.path.abspath(stable),
                                                   "timestamped_csv": os.path.abspath(stamped),
                                                   "json": os.path.abspath(js)},
                   "rows": rows}, f, indent=2)
    print(f"{'size':>6} {'backend':>14} {'parity':>8} {'median_ms':>11} {'GFLOP/s':>10} {'speedup':>9}")
    for r in rows:
        fmt = lambda v, spec: format(v, spec) if isinstance(v, (int, float)) and v is not None else "-"
        print(f"{r['size']:>6} {r['backend']:>14} {r['parity_status']:>8} {fmt(r['median_ms'], '11.4f'):>11} "
              f"{fmt(r['gflops_median'], '10.1f'):>10} {fmt(r['speedup_vs_baseline'], '9.2f'):>9}")
    print(json.dumps({"harness_rows": len(rows), "fail": sum(r["parity_status"] == "FAIL" for r in rows),
                      "artifacts": [stable, stamped, js]}), flush=True)
    return 1 if any(r["parity_status"] == "FAIL" for r in rows) else 0


def run_shape(args):
    """One device product of the given shape and precision, timed (the case an
    ncu capture of a single kernel runs: few launches before the timed ones)."""
    import torch
    import jlc_b200
    m, n, k = (int(x) for x in args.mnk.split(","))
    torch.cuda.set_device(0)
    ctx = jlc_b200.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    g = torch.Generator(device="cuda")
    g.manual_seed(20260604)
    la, lb = (0 if x == "r" else 1 for x in args.layouts)
    with torch.cuda.stream(stream):
        # op(A) is m x k, op(B) k x n; a column-major operand is stored as its transpose
        A = torch.rand((m, k) if la == 0 else (k, m), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        B = torch.rand((k, n) if lb == 0 else (n, k), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        C = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    stream.synchronize()

    def call(report=False):
        return ctx.dgemm_device(la, lb, m, n, k, 1.0, A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1], 0.0,
                                C.data_ptr(), n, precision=args.precision, report=report)

    rep = call(report=True)
    for _ in range(args.warmup - 1):
        call()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        call()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    nbytes = 8.0 * (m * k + k * n + m * n)
    print(json.dumps({"workload": "shape", "m": m, "n": n, "k": k, "layouts": args.layouts,
                      "precision": args.precision,
                      "kernel": rep["kernel"], "ms": round(ms, 4),
                      "gflops": round(2.0 * m * n * k / (ms * 1e-3) / 1e9, 1),
                      "gbs_algorithmic": round(nbytes / (ms * 1e-3) / 1e9, 1)}), flush=True)
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "grouped":
        return run_grouped(args)
    if args.workload == "configs":
        return run_configs(args)
    if args.workload == "harness":
        return run_harness(args)
    if args.workload == "shape":
        return run_shape(args)
    if args.workload == "hessenberg":
        return run_hessenberg(args)
    if args.workload == "bidiag":
        return run_bidiag(args)
    if args.workload == "qr":
        return run_qr(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
