#!/usr/bin/env python
"""Benchmark of the SGEMM hot path: C = A*B in FP32 at M = N = K = 8192.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--variant bf16x6|bf16x3|bf16x6_scaled|bf16x3_scaled|ffma] [--n 8192]

Metric: effective FP32 TFLOP/s (2*N^3 / step time) at a stated error against
an FP64 product. One step = one full C = A*B through the C ABI: for the
split-BF16 forms the split pass (split-only call) followed by the
tensor-core product (pre-split call), for FFMA one call. Inputs are seeded
i.i.d. U[-1,1) float32 built on the device; each operand is 268 MB (larger
than the 126 MB L2), so no flush is needed between steps. `value` sums over
ranks: every rank runs its own replica (the path does not shard).

The same line carries the plain FFMA kernel on the same inputs ("ffma"), the
error of both against the FP64 product, `e2e` (the public call with pinned
host buffers: H2D of A and B and D2H of C of every step inside the timed
region, steps pipelined over copy and compute streams), the
roofline of the dominant kernel, the clocks seen during the timed region and
the CPU baseline (the reference host_mm loop on the host cores).

--impl reference times the reference's CPU implementation of the path (the
host_mm loop of apps/sgemm/main.cpp:15-26, restated in oracle/oracle.c) on
the host cores, on a row sample of the same workload (rows are independent,
so cost is linear in rows).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "effective FP32 TFLOP/s at stated error vs FP64: split-BF16 TC vs plain FFMA, 1 B200"
SMS = 148  # B200 SM count, for the derived FP32 figure reported beside the measured one
FP32_LANES_PER_SM = 128
PRODUCTS = {"bf16x3": 3, "bf16x6": 6, "bf16x3_scaled": 3, "bf16x6_scaled": 6}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        d["source"] = "measured"
        return d
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "sm_max_mhz": 1965.0, "source": "fallback"}


def _profile_traffic(name: str):
    """DRAM bytes per launch of a kernel and workload from one ncu capture, as
    recorded in profiles/traffic.json (key: kernel and workload), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        entry = json.load(open(p)).get(name)
    except (OSError, ValueError):
        return None
    return int(entry["dram_bytes_per_launch"]) if entry else None


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    """nvidia-smi samples every 100 ms; only samples taken inside the marked
    timed windows are summarised."""
    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None
        self.windows = []

    def window(self, t0: float, t1: float):
        import datetime
        self.windows.append((datetime.datetime.fromtimestamp(t0),
                             datetime.datetime.fromtimestamp(t1)))

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu_index)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        import datetime
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
            except ValueError:
                continue
            if self.windows and not any(a <= ts <= b for a, b in self.windows):
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                pw.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference host_mm loop on a row sample

class _CpuSampler:
    """The reference's host_mm loop (the oracle port) on a bounded row sample
    of the n^3 product: B and the per-row cost are prepared once, and each
    sample() times `seconds` worth of rows (the cost is linear in rows)."""

    def __init__(self, n: int, threads: int = 0):
        import numpy as np

        from oracle import oracle
        self.oracle = oracle
        self.n = n
        self.rng = np.random.Generator(np.random.PCG64(42))
        self.B = self.rng.uniform(-1, 1, size=(n, n)).astype(np.float32)
        self.nthreads = threads or len(os.sched_getaffinity(0))
        nt = self.nthreads
        # one untimed pass starts the thread pool and touches B, then the
        # per-row cost is timed over two rows per thread
        oracle.host_mm(self.rng.uniform(-1, 1, size=(nt, n)).astype(np.float32), self.B,
                       threads=nt)
        A = self.rng.uniform(-1, 1, size=(2 * nt, n)).astype(np.float32)
        t0 = time.perf_counter()
        oracle.host_mm(A, self.B, threads=nt)
        self.per_row = (time.perf_counter() - t0) / (2 * nt)

    def sample(self, seconds: float, min_rows: int = 0) -> dict:
        import numpy as np
        n, nt = self.n, self.nthreads
        rows = int(max(nt, min_rows, min(n, seconds / max(self.per_row, 1e-9))))
        rows = min(n, max(nt, -(-rows // nt) * nt))
        A = self.rng.uniform(-1, 1, size=(rows, n)).astype(np.float32)
        t0 = time.perf_counter()
        self.oracle.host_mm(A, self.B, threads=nt)
        dt = time.perf_counter() - t0
        flops = 2.0 * rows * n * n
        return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": nt, "kind": "port",
                "sample": f"host_mm loop (apps/sgemm/main.cpp:15-26 restated, gcc -O3) on {rows} of "
                          f"{n} output rows of the {n}^3 product, {dt:.1f} s, OpenMP over rows; "
                          "cost is linear in rows"}


def cpu_baseline(n: int, seconds: float = 12.0, threads: int = 0) -> dict:
    return _CpuSampler(n, threads).sample(seconds)


# ---------------------------------------------------------------------------

def replica_throughput(local_ms: float, flops_per_step: float, steps: int,
                       world: int = 1, device=None) -> tuple[float, float]:
    """Whole-job throughput of `world` replicas that each ran `steps` steps of
    `flops_per_step`: the job time is the maximum of the ranks' device times
    (an all-reduce over the default process group when world > 1). Returns
    (max time in ms, TFLOP/s summed over ranks)."""
    t = local_ms
    if world > 1:
        import torch
        import torch.distributed as dist
        x = torch.tensor([local_ms], dtype=torch.float64, device=device)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        t = float(x.item())
    return t, world * flops_per_step * steps / (t * 1e-3) / 1e12


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


REF_MIN_ROWS = 128  # rows of the product timed per reference step, at least


def run_reference(args) -> None:
    ws, rank, _ = _dist()
    if rank != 0:
        return
    n = args.n
    per_step = max(2.0, 60.0 / (args.steps + args.warmup))
    vals = []
    cb = None
    sampler = _CpuSampler(n)
    for i in range(args.warmup + args.steps):
        cb = sampler.sample(per_step, min_rows=REF_MIN_ROWS)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.median(vals)
    flops = 2.0 * n ** 3
    line = {
        "impl": "reference", "metric": METRIC,
        "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": flops / (v * 1e12) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded i.i.d. U[-1,1) float32",
        "config": {"workload": f"sgemm M=N=K={n} fp32 row-major", "m": n, "n": n, "k": n},
        "cpu_baseline": {**cb, "value": v},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _err(C, ref) -> dict:
    import torch
    d = C.double() - ref
    return {"max_abs": float(d.abs().max()),
            "rel_fro": float(torch.linalg.norm(d) / torch.linalg.norm(ref))}


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    import hb_hammerbench_b200 as hb
    from hb_hammerbench_b200 import _lib

    ws, rank, local = _dist()
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    variant = args.variant
    split = variant != "ffma"
    flops = 2.0 * n ** 3
    warmup = max(3, args.warmup)

    g = torch.Generator(device=dev).manual_seed(42 + rank)
    A = torch.rand((n, n), device=dev, generator=g) * 2 - 1
    B = torch.rand((n, n), device=dev, generator=g) * 2 - 1
    C = torch.empty((n, n), device=dev)
    # the schedule every call below runs: the autotuner's choice for this
    # shape class when the package ships one, else the library heuristic
    sched = hb.resolve_config(n, n, n, variant, False, None) or {}
    tile_info = {t["tile"]: t for t in hb.tiles()}
    if split:
        tile = sched.get("tile") or 0
        fused = bool(tile and tile_info[tile]["fused"])
    else:
        fused = False
    wsz = hb.gemm_workspace_size(n, n, n, variant, config=sched or None)
    wsp = torch.empty(max(wsz, 256), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    # split-BF16 step = split-only call (the split passes; for a fused-split
    # schedule only the scaled forms' row/column maxima) + pre-split call (the
    # tensor-core product), so the product kernel can be timed on its own
    split_only = {**sched, "flags": _lib.FLAG_SPLIT_ONLY}
    presplit = {**sched, "flags": _lib.FLAG_PRESPLIT_A | _lib.FLAG_PRESPLIT_B}

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    sampler = ClockSampler(local)  # summarises the samples inside the timed windows

    def timed(step_fn, steps, per_step=True):
        """K steps on `stream`; returns (total ms max over ranks, per-step kernel ms)."""
        for _ in range(warmup):
            step_fn(None)
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        barrier()
        w0 = time.time()
        t0.record(stream)
        for i in range(steps):
            step_fn(evs[i] if per_step else None)
        t1.record(stream)
        barrier()
        sampler.window(w0, time.time())
        total, _ = replica_throughput(t0.elapsed_time(t1), flops, steps, ws, dev)
        return total, ([a.elapsed_time(b) for a, b in evs] if per_step else [])

    def step_main(ev):
        if split:
            hb.gemm(A, B, C, variant=variant, workspace=wsp, config=split_only)
            if ev:
                ev[0].record(stream)
            hb.gemm(A, B, C, variant=variant, workspace=wsp, config=presplit)
            if ev:
                ev[1].record(stream)
        else:
            if ev:
                ev[0].record(stream)
            hb.gemm(A, B, C, variant="ffma")
            if ev:
                ev[1].record(stream)

    sampler.start()
    time.sleep(0.3)
    total_ms, kern_ms = timed(step_main, args.steps)
    ms_per_step = total_ms / args.steps
    value = ws * flops * args.steps / (total_ms * 1e-3) / 1e12  # total_ms: max over ranks

    if args.profile:
        sampler.stop()
        if rank == 0:
            print(json.dumps({"profile_run": True, "variant": variant, "ms_per_step": ms_per_step}),
                  flush=True)
        if ws > 1:
            dist.destroy_process_group()
        return

    ref = A.double() @ B.double()
    err = _err(C, ref)

    # plain FFMA kernel on the same inputs, for the comparison the metric names
    ffma = None
    if split and not args.no_compare:
        C2 = torch.empty_like(C)

        def step_ffma(ev):
            if ev:
                ev[0].record(stream)
            hb.gemm(A, B, C2, variant="ffma")
            if ev:
                ev[1].record(stream)
        f_total, f_kern = timed(step_ffma, max(3, args.steps // 2))
        f_steps = max(3, args.steps // 2)
        f_val = ws * flops * f_steps / (f_total * 1e-3) / 1e12
        ffma = {"value": f_val, "unit": "TFLOP/s", "ms_per_step": f_total / f_steps,
                "error_vs_fp64": _err(C2, ref), "kernel": "ffma_sgemm_kernel",
                "schedule": hb.resolve_config(n, n, n, "ffma", False, None) or "heuristic",
                "kernel_ms": statistics.mean(f_kern)}
        del C2
    del ref

    # e2e through the public API with pinned host buffers: every step copies
    # its A and B host->device and its C device->host inside the timed
    # region. Steps are pipelined over three streams (H2D, compute, D2H) with
    # double-buffered device operands, so a step's copies overlap its
    # neighbours' compute and the two copy directions overlap each other.
    hA = A.cpu().pin_memory()
    hB = B.cpu().pin_memory()
    hC = [torch.empty((n, n), dtype=torch.float32).pin_memory() for _ in range(2)]
    dA = [torch.empty_like(A) for _ in range(2)]
    dB = [torch.empty_like(B) for _ in range(2)]
    dC = [torch.empty_like(C) for _ in range(2)]
    s_in = torch.cuda.Stream(device=dev)
    s_out = torch.cuda.Stream(device=dev)

    def e2e_steps(steps, start=None, end=None):
        ev = lambda: torch.cuda.Event()  # noqa: E731
        in_done = [ev() for _ in range(steps)]
        cmp_done = [ev() for _ in range(steps)]
        out_done = [ev() for _ in range(steps)]
        s_in.wait_stream(stream)
        if start is not None:
            start.record(s_in)
        for i in range(steps):
            b = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(cmp_done[i - 2])  # buffers b no longer read
                dA[b].copy_(hA, non_blocking=True)
                dB[b].copy_(hB, non_blocking=True)
                in_done[i].record(s_in)
            stream.wait_event(in_done[i])
            if i >= 2:
                stream.wait_event(out_done[i - 2])  # dC[b] already copied out
            hb.gemm(dA[b], dB[b], dC[b], variant=variant, workspace=wsp, config=sched or None)
            cmp_done[i].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(cmp_done[i])
                hC[b].copy_(dC[b], non_blocking=True)
                out_done[i].record(s_out)
        if end is not None:
            end.record(s_out)
        stream.wait_stream(s_out)

    e2e_steps(3)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e2e_steps(args.steps, e0, e1)
    barrier()
    sampler.window(w0, time.time())
    e_total, e2e_val = replica_throughput(e0.elapsed_time(e1), flops, args.steps, ws, dev)
    clocks = sampler.stop()
    assert torch.equal(hC[(args.steps - 1) % 2], dC[(args.steps - 1) % 2].cpu())
    assert torch.equal(dC[(args.steps - 1) % 2], C)  # same inputs, same result

    peaks = _peaks()
    fp32 = hb.fp32_peak(packed=True, iters=200000)  # measured FP32 SIMT roof, this device
    fp32_scalar = hb.fp32_peak(packed=False, iters=200000)
    avg_kernel_ms = statistics.mean(kern_ms)
    if split:
        prods = PRODUCTS[variant]
        mma_flops = prods * flops
        achieved = mma_flops / (avg_kernel_ms * 1e-3) / 1e12
        tile = sched.get("tile") or 0
        pair = bool(tile and tile_info[tile]["bm"] == 256)
        kname = "tc_fused_kernel" if fused else ("tc_pair_kernel" if pair else "tc_gemm_kernel")
        traffic = _profile_traffic(f"{kname[:-7]}_{variant}_n{n}")
        roof = {"bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"],
                "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops"], "traffic": traffic,
                "kernel": kname, "algorithmic_flops_per_launch": mma_flops,
                "flops_note": f"{prods} BF16 products x 2*N^3 executed on the tensor cores per launch; "
                              f"peak = {peaks['source']} cuBLAS bf16 burst",
                "frac_of_sustained": achieved / peaks["bf16_tflops_sustained"],
                "kernel_ms": avg_kernel_ms,
                "effective_fp32_tflops_of_kernel": flops / (avg_kernel_ms * 1e-3) / 1e12}
        # per step: split passes (A, B; none when fused), row/column maxima
        # (scaled forms), the product kernel
        launches = args.steps * ((0 if fused else 2) + (2 if "scaled" in variant else 0) + 1)
    else:
        roof = _ffma_roofline(statistics.mean(kern_ms), flops, fp32, n)
        launches = args.steps
    if ffma is not None:
        ffma["roofline"] = _ffma_roofline(ffma.pop("kernel_ms"), flops, fp32, n)

    line = {
        "metric": METRIC,
        "value": value, "unit": "TFLOP/s", "n_gpus": ws, "steps": args.steps,
        "warmup": warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded i.i.d. U[-1,1) float32, built on the device",
        "config": {"workload": f"sgemm M=N=K={n} fp32 row-major, variant {variant}",
                   "m": n, "n": n, "k": n, "variant": variant, "schedule": sched or "heuristic",
                   "fused_split": fused,
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single",
                   "l2": "inputs (268 MB each) larger than L2; no flush"},
        "error_vs_fp64": {**err, "reference": "FP64 product of the same inputs (torch float64 "
                                               "matmul on the GPU)"},
        "e2e": {"value": e2e_val, "unit": "TFLOP/s", "h2d_bytes_per_step": 2 * n * n * 4,
                "d2h_bytes_per_step": n * n * 4, "ms_per_step": e_total / args.steps,
                "pipelining": "H2D / compute / D2H streams, double-buffered device operands"},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clocks,
    }
    line["fp32_peak_measured"] = {
        "packed_ffma2_tflops": fp32["tflops"], "scalar_ffma_tflops": fp32_scalar["tflops"],
        "probe": "hbsg_fp32_peak_probe: 8 independent FMA chains per thread, 4 CTAs x 256 "
                 "threads per SM, best of 5 launches (CUDA events)",
        "derived_tflops_at_sm_max": SMS * FP32_LANES_PER_SM * 2 *
        (clocks.get("sm_max_mhz") or peaks["sm_max_mhz"]) * 1e6 / 1e12}
    if ffma is not None:
        line["ffma"] = ffma
        line["speedup_vs_ffma"] = value / ffma["value"]
        line["error_ratio_vs_ffma"] = err["rel_fro"] / ffma["error_vs_fp64"]["rel_fro"]
    if not args.no_legs:
        del A, B, C, wsp, dA, dB, dC, hA, hB, hC
        torch.cuda.empty_cache()
        line["configs"] = _config_legs(hb, peaks, fp32["tflops"], value,
                                       ffma["value"] if ffma else None)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


def _ffma_roofline(kernel_ms: float, flops: float, fp32: dict, n: int) -> dict:
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    return {"bound": "fp32_simt", "achieved": achieved, "peak": fp32["tflops"],
            "unit": "TFLOP/s", "frac": achieved / fp32["tflops"],
            "traffic": _profile_traffic(f"ffma_sgemm_n{n}"), "kernel": "ffma_sgemm_kernel",
            "algorithmic_flops_per_launch": flops, "kernel_ms": kernel_ms,
            "flops_note": "2*N^3 FP32 flops per launch; peak = the FP32 SIMT probe "
                          "(packed __ffma2_rn, the instruction the kernel issues) measured "
                          "on this device in this run"}


# Workloads measured beside the headline: the uneven grouped
# batch (512 problems) and the two awkward shapes, each one named case of the
# sweep driver (seeded device inputs larger than L2; error vs FP64).
LEGS = [
    ("grouped_512_bf16x6", "GROUPED_512__SEED_0__V_bf16x6", 6),
    ("grouped_512_ffma", "GROUPED_512__SEED_0__V_ffma", 0),
    ("tallk_256x256x1048576_bf16x6", "M_256__N_256__K_1048576__V_bf16x6", 6),
    ("tallk_256x256x1048576_bf16x3", "M_256__N_256__K_1048576__V_bf16x3", 3),
    ("tallm_65536x64x4096_bf16x6", "M_65536__N_64__K_4096__V_bf16x6", 6),
    ("tallm_65536x64x4096_bf16x3", "M_65536__N_64__K_4096__V_bf16x3", 3),
    ("tallm_65536x64x4096_ffma", "M_65536__N_64__K_4096__V_ffma", 0),
]


BS_LEGS = [
    ("blackscholes_10M_records", "num-option_10000000"),
    ("blackscholes_10M_arrays", "num-option_10000000__LAYOUT_arrays"),
]
JACOBI_LEG = ("jacobi_512x512x512", "nx_512__ny_512__nz_512")


def _config_legs(hb, peaks: dict, fp32_tflops: float, single_x6: float, single_ffma) -> dict:
    """Each leg: effective TFLOP/s of the whole step (split passes included),
    its error vs FP64, and the fraction of its roof: the lower of the compute
    roof (BF16 burst / products, or the measured FP32 SIMT roof) and the HBM
    roof (measured copy bandwidth x the step's algorithmic flop per byte:
    2*M*N*K over 4*(M*K + K*N + M*N) bytes, summed over problems)."""
    import torch

    from hb_hammerbench_b200 import sweep
    out = {}
    for key, case, prods in LEGS:
        r = sweep.run_case(case, steps=5, warmup=3)
        c = sweep.parse_case(case)
        if "GROUPED" in c:
            dims = sweep.grouped_dims(c["GROUPED"], c.get("SEED", 0))
        else:
            dims = [(c["M"], c["N"], c["K"])]
        fl = float(sum(2.0 * m * n * k for m, n, k in dims))
        by = float(sum(4.0 * (m * k + k * n + m * n) for m, n, k in dims))
        compute = peaks["bf16_tflops"] / prods if prods else fp32_tflops
        hbm = peaks["hbm_gbs"] * 1e9 * (fl / by) / 1e12
        roof = min(compute, hbm)
        leg = {"case": case, "value": r["tflops"], "unit": "TFLOP/s", "ms_per_step": r["ms"],
               "error_vs_fp64": r["error_vs_fp64"],
               "roofline": {"bound": "hbm" if hbm < compute else ("tensor" if prods else "fp32_simt"),
                            "roof_tflops": roof, "compute_roof_tflops": compute,
                            "hbm_roof_tflops": hbm, "frac": r["tflops"] / roof,
                            "algorithmic_bytes": by}}
        if "GROUPED" in c:
            single = single_x6 if prods else single_ffma
            if single:
                leg["ratio_to_single_8192"] = r["tflops"] / single
        out[key] = leg
        torch.cuda.empty_cache()
    # Black-Scholes (apps/blackscholes) at the size of the benchmark's input
    # file, 10 M options, on both layouts: HBM-bound, so the roof is the
    # measured copy bandwidth over the layout's DRAM bytes per option.
    for key, case in BS_LEGS:
        r = sweep.run_case(case, steps=20, warmup=3)
        out[key] = {"case": case, "value": r["moptions_per_s"], "unit": "Moptions/s",
                    "ms_per_step": r["ms"], "changed_after_repeat": r["changed_after_repeat"],
                    "roofline": {"bound": "hbm", "achieved": r["dram_gbs"],
                                 "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                 "frac": r["dram_gbs"] / peaks["hbm_gbs"],
                                 "bytes_per_option": r["bytes_per_option"]}}
        torch.cuda.empty_cache()
    # Jacobi 7-point step (apps/jacobi) on a 512^3 grid (512 MB in, 512 MB
    # out, larger than L2): HBM-bound at 8 bytes per point
    key, case = JACOBI_LEG
    r = sweep.run_case(case, steps=20, warmup=3)
    out[key] = {"case": case, "value": r["gpoints_per_s"], "unit": "Gpoints/s",
                "ms_per_step": r["ms"], "changed_after_repeat": r["changed_after_repeat"],
                "roofline": {"bound": "hbm", "achieved": r["dram_gbs"], "peak": peaks["hbm_gbs"],
                             "unit": "GB/s", "frac": r["dram_gbs"] / peaks["hbm_gbs"],
                             "bytes_per_point": r["bytes_per_point"]}}
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", default="bf16x6",
                    choices=["ffma", "bf16x3", "bf16x6", "bf16x3_scaled", "bf16x6_scaled"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FFMA comparison run")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the grouped and awkward-shape configuration legs")
    ap.add_argument("--profile", action="store_true",
                    help="timed steps only (no error check, e2e or CPU baseline): for ncu")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
