"""Benchmark driver for named SGEMM cases (the measurement sweep).

    python -m hb_hammerbench_b200.sweep CASE [CASE ...] [--steps K] [--warmup W]
                                        [--profile] [--no-error]

Case names follow the HammerBench launch-directory convention
`N_<n>__NITER_<k>` (apps/sgemm/Makefile:7-12, tests.mk:1): `__`-separated
KEY_value fields. Recognised keys:

  N_<n>__NITER_<k>           NITER independent n x n products (hbsg_sgemm layout)
  M_<m>__N_<n>__K_<k>        one general row-major product
  GROUPED_<count>__SEED_<s>  <count> products with M, N, K drawn uniform from the
                             multiples of 32 in [64, 2048] (numpy PCG64(seed)),
                             run as one grouped plan (CUDA-graph replay)
  V_<variant>                ffma | bf16x3 | bf16x6 | bf16x3_scaled | bf16x6_scaled
  DIST_<d>                   uniform (U[-1,1), default) | wide (sign * 2^u, u ~ U[-20,20])
  SPLITK_<s> / TILE_<t> / CHUNK_<c> / RASTER_<r>
                             explicit schedule (hbsg_config.split_k / .tile / .chunk_k /
                             .raster_group)
  num-option_<n>             Black-Scholes (apps/blackscholes/tests.mk:1): n seeded
                             synthetic option records priced in place
  LAYOUT_<l>                 Black-Scholes layout: records (default) | arrays
  nx_<x>__ny_<y>__nz_<z>     Jacobi 7-point step (apps/jacobi/tests.mk:1-2) on a
                             seeded U[-1,1) grid, c0 = 2, c1 = 4

Examples: N_512__NITER_2, N_8192__NITER_1__V_bf16x6, M_256__N_256__K_1048576__V_bf16x6,
GROUPED_512__SEED_0__V_bf16x6, N_8192__NITER_1__V_bf16x6_scaled__DIST_wide,
num-option_32768, num-option_10000000__LAYOUT_arrays, nx_512__ny_512__nz_512.

Each case prints one JSON line: effective TFLOP/s (sum of 2*M*N*K over the
step time, CUDA events over the timed steps), and unless --no-error the
max-abs and relative Frobenius error of the result against an FP64 product
of the same inputs (torch float64 matmul on the GPU). Inputs are seeded and
generated on the device. --profile runs warm-up and timed steps only (for
Nsight Compute). Black-Scholes cases print options per second and the DRAM
bytes per second of the layout (records: the 32-byte record read and written
back, 64 bytes per option; arrays: 20 bytes read and 8 written), and instead
of the FP64 error the count of options that differ from the first step.
Jacobi cases print grid points per second and DRAM bytes per second (4 bytes
read and 4 written per point), and the count of points that differ from the
first step.
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np
import torch

from .sgemm import GroupedPlan, gemm, gemm_workspace_size, sgemm, sgemm_workspace_size

VARIANTS = ("ffma", "bf16x3", "bf16x6", "bf16x3_scaled", "bf16x6_scaled")


def parse_case(name: str) -> dict:
    """`N_512__NITER_2` -> {'N': 512, 'NITER': 2}; values stay strings when
    they are not integers."""
    out = {}
    for field in name.split("__"):
        key, _, val = field.partition("_")
        if not key or not val:
            raise ValueError(f"bad case field {field!r} in {name!r}")
        out[key.upper()] = int(val) if val.lstrip("-").isdigit() else val.lower()
    if "V" in out and out["V"] not in VARIANTS:
        raise ValueError(f"unknown variant {out['V']!r}")
    if ("GROUPED" not in out and "N" not in out and "NUM-OPTION" not in out
            and "NX" not in out):
        raise ValueError(f"case {name!r} names no problem size")
    return out


def grouped_dims(count: int, seed: int) -> np.ndarray:
    """M, N, K for the uneven batch: uniform over the multiples of 32 in [64, 2048]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.integers(2, 65, size=(count, 3)) * 32


def _inputs(shapes, dist: str, seed: int, device):
    """One device buffer holding every operand (few launches), as views."""
    total = int(sum(m * k + k * n for m, n, k in shapes))
    g = torch.Generator(device=device).manual_seed(seed)
    buf = torch.rand(total, device=device, generator=g) * 2 - 1
    if dist == "wide":
        u = torch.rand(total, device=device, generator=g) * 40 - 20
        buf = torch.sign(buf) * torch.exp2(u)
    As, Bs, off = [], [], 0
    for m, n, k in shapes:
        As.append(buf[off:off + m * k].view(m, k))
        off += m * k
        Bs.append(buf[off:off + k * n].view(k, n))
        off += k * n
    return As, Bs


def _config(c: dict):
    cfg = {}
    if "SPLITK" in c:
        cfg["split_k"] = c["SPLITK"]
    if "TILE" in c:
        cfg["tile"] = c["TILE"]
    if "CHUNK" in c:
        cfg["chunk_k"] = c["CHUNK"]
    if "RASTER" in c:
        cfg["raster_group"] = c["RASTER"]
    return cfg or None


BS_LAYOUT_BYTES = {"records": 64, "arrays": 28}  # DRAM bytes per option


def _timed(step, steps: int, warmup: int) -> float:
    """Mean ms per step over `steps` steps after `warmup`, CUDA events on the
    current stream."""
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_blackscholes(name: str, steps: int = 10, warmup: int = 3, check: bool = True,
                     device=None) -> dict:
    from . import blackscholes as bs
    c = parse_case(name)
    n = c["NUM-OPTION"]
    layout = c.get("LAYOUT", "records")
    if layout not in BS_LAYOUT_BYTES:
        raise ValueError(f"unknown layout {layout!r}")
    device = device or torch.device("cuda", torch.cuda.current_device())
    rec = torch.from_numpy(bs.option_records(n, c.get("SEED", 0))).to(device)
    if layout == "records":
        def step():
            bs.price(rec)
        outputs = lambda: rec[:, 5:7].clone()  # noqa: E731
    else:
        cols = [rec[:, j].contiguous() for j in range(5)]
        call, put = torch.empty_like(cols[0]), torch.empty_like(cols[0])

        def step():
            bs.price_arrays(*cols, call=call, put=put)
        outputs = lambda: torch.stack([call, put], 1)  # noqa: E731
    step()
    torch.cuda.synchronize()
    first = outputs()
    ms = _timed(step, steps, warmup)
    res = {"case": name, "layout": layout, "options": n, "ms": ms,
           "moptions_per_s": n / (ms * 1e-3) / 1e6,
           "dram_gbs": n * BS_LAYOUT_BYTES[layout] / (ms * 1e-3) / 1e9,
           "bytes_per_option": BS_LAYOUT_BYTES[layout]}
    if check:
        res["changed_after_repeat"] = int((outputs() != first).any(1).sum())
    return res


def run_jacobi(name: str, steps: int = 10, warmup: int = 3, check: bool = True,
               device=None) -> dict:
    from .sgemm import jacobi
    c = parse_case(name)
    nx, ny, nz = c["NX"], c["NY"], c["NZ"]
    device = device or torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=device).manual_seed(c.get("SEED", 0))
    a = torch.rand(nx * ny * nz, device=device, generator=g) * 2 - 1
    out = torch.empty_like(a)

    def step():
        jacobi(a, nx, ny, nz, out=out)
    step()
    torch.cuda.synchronize()
    first = out.clone()
    ms = _timed(step, steps, warmup)
    n = nx * ny * nz
    res = {"case": name, "points": n, "ms": ms, "gpoints_per_s": n / (ms * 1e-3) / 1e9,
           "dram_gbs": 8.0 * n / (ms * 1e-3) / 1e9, "bytes_per_point": 8}
    if check:
        res["changed_after_repeat"] = int((out != first).sum())
    return res


def run_case(name: str, steps: int = 10, warmup: int = 3, error: bool = True,
             profile: bool = False, device=None) -> dict:
    c = parse_case(name)
    if "NX" in c:
        return run_jacobi(name, steps, warmup, error and not profile, device)
    if "NUM-OPTION" in c:
        return run_blackscholes(name, steps, warmup, error and not profile, device)
    device = device or torch.device("cuda", torch.cuda.current_device())
    variant = c.get("V", "ffma")
    dist = c.get("DIST", "uniform")
    cfg = _config(c)
    stream = torch.cuda.current_stream()
    if "GROUPED" in c:
        dims = grouped_dims(c["GROUPED"], c.get("SEED", 0))
        shapes = [(int(m), int(n), int(k)) for m, n, k in dims]
        As, Bs = _inputs(shapes, dist, c.get("SEED", 0), device)
        plan = GroupedPlan(As, Bs, variant=variant, config=cfg)
        step = plan.run
        outputs = lambda: plan.Cs  # noqa: E731
    elif "NITER" in c:
        n, niter = c["N"], c["NITER"]
        shapes = [(n, n, n)] * niter
        g = torch.Generator(device=device).manual_seed(c.get("SEED", 42))
        A = torch.rand((niter, n, n), device=device, generator=g) * 2 - 1
        B = torch.rand((niter, n, n), device=device, generator=g) * 2 - 1
        if dist == "wide":
            A = torch.sign(A) * torch.exp2(torch.rand_like(A) * 40 - 20)
            B = torch.sign(B) * torch.exp2(torch.rand_like(B) * 40 - 20)
        C = torch.empty_like(A)
        ws = torch.empty(max(sgemm_workspace_size(n, niter, variant), 256),
                         dtype=torch.uint8, device=device)
        As, Bs = list(A), list(B)

        def step():
            sgemm(A, B, C, n=n, niter=niter, variant=variant, workspace=ws)
        outputs = lambda: list(C)  # noqa: E731
    else:
        m, n, k = c["M"], c["N"], c["K"]
        shapes = [(m, n, k)]
        As, Bs = _inputs(shapes, dist, c.get("SEED", 42), device)
        C = torch.empty((m, n), device=device)
        ws = torch.empty(max(gemm_workspace_size(m, n, k, variant, cfg), 256),
                         dtype=torch.uint8, device=device)

        def step():
            gemm(As[0], Bs[0], C, variant=variant, config=cfg, workspace=ws)
        outputs = lambda: [C]  # noqa: E731

    flops = float(sum(2.0 * m * n * k for m, n, k in shapes))
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    res = {"case": name, "variant": variant, "problems": len(shapes), "gflop": flops / 1e9,
           "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
    if profile or not error:
        return res
    # error against the FP64 product, accumulated over all problems
    num = den = 0.0
    max_abs = 0.0
    for a, b, out in zip(As, Bs, outputs()):
        ref = a.double() @ b.double()
        d = out.double() - ref
        num += float((d * d).sum())
        den += float((ref * ref).sum())
        max_abs = max(max_abs, float(d.abs().max()) if d.numel() else 0.0)
    res["error_vs_fp64"] = {"max_abs": max_abs, "rel_fro": (num / den) ** 0.5 if den else num ** 0.5}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("cases", nargs="+")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--no-error", action="store_true")
    args = ap.parse_args(argv)
    for name in args.cases:
        print(json.dumps(run_case(name, args.steps, args.warmup, not args.no_error,
                                  args.profile)), flush=True)


if __name__ == "__main__":
    sys.exit(main())
