"""Autotuner for the SGEMM schedules (tile shape, K slices, TMEM drain
interval, rasterisation group) and the grouped plans.

The library's built-in heuristic picks a schedule from the shape alone; the
tuner measures candidate schedules on the GPU through the C ABI
(hbsg_gemm_ex / grouped plans with an explicit hbsg_config) and remembers the
fastest per shape class in a JSON cache, together with every candidate's
time as evidence. The reference's nearest analogue is its tile-group shape
sweep (apps/legacy/gemm/sgemm_512/tests.mk:1-6), run by hand.

    from hb_hammerbench_b200 import autotune
    cfg = autotune.tune(4096, 4096, 4096, "bf16x6")   # measures, caches
    cfg = autotune.lookup(4000, 4100, 4096, "bf16x6")  # same shape class
    C = hb.gemm(A, B, variant="bf16x6", config=cfg)

Shape class: the variant and the power-of-two bucket (ceil log2) of M, N
and K. Cache file: $HBSG_AUTOTUNE_CACHE, else
~/.cache/hb_hammerbench_b200/autotune.json (written atomically).

Defaults: the package ships the table this tuner produced on a B200
(tuned_b200.json, regenerated with `python -m hb_hammerbench_b200.autotune
--ship`). lookup() answers from the user cache first, then from that table, so
the host interface (sgemm.gemm, sgemm.GroupedPlan) runs the tuner's choice
for every tuned shape class when the caller passes no schedule; shapes of no
tuned class keep the C library's heuristic. HBSG_AUTOTUNE=0 turns the lookup
off.
"""
from __future__ import annotations

import itertools
import json
import math
import os
import tempfile
import threading

_lock = threading.Lock()
_mem: dict | None = None
_shipped: dict | None = None
_last_entry: dict | None = None  # the table entry of the latest tune / tune_grouped

SHIPPED_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json")


def enabled() -> bool:
    return os.environ.get("HBSG_AUTOTUNE", "1") != "0"


def _load_shipped() -> dict:
    global _shipped
    if _shipped is None:
        try:
            with open(SHIPPED_PATH) as f:
                _shipped = json.load(f)
        except (OSError, ValueError):
            _shipped = {}
    return _shipped


def cache_path() -> str:
    p = os.environ.get("HBSG_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "hb_hammerbench_b200", "autotune.json")


def shape_key(m: int, n: int, k: int, variant: str) -> str:
    def b(x):
        return max(0, math.ceil(math.log2(max(1, x))))
    return f"{variant}:m{b(m)}:n{b(n)}:k{b(k)}"


def grouped_key(dims, variant: str) -> str:
    """Grouped plans: variant, problem count and the bucket of the mean size."""
    dims = list(dims)
    mean = sum(m * n * k for m, n, k in dims) / max(1, len(dims))
    return f"grouped:{variant}:p{len(dims)}:s{round(math.log2(max(1.0, mean)))}"


def _load() -> dict:
    global _mem
    if _mem is None:
        try:
            with open(cache_path()) as f:
                _mem = json.load(f)
        except (OSError, ValueError):
            _mem = {}
    return _mem


def _store(key: str, entry: dict) -> None:
    with _lock:
        data = _load()
        data[key] = entry
        path = cache_path()
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path) or ".", suffix=".tmp")
        with os.fdopen(fd, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def clear_memory_cache() -> None:
    global _mem, _shipped
    _mem = None
    _shipped = None


def _entry(key: str):
    return _load().get(key) or _load_shipped().get(key)


def lookup(m: int, n: int, k: int, variant: str) -> dict | None:
    """Best measured schedule for the shape class (user cache, then the
    shipped table), or None."""
    e = _entry(shape_key(m, n, k, variant))
    return dict(e["config"]) if e else None


def lookup_grouped(dims, variant: str) -> dict | None:
    e = _entry(grouped_key(dims, variant))
    return dict(e["config"]) if e else None


def candidates(m: int, n: int, k: int, variant: str, tiles: list[dict]) -> list[dict]:
    """Schedules worth measuring for one problem shape."""
    fam = "ffma" if variant == "ffma" else "bf16"
    parts = 0 if fam == "ffma" else (3 if "x6" in variant else 2)
    ids = [t["tile"] for t in tiles if t["family"] == fam and t["parts"] == parts]
    out = []
    for tile in ids:
        t = next(x for x in tiles if x["tile"] == tile)
        n_tiles = math.ceil(m / t["bm"]) * math.ceil(n / t["bn"])
        splits = [0]
        if n_tiles < 148 and k >= 1024:
            splits = sorted({1, max(1, 148 // n_tiles), max(1, 296 // n_tiles)})
        if fam == "ffma":
            splits = [1] + ([s for s in splits if s > 1] if n_tiles < 148 else [])
        chunks = [0] if fam == "ffma" else ([32, 64] if parts == 3 else [64, 128, 256])
        rasters = [8, 16] if n_tiles >= 148 else [8]
        for s, c, r in itertools.product(splits, chunks, rasters):
            out.append({"tile": tile, "split_k": s, "chunk_k": c, "raster_group": r})
    return out


def _time(fn, steps: int) -> float:
    import torch
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def tune(m: int, n: int, k: int, variant: str = "bf16x6", steps: int = 5,
         max_candidates: int = 24, store: bool = True) -> dict:
    """Measure candidate schedules for an m x n x k product and cache the best.

    FFMA candidates that slice K change the summation order; they are only
    considered when the output has too few tiles to fill the GPU."""
    import torch

    from .sgemm import gemm, gemm_workspace_size, tiles
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.rand((m, k), device="cuda", generator=g) * 2 - 1
    B = torch.rand((k, n), device="cuda", generator=g) * 2 - 1
    C = torch.empty((m, n), device="cuda")
    table = []
    cands = candidates(m, n, k, variant, tiles())[:max_candidates]
    for cfg in cands:
        ws = torch.empty(max(gemm_workspace_size(m, n, k, variant, cfg), 256),
                         dtype=torch.uint8, device="cuda")
        try:
            ms = _time(lambda: gemm(A, B, C, variant=variant, config=cfg, workspace=ws), steps)
        except Exception as e:  # a schedule the library rejects for this shape
            table.append({"config": cfg, "error": str(e)})
            continue
        table.append({"config": cfg, "ms": ms, "tflops": 2.0 * m * n * k / (ms * 1e-3) / 1e12})
    ok = [t for t in table if "ms" in t]
    if not ok:
        raise RuntimeError("no candidate schedule ran")
    best = min(ok, key=lambda t: t["ms"])
    entry = {"config": best["config"], "ms": best["ms"], "shape": [m, n, k],
             "candidates": table}
    global _last_entry
    _last_entry = entry
    if store:
        _store(shape_key(m, n, k, variant), entry)
    return dict(best["config"])


def tune_grouped(As, Bs, variant: str = "bf16x6", steps: int = 3, store: bool = True) -> dict:
    """Measure grouped-plan schedules (tile shape, rasterisation) on the given
    problems and cache the best for their class."""
    from .sgemm import GroupedPlan, tiles
    fam = "ffma" if variant == "ffma" else "bf16"
    parts = 0 if fam == "ffma" else (3 if "x6" in variant else 2)
    # grouped plans run every tile family except the A-in-TMEM fused tiles
    # (fused tiles 128 rows high)
    ids = [t["tile"] for t in tiles() if t["family"] == fam and t["parts"] == parts
           and not (t["fused"] and t["bm"] == 128)]
    table = []
    for tile, raster in itertools.product(ids, (8, 16)):
        cfg = {"tile": tile, "raster_group": raster}
        try:
            plan = GroupedPlan(As, Bs, variant=variant, config=cfg)
            ms = _time(plan.run, steps)
            plan.close()
        except Exception as e:
            table.append({"config": cfg, "error": str(e)})
            continue
        table.append({"config": cfg, "ms": ms})
    ok = [t for t in table if "ms" in t]
    if not ok:
        raise RuntimeError("no candidate schedule ran")
    best = min(ok, key=lambda t: t["ms"])
    dims = [(a.shape[0], b.shape[1], a.shape[1]) for a, b in zip(As, Bs)]
    entry = {"config": best["config"], "ms": best["ms"], "problems": len(dims),
             "candidates": table}
    global _last_entry
    _last_entry = entry
    if store:
        _store(grouped_key(dims, variant), entry)
    return dict(best["config"])


# Shape classes the shipped table covers: the benchmark's named
# configurations (square sweep, the 8192^3 precision forms, the awkward
# shapes, the uneven 512-problem batch).
SHIP_SHAPES = [
    ((1024, 1024, 1024), ("ffma", "bf16x6", "bf16x3")),
    ((2048, 2048, 2048), ("ffma", "bf16x6", "bf16x3")),
    ((4096, 4096, 4096), ("ffma", "bf16x6", "bf16x3")),
    ((8192, 8192, 8192), ("ffma", "bf16x6", "bf16x3", "bf16x6_scaled", "bf16x3_scaled")),
    ((256, 256, 1 << 20), ("ffma", "bf16x6", "bf16x3")),
    ((65536, 64, 4096), ("ffma", "bf16x6", "bf16x3")),
]
SHIP_GROUPED = [(512, 0, ("ffma", "bf16x6", "bf16x3"))]


def ship(path: str = SHIPPED_PATH, steps: int = 3) -> dict:
    """Tune every shipped shape class on the current GPU and write the table
    (with each candidate's measured time as evidence) to `path`."""
    import torch

    from . import sweep
    out = {}
    for (m, n, k), variants in SHIP_SHAPES:
        for v in variants:
            cfg = tune(m, n, k, v, steps=steps, max_candidates=64, store=False)
            out[shape_key(m, n, k, v)] = _last_entry
            print(json.dumps({"shape": [m, n, k], "variant": v, "config": cfg,
                              "ms": _last_entry["ms"]}), flush=True)
            torch.cuda.empty_cache()
    for count, seed, variants in SHIP_GROUPED:
        dims = sweep.grouped_dims(count, seed)
        shapes = [(int(a), int(b), int(c)) for a, b, c in dims]
        As, Bs = sweep._inputs(shapes, "uniform", seed, "cuda")
        for v in variants:
            cfg = tune_grouped(As, Bs, v, steps=steps, store=False)
            out[grouped_key(shapes, v)] = _last_entry
            print(json.dumps({"grouped": count, "variant": v, "config": cfg,
                              "ms": _last_entry["ms"]}), flush=True)
        del As, Bs
        torch.cuda.empty_cache()
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    return out


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="autotuner")
    ap.add_argument("--ship", action="store_true", help="tune the shipped shape classes")
    ap.add_argument("--out", default=SHIPPED_PATH)
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args()
    if a.ship:
        ship(a.out, a.steps)
