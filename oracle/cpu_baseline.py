"""CPU baseline table for the SGEMM hot path (measurement infrastructure; the
product never imports this).

Times the reference's CPU path on the host it runs on, as one JSON line per
measurement:
  1. the reference's own host_mm (apps/sgemm/main.cpp:15-26), compiled from
     its source at -O3 and at -O0 (oracle/_ref, one object per N, because N
     is a compile-time macro there), single core, in full at N = 512, 1024,
     2048, checked bit-exact against the oracle's restatement;
  2. the restatement (oracle_host_mm_rows, the same loop) on a 64-row sample
     at N = 4096 and 8192, single core, extrapolated by N / rows (the work is
     linear in rows);
  3. the restatement over all host cores (OpenMP over rows) on a row sample
     at N = 8192, extrapolated the same way.
Inputs: seeded U[-1, 1) (oracle.uniform_inputs).

    python -m oracle.cpu_baseline            # the whole table (a few minutes)
    python -m oracle.cpu_baseline --quick    # N = 512 only, for a dry run
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from oracle import oracle


def _line(**kw):
    print(json.dumps(kw), flush=True)


def reference_full(n: int, opt: str) -> None:
    A, B = oracle.uniform_inputs((n, n), (n, n), seed=n)
    t0 = time.perf_counter()
    out = oracle.ref_host_mm(A, B, n, opt)
    dt = time.perf_counter() - t0
    same = bool(np.array_equal(out, oracle.host_mm(A, B)))
    _line(kind="reference", build=opt, n=n, rows=n, cores=1, seconds=round(dt, 3),
          gflops=round(2.0 * n ** 3 / dt / 1e9, 3), extrapolated=False,
          bit_exact_with_restatement=same)


def port_sample(n: int, rows: int, threads: int) -> None:
    A, B = oracle.uniform_inputs((rows, n), (n, n), seed=n)
    t0 = time.perf_counter()
    oracle.host_mm(A, B, threads=threads)
    dt = time.perf_counter() - t0
    _line(kind="port", build="O3", n=n, rows=rows, cores=threads, seconds=round(dt, 3),
          gflops=round(2.0 * rows * n * n / dt / 1e9, 3), extrapolated=True,
          full_product_seconds=round(dt * n / rows, 1))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    args = ap.parse_args()
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    ns = (512,) if args.quick else (512, 1024, 2048)
    for n in ns:
        for opt in ("O3", "O0"):
            reference_full(n, opt)
    if args.quick:
        return
    for n in (4096, 8192):
        port_sample(n, 64, 1)
    cores = len(os.sched_getaffinity(0))
    port_sample(8192, 8 * cores, cores)


if __name__ == "__main__":
    main()
