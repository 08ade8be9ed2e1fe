"""Concurrent host threads, one CUDA stream each, calling the C ABI.

The library keeps only immutable or atomically published state (device
properties under a mutex, the tensor-map encoder and tuning knobs resolved by
thread-safe one-time initialisation, per-kernel shared-memory attributes set
through atomic masks), so calls from several host threads on distinct streams
need no external lock. The check runs in a fresh process so that the threads'
first calls, which perform that one-time set-up, overlap; each thread's
results must equal the same products computed afterwards on one thread.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import threading, torch
import hb_hammerbench_b200 as hb
torch.cuda.init()
shapes = [(384, 256, 512), (256, 640, 1024), (512, 512, 256), (128, 384, 2048)]
variants = ["bf16x6", "ffma", "bf16x3_scaled", "bf16x6"]
inputs = []
for i, (m, n, k) in enumerate(shapes):
    g = torch.Generator(device="cuda").manual_seed(100 + i)
    inputs.append((torch.rand((m, k), device="cuda", generator=g) * 2 - 1,
                   torch.rand((k, n), device="cuda", generator=g) * 2 - 1))
torch.cuda.synchronize()
barrier = threading.Barrier(len(shapes))
out = [None] * len(shapes)
errors = []
def work(i):
    try:
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            barrier.wait()
            C = [hb.gemm(*inputs[i], variant=variants[i]) for _ in range(3)]
        s.synchronize()
        out[i] = C
    except Exception as e:
        errors.append(repr(e))
ts = [threading.Thread(target=work, args=(i,)) for i in range(len(shapes))]
for t in ts: t.start()
for t in ts: t.join()
assert not errors, errors
for i in range(len(shapes)):
    ref = hb.gemm(*inputs[i], variant=variants[i])
    torch.cuda.synchronize()
    for C in out[i]:
        assert torch.equal(C, ref), i
print("threads ok")
"""


def test_concurrent_first_calls_from_threads():
    env = dict(os.environ)
    env["PYTHONPATH"] = ROOT + os.pathsep + env.get("PYTHONPATH", "")
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "threads ok" in r.stdout, r.stdout + r.stderr
