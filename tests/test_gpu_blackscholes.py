"""Black-Scholes pricing (the suite's apps/blackscholes benchmark) on the GPU
through the C ABI, bit for bit against the oracle's restatement of the device
kernel's arithmetic (oracle.bs_device, bs_kernel.hpp:163-198), and inside the
testbench's own check against the host reference (sum of squared call and put
differences <= 0.01, apps/blackscholes/main.cpp:119-141). The reference's
registered launch is num-option_32768 (apps/blackscholes/tests.mk:1); its
input file holds 10 M options (in_10M.txt), the size of the large case."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sha(x):
    return hashlib.sha256(np.ascontiguousarray(x, np.float32).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def bs():
    from hb_hammerbench_b200 import blackscholes
    return blackscholes


def _price(bs, rec):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(rec, np.float32)).cuda()
    bs.price(d)
    return d.cpu().numpy()


def test_reference_launch_32768(bs, oracle_mod, golden_dir):
    with open(os.path.join(golden_dir, "blackscholes_32768.json")) as f:
        fx = json.load(f)
    rec = bs.option_records(fx["num_option"], fx["seed"])
    assert _sha(rec) == fx["sha256_inputs_f32"]
    out = _price(bs, rec)
    assert _sha(out[:, 5:7]) == fx["sha256_device_call_put_f32"]
    host = oracle_mod.bs_host(rec)
    assert _sha(host[:, 5:7]) == fx["sha256_host_call_put_f32"]
    assert oracle_mod.bs_validation_error(out, host) <= 0.01


@pytest.mark.parametrize("n", [1, 2, 3, 5, 255, 257, 1000, 32768 + 7, 148 * 256 * 16 + 3])
def test_ragged_counts_exact(bs, oracle_mod, n):
    rec = bs.option_records(n, seed=n)
    out = _price(bs, rec)
    exp = oracle_mod.bs_device(rec)
    assert np.array_equal(out.view(np.uint32), exp.view(np.uint32))


def test_unaligned_records_exact(bs, oracle_mod):
    """Records starting 4 bytes into a buffer take the scalar path."""
    import torch
    n = 4099
    rec = bs.option_records(n, seed=17)
    buf = torch.zeros(n * 8 + 1, dtype=torch.float32, device="cuda")
    view = buf[1:].view(n, 8)
    assert view.data_ptr() % 16 == 4
    view.copy_(torch.from_numpy(rec))
    bs.price(view)
    out = view.cpu().numpy()
    assert np.array_equal(out.view(np.uint32), oracle_mod.bs_device(rec).view(np.uint32))
    assert float(buf[0]) == 0.0


@pytest.mark.parametrize("n,offset", [(4096, 0), (4099, 0), (4099, 1), (3, 0)])
def test_arrays_match_records(bs, oracle_mod, n, offset):
    import torch
    rec = bs.option_records(n, seed=n + offset)
    exp = oracle_mod.bs_device(rec)
    cols = []
    for j in range(5):
        b = torch.empty(n + offset, dtype=torch.float32, device="cuda")
        b[offset:].copy_(torch.from_numpy(np.ascontiguousarray(rec[:, j])))
        cols.append(b[offset:])
    call, put = bs.price_arrays(*cols)
    assert np.array_equal(call.cpu().numpy().view(np.uint32), exp[:, 5].view(np.uint32))
    assert np.array_equal(put.cpu().numpy().view(np.uint32), exp[:, 6].view(np.uint32))


def test_edges_exact(bs, oracle_mod):
    rec = np.zeros((8, 8), np.float32)
    rec[:, :5] = [[50, 50, 0.05, 0.3, 0.5], [100, 100, 0.0275, 0.05, 0.05],
                  [100, 40, 0.1, 0.05, 0.05], [40, 100, 0.1, 0.05, 0.05],
                  [60, 65, 0.08, 0.65, 1.0], [42, 40, 0.1, 0.2, 0.5],
                  [100, 90, 0.1, 0.1, 0.1], [60.75, 60.75, 0.0725, 0.45, 0.15]]
    rec[:, 7] = np.arange(8, dtype=np.float32) + 0.5  # the unused field is kept
    out = _price(bs, rec)
    exp = oracle_mod.bs_device(rec)
    assert np.array_equal(out.view(np.uint32), exp.view(np.uint32))
    assert np.array_equal(out[:, 7], rec[:, 7])


def test_dataset_size_exact(bs, oracle_mod):
    """10 M options, the size of the benchmark's input file, every record
    against the oracle (records and arrays)."""
    import torch
    n = 10_000_000
    rec = bs.option_records(n, seed=10)
    exp = oracle_mod.bs_device(rec)
    d = torch.from_numpy(rec).cuda()
    cols = [d[:, j].contiguous() for j in range(5)]
    bs.price(d)
    out = d.cpu().numpy()
    assert np.array_equal(out.view(np.uint32), exp.view(np.uint32))
    call, put = bs.price_arrays(*cols)
    assert np.array_equal(call.cpu().numpy().view(np.uint32), exp[:, 5].view(np.uint32))
    assert np.array_equal(put.cpu().numpy().view(np.uint32), exp[:, 6].view(np.uint32))


def test_errors(bs):
    import torch
    from hb_hammerbench_b200 import HbsgError, lib
    ok = torch.zeros(16, 8, device="cuda")
    bs.price(ok[:0])  # zero options: no launch, success
    with pytest.raises(ValueError):
        bs.price(torch.zeros(16, 7, device="cuda"))
    x = torch.zeros(64, device="cuda")
    with pytest.raises(HbsgError):
        bs.price_arrays(x, x, x, x, x, call=x, put=torch.zeros(64, device="cuda"))
    assert lib().hbsg_blackscholes(None, 4, None) < 0


@pytest.mark.parametrize("case", ["num-option_32768", "num-option_10000000",
                                  "num-option_10000000__LAYOUT_arrays"])
def test_sweep_named_case(case):
    from hb_hammerbench_b200 import sweep
    r = sweep.run_case(case, steps=2, warmup=1)
    assert r["options"] == sweep.parse_case(case)["NUM-OPTION"]
    assert r["changed_after_repeat"] == 0 and r["moptions_per_s"] > 0
