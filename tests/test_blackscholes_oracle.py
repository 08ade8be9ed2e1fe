"""The Black-Scholes oracle on the CPU: the host reference restatement is
pinned bit for bit to the reference's own BlkSchlsEqEuroNoDiv (bs.hpp)
compiled from the reference tree, and to the committed fixture; the
restatement of the device kernel's arithmetic (bs_kernel.hpp) matches the
fixture and stays inside the testbench's own bound (main.cpp:119-141)
against the host reference."""
import hashlib
import json
import os

import numpy as np
import pytest


def _sha(x):
    return hashlib.sha256(np.ascontiguousarray(x, np.float32).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def fixture(golden_dir):
    with open(os.path.join(golden_dir, "blackscholes_32768.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def records(fixture):
    from hb_hammerbench_b200.blackscholes import option_records
    rec = option_records(fixture["num_option"], fixture["seed"])
    assert _sha(rec) == fixture["sha256_inputs_f32"], "synthetic generator changed"
    return rec


def test_host_restatement_matches_fixture(oracle_mod, fixture, records):
    host = oracle_mod.bs_host(records)
    assert _sha(host[:, 5:7]) == fixture["sha256_host_call_put_f32"]
    for i, c, p, _, _ in fixture["samples"]:
        assert host[i, 5] == np.float32(c) and host[i, 6] == np.float32(p)


def test_host_restatement_matches_reference_build(oracle_mod, records):
    if not oracle_mod.ref_bs_available():
        pytest.skip("reference Black-Scholes host library not built here")
    rng = np.random.Generator(np.random.PCG64(5))
    wide = records.copy()
    wide[:, 0] *= rng.uniform(0.2, 5.0, len(wide)).astype(np.float32)  # ratios far from 1
    for rec in (records, wide):
        assert np.array_equal(oracle_mod.ref_bs_host(rec), oracle_mod.bs_host(rec))


def test_device_restatement_matches_fixture(oracle_mod, fixture, records):
    dev = oracle_mod.bs_device(records)
    assert _sha(dev[:, 5:7]) == fixture["sha256_device_call_put_f32"]
    host = oracle_mod.bs_host(records)
    err = oracle_mod.bs_validation_error(dev, host)
    assert err == pytest.approx(fixture["validation_error_device_vs_host"], rel=0, abs=0)
    assert err <= 0.01


def test_device_restatement_writes_call_put_only(oracle_mod, records):
    dev = oracle_mod.bs_device(records)
    keep = [0, 1, 2, 3, 4, 7]
    assert np.array_equal(dev[:, keep].view(np.uint32), records[:, keep].view(np.uint32))


def test_device_restatement_edges(oracle_mod):
    # at the money (ln term exactly 0), deep in / out of the money (the
    # cumulative normal's exp below -15 returns 0), short and long maturities
    rec = np.zeros((6, 8), np.float32)
    rec[:, :5] = [[50, 50, 0.05, 0.3, 0.5], [100, 100, 0.0275, 0.05, 0.05],
                  [100, 40, 0.1, 0.05, 0.05], [40, 100, 0.1, 0.05, 0.05],
                  [60, 65, 0.08, 0.65, 1.0], [42, 40, 0.1, 0.2, 0.5]]
    dev = oracle_mod.bs_device(rec)
    host = oracle_mod.bs_host(rec)
    assert np.all(np.isfinite(dev[:, 5:7]))
    # deep in the money: call = s - strike * exp(-rt) to the kernel's exp
    # series accuracy, put = 0
    assert dev[2, 6] == 0.0 and host[2, 6] == pytest.approx(0.0, abs=1e-6)
    assert dev[3, 5] == 0.0
    # at-the-money records agree with the host within the testbench scale
    assert np.max(np.abs(dev[[0, 1, 4, 5], 5:7] - host[[0, 1, 4, 5], 5:7])) < 1e-3
