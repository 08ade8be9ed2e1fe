"""The CPU oracle checked against the reference's own golden vectors.

The golden fixtures were produced by the reference testbench's host_mm
(apps/sgemm/main.cpp:15-26) compiled from the reference source
(tests/golden/make_golden.py). When that compiled reference is present
(oracle/_ref), it is also compared with the oracle directly.
"""
import hashlib
import json
import os

import numpy as np
import pytest


def _sha(x):
    return hashlib.sha256(np.ascontiguousarray(x, np.float32).tobytes()).hexdigest()


def test_mod_fixture_matches_golden(oracle_mod, golden_dir):
    fix = json.load(open(os.path.join(golden_dir, "sgemm_mod_N512_NITER2.json")))
    n, niter = fix["N"], fix["NITER"]
    m1, m2 = oracle_mod.fill_mod(niter * n * n)
    out = oracle_mod.host_mm_batched(m1, m2, n, niter)
    assert _sha(out) == fix["sha256_result_f32"]
    assert out[0] == fix["first"] and out[-1] == fix["last"]
    for i, v in fix["samples"]:
        assert out[i] == v


def test_mod_fixture_device_arithmetic_is_exact(oracle_mod, golden_dir):
    # Small integers: the fused chain and the two-rounding chain agree exactly.
    fix = json.load(open(os.path.join(golden_dir, "sgemm_mod_N512_NITER2.json")))
    n = fix["N"]
    m1, m2 = oracle_mod.fill_mod(n * n)
    a = m1.reshape(n, n)
    b = m2.reshape(n, n)
    assert np.array_equal(oracle_mod.host_mm_fma(a, b), oracle_mod.host_mm(a, b))


@pytest.mark.parametrize("name", ["sgemm_uniform_N64_NITER2.npz", "sgemm_uniform_N128_NITER1.npz"])
def test_uniform_golden_bit_exact(oracle_mod, golden_dir, name):
    z = np.load(os.path.join(golden_dir, name))
    A, B, C = z["A"], z["B"], z["C_ref"]
    for i in range(A.shape[0]):
        assert np.array_equal(oracle_mod.host_mm(A[i], B[i]), C[i])


def test_uniform_golden_inputs_reproducible(oracle_mod, golden_dir):
    z = np.load(os.path.join(golden_dir, "sgemm_uniform_N64_NITER2.npz"))
    A, B = oracle_mod.uniform_inputs(z["A"].shape, z["B"].shape, int(z["seed"]))
    assert np.array_equal(A, z["A"]) and np.array_equal(B, z["B"])


def test_ramp_identity_golden(oracle_mod, golden_dir):
    fix = json.load(open(os.path.join(golden_dir, "sgemm_ramp_identity_N512.json")))
    a, b = oracle_mod.fill_ramp_identity(fix["N"])
    out = oracle_mod.host_mm(a, b)
    assert np.array_equal(out, a)
    assert _sha(out) == fix["sha256_result_f32"]


def test_identity_ramp_legacy(oracle_mod):
    a, b = oracle_mod.fill_identity_ramp(64, 96, 80)
    out = oracle_mod.host_mm(a, b)
    assert np.array_equal(out, b[:64])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), "oracle", "_ref", "libref_host_mm.so")),
    reason="compiled reference host_mm not present")
@pytest.mark.parametrize("n", [64, 128, 512])
def test_oracle_equals_compiled_reference(oracle_mod, n):
    A, B = oracle_mod.uniform_inputs((n, n), (n, n), seed=1000 + n)
    for opt in ("O3", "O0"):
        assert np.array_equal(oracle_mod.ref_host_mm(A, B, n, opt), oracle_mod.host_mm(A, B))


def test_row_range_is_exact_subcomputation(oracle_mod):
    A, B = oracle_mod.uniform_inputs((96, 40), (40, 72), seed=3)
    full = oracle_mod.host_mm(A, B)
    part = oracle_mod.host_mm(A, B, rows=(17, 61))
    mt = oracle_mod.host_mm(A, B, rows=(17, 61), threads=4)
    assert np.array_equal(part, full[17:61]) and np.array_equal(mt, part)


def test_fma_and_two_rounding_differ_but_close(oracle_mod):
    A, B = oracle_mod.uniform_inputs((64, 256), (256, 64), seed=5)
    c1 = oracle_mod.host_mm(A, B)
    c2 = oracle_mod.host_mm_fma(A, B)
    ref = oracle_mod.gemm_f64(A, B)
    assert not np.array_equal(c1, c2)
    for c in (c1, c2):
        e = oracle_mod.error_vs_f64(c, ref)
        assert e["rel_fro"] < 1e-6


def test_f64_product_exact_on_integers(oracle_mod):
    m1, m2 = oracle_mod.fill_mod(128 * 128)
    a = m1.reshape(128, 128)
    b = m2.reshape(128, 128)
    ref = oracle_mod.gemm_f64(a, b)
    assert np.array_equal(ref, a.astype(np.float64) @ b.astype(np.float64))


@pytest.mark.parametrize("parts", [2, 3])
def test_split_bf16_properties(oracle_mod, parts):
    rng = np.random.Generator(np.random.PCG64(11))
    x = (rng.uniform(-1, 1, 4096) * np.exp2(rng.uniform(-20, 20, 4096))).astype(np.float32)
    e = oracle_mod.pow2_exponent(x)
    hi, mid, lo = oracle_mod.split_bf16(x, e, parts)
    h = oracle_mod.bf16_to_f32(hi).astype(np.float64)
    m = oracle_mod.bf16_to_f32(mid).astype(np.float64)
    xs = np.ldexp(x.astype(np.float64), -e)
    if parts == 3:
        l = oracle_mod.bf16_to_f32(lo).astype(np.float64)
        assert np.array_equal(h + m + l, xs)  # three parts hold FP32 exactly
    else:
        rel = np.abs(h + m - xs) / np.maximum(np.abs(xs), 1e-300)
        assert rel.max() <= 2.0 ** -16
    assert np.all(np.abs(m) <= np.abs(h) * 2.0 ** -8 + 1e-300)


def test_bf16_rounding_ties_to_even(oracle_mod):
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 in BF16: rounds to even (1.0).
    x = np.array([1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -(1.0 + 2.0 ** -8)], np.float32)
    hi, _, _ = oracle_mod.split_bf16(x, 0, 3)
    assert list(oracle_mod.bf16_to_f32(hi)) == [1.0, 1.0 + 2.0 ** -6, -1.0]


@pytest.mark.parametrize("nx,ny,nz", [(64, 8, 512), (32, 8, 512), (5, 3, 7)])
def test_host_jacobi_matches_reference(oracle_mod, nx, ny, nz):
    # the restatement against the reference's own host_jacobi, compiled from
    # apps/jacobi/main.cpp: the i % 13 fixture and random floats, bit for bit
    if not oracle_mod.ref_jacobi_available():
        pytest.skip("reference host_jacobi library not built (no reference tree)")
    a = oracle_mod.fill_jacobi(nx * ny * nz)
    assert np.array_equal(oracle_mod.ref_host_jacobi(a, nx, ny, nz),
                          oracle_mod.host_jacobi(a, nx, ny, nz))
    rng = np.random.Generator(np.random.PCG64(nz))
    r = rng.uniform(-1, 1, nx * ny * nz).astype(np.float32)
    assert np.array_equal(oracle_mod.ref_host_jacobi(r, nx, ny, nz, 3, -5),
                          oracle_mod.host_jacobi(r, nx, ny, nz, 3, -5))


def test_jacobi_fixture_golden(oracle_mod, golden_dir):
    # tests/golden/jacobi_mod_64x8x512.json: SHA-256 of host_jacobi's output on
    # the reference launch nx_64__ny_8__nz_512 (made by make_golden.py from
    # the reference's own host_jacobi)
    import hashlib
    import json
    import os
    fix = json.load(open(os.path.join(golden_dir, "jacobi_mod_64x8x512.json")))
    nx, ny, nz = fix["nx"], fix["ny"], fix["nz"]
    out = oracle_mod.host_jacobi(oracle_mod.fill_jacobi(nx * ny * nz), nx, ny, nz,
                                 fix["c0"], fix["c1"])
    assert hashlib.sha256(out.tobytes()).hexdigest() == fix["sha256_anext_f32"]
