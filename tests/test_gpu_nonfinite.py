"""Non-finite and extreme inputs through the C ABI.

The reference computes in IEEE FP32 (host_mm, apps/sgemm/main.cpp:15-26), so
an output is non-finite exactly when its row of A or its column of B holds a
NaN or an infinity (Inf * b = +-Inf, Inf * 0 = NaN, Inf + -Inf = NaN), and
every other output is the ordinary finite product. Bars:
  - FFMA: bit-exact against the oracle's fmaf chain, the positions and signs
    of NaN and Inf included (NaN payloads are not compared);
  - split-BF16, every form: the oracle's non-finite mask exactly, and the
    finite outputs within the form's error bound. An infinite element splits
    into Inf + NaN + NaN (its residual is Inf - Inf), so outputs that the FP32
    reference gives as +-Inf may come out NaN: both are non-finite, and no
    other output is touched;
  - grouped plans: a problem with non-finite inputs leaves the others exact;
  - range: the scaled forms cover the whole FP32 range (values up to 3.4e38
    with products that stay finite); the unscaled forms hold values up to
    bf16's largest finite, 3.39e38, beyond which the high part rounds to Inf.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPLIT = ["bf16x3", "bf16x6", "bf16x3_scaled", "bf16x6_scaled"]
BOUND = {"bf16x3": 2e-5, "bf16x6": 1e-6, "bf16x3_scaled": 2e-5, "bf16x6_scaled": 1e-6}


@pytest.fixture(scope="module")
def hb():
    import hb_hammerbench_b200 as hb
    return hb


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()


def _poisoned(m, n, k, seed):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    B = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    A[3, 10] = np.nan
    A[17, 50] = np.inf
    A[40, 0] = -np.inf
    A[60, :] = np.inf           # a row with no finite value (row maximum 0)
    B[50, 7] = 0.0              # Inf * 0 = NaN in row 17, column 7
    B[5, 9] = np.inf
    B[k - 1, n - 1] = np.nan
    B[0, 100] = -np.inf
    bad_rows = [3, 17, 40, 60]
    bad_cols = [9, n - 1, 100]
    return A, B, bad_rows, bad_cols


def _expected_mask(m, n, bad_rows, bad_cols):
    mask = np.zeros((m, n), bool)
    mask[bad_rows, :] = True
    mask[:, bad_cols] = True
    return mask


def test_ffma_nonfinite_bit_exact(hb, oracle_mod):
    m, n, k = 130, 200, 96
    A, B, rows, cols = _poisoned(m, n, k, 1)
    out = hb.gemm(_dev(A), _dev(B), variant="ffma").cpu().numpy()
    ref = oracle_mod.host_mm_fma(A, B)
    assert np.array_equal(~np.isfinite(ref), _expected_mask(m, n, rows, cols))
    assert np.array_equal(out, ref, equal_nan=True)
    assert np.array_equal(np.isnan(out), np.isnan(ref))


@pytest.mark.parametrize("variant", SPLIT)
def test_split_nonfinite_mask_and_finite_accuracy(hb, oracle_mod, variant):
    m, n, k = 130, 200, 96
    A, B, rows, cols = _poisoned(m, n, k, 2)
    out = hb.gemm(_dev(A), _dev(B), variant=variant).cpu().numpy()
    mask = _expected_mask(m, n, rows, cols)
    assert np.array_equal(~np.isfinite(out), mask)
    ok_r = np.setdiff1d(np.arange(m), rows)
    ok_c = np.setdiff1d(np.arange(n), cols)
    ref = oracle_mod.gemm_f64(A[ok_r], B[:, ok_c])
    got = out[np.ix_(ok_r, ok_c)].astype(np.float64)
    rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert rel < BOUND[variant], rel


@pytest.mark.parametrize("variant", ["ffma", "bf16x6"])
def test_grouped_nonfinite_stays_in_its_problem(hb, variant):
    import torch
    m, n, k = 130, 200, 96
    A0, B0, rows, cols = _poisoned(m, n, k, 3)
    rng = np.random.default_rng(4)
    A1 = rng.uniform(-1, 1, (96, 64)).astype(np.float32)
    B1 = rng.uniform(-1, 1, (64, 160)).astype(np.float32)
    As, Bs = [_dev(A0), _dev(A1)], [_dev(B0), _dev(B1)]
    Cs = hb.gemm_grouped(As, Bs, variant=variant, config={"split_k": 1})
    torch.cuda.synchronize()
    assert np.array_equal(~np.isfinite(Cs[0].cpu().numpy()), _expected_mask(m, n, rows, cols))
    alone = hb.gemm(As[1], Bs[1], variant=variant, config={"split_k": 1})
    assert torch.equal(Cs[1], alone)


@pytest.mark.parametrize("variant", ["bf16x3_scaled", "bf16x6_scaled"])
def test_scaled_forms_cover_full_fp32_range(hb, oracle_mod, variant):
    rng = np.random.default_rng(5)
    m, n, k = 64, 96, 128
    A = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    B = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    A[:8] *= np.float32(3.4e38)   # beyond bf16's largest finite (3.39e38)
    B *= np.float32(1e-30)        # products stay near 3.4e8
    out = hb.gemm(_dev(A), _dev(B), variant=variant).cpu().numpy()
    assert np.isfinite(out).all()
    ref = oracle_mod.gemm_f64(A, B)
    rel = np.linalg.norm(out.astype(np.float64) - ref) / np.linalg.norm(ref)
    assert rel < BOUND[variant], rel


@pytest.mark.parametrize("variant", ["bf16x3", "bf16x6"])
def test_unscaled_forms_hold_up_to_bf16_max(hb, oracle_mod, variant):
    rng = np.random.default_rng(6)
    m, n, k = 64, 96, 128
    A = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    B = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    A[:8] *= np.float32(3.38e38)  # below bf16's largest finite
    B *= np.float32(1e-30)
    out = hb.gemm(_dev(A), _dev(B), variant=variant).cpu().numpy()
    assert np.isfinite(out).all()
    ref = oracle_mod.gemm_f64(A, B)
    rel = np.linalg.norm(out.astype(np.float64) - ref) / np.linalg.norm(ref)
    assert rel < BOUND[variant], rel
