"""The benchmark's named configurations at their stated sizes, on the GPU.

One test per named launch, each checked against the host oracle or the FP64
product, in the way the reference registers one launch per named config with
a host-oracle check (apps/sgemm/tests.mk:1, apps/sgemm/main.cpp:119-134):

  3(b)  M = N = K = 8192, wide-range inputs sign * 2^u, u ~ U[-20, 20]
  4     512 problems, M, N, K uniform over the multiples of 32 in [64, 2048],
        one grouped plan (CUDA-graph replay)
  5(i)  M = N = 256, K = 1,048,576 (error against K over prefixes 2^10 .. 2^20)
  5(ii) M = 65536, N = 64, K = 4096

plus a check of the FP64 yardstick itself at 8192^3: the GPU float64 product
every split-BF16 test compares with equals the oracle's FP64 product (oracle.c,
sequential double accumulation) on sampled rows.

Bars: the 6-product forms are no worse than the FFMA kernel against FP64 (the
precision form's error bar); the 3-product forms stay within 2^-16 relative
Frobenius error (their 2-part split holds ~16 bits).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

X3_BOUND = 2.0 ** -16


@pytest.fixture(scope="module")
def hb():
    import hb_hammerbench_b200 as hb
    return hb


def _err(C, ref):
    import torch
    d = C.double() - ref
    return float(torch.linalg.norm(d) / torch.linalg.norm(ref)), float(d.abs().max())


def _uniform(shape, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.rand(shape, device="cuda", generator=g) * 2 - 1


def _wide(shape, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    s = torch.rand(shape, device="cuda", generator=g) * 2 - 1
    u = torch.rand(shape, device="cuda", generator=g) * 40 - 20
    return torch.sign(s) * torch.exp2(u)


# --------------------------------------------------------------------------
# 3(b) and the FP64 yardstick at 8192^3

@pytest.fixture(scope="module")
def wide8192():
    import torch
    n = 8192
    A = _wide((n, n), 3001)
    B = _wide((n, n), 3002)
    ref = A.double() @ B.double()
    yield A, B, ref
    del A, B, ref
    torch.cuda.empty_cache()


def test_fp64_reference_pinned_to_oracle_at_8192(wide8192, oracle_mod):
    # rows of a product are independent: 8 sampled rows through the oracle's
    # FP64 product must agree with the GPU float64 product to FP64 rounding
    A, B, ref = wide8192
    rows = np.random.Generator(np.random.PCG64(5)).choice(A.shape[0], 8, replace=False)
    a = A[rows].cpu().numpy()
    b = B.cpu().numpy()
    want = oracle_mod.gemm_f64(a, b)
    got = ref[rows].cpu().numpy()
    scale = np.abs(a.astype(np.float64)) @ np.abs(b.astype(np.float64))
    assert np.all(np.abs(got - want) <= 1e-12 * scale + 1e-300)


def test_config3b_wide_range_8192(hb, wide8192):
    A, B, ref = wide8192
    e_ffma = _err(hb.gemm(A, B), ref)
    e6s = _err(hb.gemm(A, B, variant="bf16x6_scaled"), ref)
    e6 = _err(hb.gemm(A, B, variant="bf16x6"), ref)
    e3s = _err(hb.gemm(A, B, variant="bf16x3_scaled"), ref)
    assert e6s[0] <= e_ffma[0], (e6s, e_ffma)
    assert e6[0] <= e_ffma[0], (e6, e_ffma)
    assert e3s[0] <= X3_BOUND, e3s


def test_config3a_uniform_8192_headline(hb):
    import torch
    n = 8192
    A = _uniform((n, n), 3101)
    B = _uniform((n, n), 3102)
    ref = A.double() @ B.double()
    e_ffma = _err(hb.gemm(A, B), ref)
    for v in ("bf16x6", "bf16x6_scaled"):
        e = _err(hb.gemm(A, B, variant=v), ref)
        assert e[0] <= e_ffma[0] and e[1] <= e_ffma[1], (v, e, e_ffma)
    for v in ("bf16x3", "bf16x3_scaled"):
        assert _err(hb.gemm(A, B, variant=v), ref)[0] <= X3_BOUND
    del A, B, ref
    torch.cuda.empty_cache()


# --------------------------------------------------------------------------
# 4: the uneven batch

GROUPED_TILE = {"ffma": 1, "bf16x6": 10, "bf16x3": 13}


def _grouped_inputs(count=512, seed=0):
    """M, N, K uniform over the multiples of 32 in [64, 2048] (numpy PCG64),
    inputs U[-1, 1) in one device buffer (the sweep driver's generator)."""
    from hb_hammerbench_b200 import sweep
    dims = sweep.grouped_dims(count, seed)
    shapes = [(int(m), int(n), int(k)) for m, n, k in dims]
    As, Bs = sweep._inputs(shapes, "uniform", seed, "cuda")
    return shapes, As, Bs


@pytest.fixture(scope="module")
def batch512():
    import torch
    shapes, As, Bs = _grouped_inputs()
    assert len(shapes) == 512
    assert all(64 <= x <= 2048 and x % 32 == 0 for s in shapes for x in s)
    yield shapes, As, Bs
    del As, Bs
    torch.cuda.empty_cache()


@pytest.mark.parametrize("variant", ["ffma", "bf16x6", "bf16x3"])
def test_config4_grouped_512(hb, batch512, variant):
    import torch
    shapes, As, Bs = batch512
    plan = hb.GroupedPlan(As, Bs, variant=variant)
    Cs = plan.run()
    torch.cuda.synchronize()
    cfg = {"tile": GROUPED_TILE[variant], "split_k": 1}
    for i, (a, b, c) in enumerate(zip(As, Bs, Cs)):
        assert torch.equal(c, hb.gemm(a, b, variant=variant, config=cfg)), (i, shapes[i])
    # the FP64 bound on a sampled subset, summed over the subset's problems
    pick = np.random.Generator(np.random.PCG64(9)).choice(len(shapes), 32, replace=False)
    num = num_f = den = 0.0
    for i in pick:
        ref = As[i].double() @ Bs[i].double()
        num += float(((Cs[i].double() - ref) ** 2).sum())
        num_f += float(((hb.gemm(As[i], Bs[i]).double() - ref) ** 2).sum())
        den += float((ref ** 2).sum())
    rel, rel_f = (num / den) ** 0.5, (num_f / den) ** 0.5
    if variant == "bf16x6":
        assert rel <= rel_f, (rel, rel_f)
    elif variant == "bf16x3":
        assert rel <= X3_BOUND, rel
    plan.close()


# --------------------------------------------------------------------------
# 5: awkward shapes (automatic K slices)

@pytest.fixture(scope="module")
def tallk():
    import torch
    m, n, k = 256, 256, 1 << 20
    A = _uniform((m, k), 5001)
    B = _uniform((k, n), 5002)
    yield A, B
    del A, B
    torch.cuda.empty_cache()


def test_config5i_tall_k(hb, tallk):
    A, B = tallk
    ref = A.double() @ B.double()
    e_ffma = _err(hb.gemm(A, B), ref)
    e6 = _err(hb.gemm(A, B, variant="bf16x6"), ref)
    e3 = _err(hb.gemm(A, B, variant="bf16x3"), ref)
    assert e6[0] <= e_ffma[0] and e6[1] <= e_ffma[1], (e6, e_ffma)
    assert e3[0] <= X3_BOUND, e3


def test_config5i_error_flat_in_k(hb, tallk):
    # the 6-product form with automatic K slices keeps its error flat over
    # K = 2^10 .. 2^20, while one FFMA chain grows like sqrt(K)
    A, B = tallk
    e6, ef = [], []
    for p in range(10, 21, 2):
        k = 1 << p
        a, b = A[:, :k], B[:k]
        ref = a.double() @ b.double()
        e6.append(_err(hb.gemm(a, b, variant="bf16x6"), ref)[0])
        ef.append(_err(hb.gemm(a, b), ref)[0])
    assert max(e6) <= 2.0 * min(e6), e6
    assert ef[-1] >= 8.0 * ef[0], ef
    assert all(x <= y for x, y in zip(e6, ef)), (e6, ef)


def test_config5ii_tall_m(hb):
    import torch
    m, n, k = 65536, 64, 4096
    A = _uniform((m, k), 5101)
    B = _uniform((k, n), 5102)
    ref = A.double() @ B.double()
    e_ffma = _err(hb.gemm(A, B), ref)
    e6 = _err(hb.gemm(A, B, variant="bf16x6"), ref)
    e3 = _err(hb.gemm(A, B, variant="bf16x3"), ref)
    assert e6[0] <= e_ffma[0] and e6[1] <= e_ffma[1], (e6, e_ffma)
    assert e3[0] <= X3_BOUND, e3
    del A, B, ref
    torch.cuda.empty_cache()


# --------------------------------------------------------------------------
# named launches through the sweep driver (the launch-directory convention)

@pytest.mark.parametrize("case", ["N_512__NITER_2", "N_1024__NITER_1__V_bf16x6",
                                  "M_300__N_200__K_520__V_bf16x3_scaled__DIST_wide",
                                  "GROUPED_24__SEED_3__V_bf16x6"])
def test_sweep_named_case(case):
    from hb_hammerbench_b200 import sweep
    r = sweep.run_case(case, steps=2, warmup=1)
    assert r["tflops"] > 0
    bound = X3_BOUND if "x3" in r["variant"] else 2e-6
    assert r["error_vs_fp64"]["rel_fro"] < bound, r
