"""Fused-split tensor-core kernels (the FP32 -> BF16 split done inside the
product kernel, CTA pairs) on the GPU, through the C ABI.

The converter warps compute exactly the split pass's parts and write them in
the layout the TMA loads produced, and the MMA issue order and TMEM drains are
those of the unfused kernels, so a fused tile's result is bit-identical to the
unfused tile of the same product count and width (the CTA-pair tensor-core
kernel is itself bit-identical to the single-CTA one). Bars otherwise as in
test_gpu_bf16.py.
"""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hb():
    import hb_hammerbench_b200 as hb
    return hb


@pytest.fixture(scope="module")
def fused_ids(hb):
    """{(parts, bn): tile id} of the fused family, and of the unfused
    single-CTA family for comparison."""
    fused, plain = {}, {}
    for t in hb.tiles():
        if t["family"] != "bf16":
            continue
        if t["fused"] and t["bm"] == 256:  # CTA-pair tiles (the A-in-TMEM ones: test_gpu_fused_ts.py)
            fused[(t["parts"], t["bn"])] = t["tile"]
        elif t["bm"] == 128:
            plain[(t["parts"], t["bn"])] = t["tile"]
    assert set(fused) == {(3, 256), (2, 256), (3, 64), (2, 64)}
    return fused, plain


def _rand(shape, seed, wide=False):
    """Seeded operand whose row stride is a multiple of 4 floats (the fused
    kernels read operands through FP32 TMA maps: 16-byte aligned rows); a
    ragged column count is a view into a padded buffer."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    rows, cols = shape
    pad = (cols + 3) // 4 * 4
    x = torch.rand((rows, pad), device="cuda", generator=g) * 2 - 1
    if wide:
        u = torch.rand((rows, pad), device="cuda", generator=g) * 40 - 20
        x = torch.sign(x) * torch.exp2(u)
    return x[:, :cols]


def _err(C, ref):
    import torch
    d = C.double() - ref
    return float(torch.linalg.norm(d) / torch.linalg.norm(ref))


PARTS = {"bf16x6": 3, "bf16x3": 2, "bf16x6_scaled": 3, "bf16x3_scaled": 2}


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3", "bf16x6_scaled", "bf16x3_scaled"])
@pytest.mark.parametrize("bn", [256, 64])
@pytest.mark.parametrize("m,n,k", [(256, 256, 64), (300, 200, 100), (1000, 700, 1031),
                                   (64, 520, 7), (777, 64, 2048)])
def test_fused_matches_unfused(hb, fused_ids, variant, bn, m, n, k):
    import torch
    fused, plain = fused_ids
    P = PARTS[variant]
    wide = "scaled" in variant
    A = _rand((m, k), m + 3 * k, wide)
    B = _rand((k, n), n + 7 * k, wide)
    cfg = {"split_k": 1, "chunk_k": 64}
    Cf = hb.gemm(A, B, variant=variant, config={**cfg, "tile": fused[(P, bn)]})
    Cu = hb.gemm(A, B, variant=variant, config={**cfg, "tile": plain[(P, bn)]})
    assert torch.equal(Cf, Cu)


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3_scaled"])
def test_fused_needs_aligned_rows(hb, fused_ids, variant):
    # the fused kernels read A and B through FP32 TMA maps: a row stride that
    # is not a multiple of 4 floats is rejected for an explicit fused tile
    # (status -2) and served by the split-pass kernels otherwise
    import torch
    fused, plain = fused_ids
    P = PARTS[variant]
    m, n, k = 333, 290, 515
    buf = _rand((m, k + 3), 5)
    A = buf[:, 1:k + 1]
    B = _rand((k, n), 6)
    with pytest.raises(hb.HbsgError) as e:
        hb.gemm(A, B, variant=variant, config={"tile": fused[(P, 256)]})
    assert e.value.status == -2
    cfg = {"split_k": 1, "chunk_k": 64}
    C = hb.gemm(A, B, variant=variant, config=cfg)
    Aa = torch.zeros((m, (k + 3) // 4 * 4), device="cuda")[:, :k]  # aligned rows
    Aa.copy_(A)
    Cu = hb.gemm(Aa, B, variant=variant, config={**cfg, "tile": plain[(P, 256)]})
    Cf = hb.gemm(Aa, B, variant=variant, config={**cfg, "tile": fused[(P, 256)]})
    assert torch.equal(Cf, Cu)
    ref = A.double() @ B.double()
    bound = 2.0 ** -16 if P == 2 else 2e-6
    assert (torch.linalg.norm(C.double() - ref) / torch.linalg.norm(ref)).item() < bound


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3_scaled"])
def test_fused_zero_k_gives_zeros(hb, fused_ids, variant):
    import torch
    fused, _ = fused_ids
    A = torch.empty((300, 0), device="cuda")
    B = torch.empty((0, 200), device="cuda")
    C = torch.full((300, 200), 7.0, device="cuda")
    hb.gemm(A, B, C, variant=variant, config={"tile": fused[(PARTS[variant], 256)]})
    assert torch.count_nonzero(C).item() == 0


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3"])
@pytest.mark.parametrize("m,n,k,splits", [(256, 256, 65536, 0), (300, 100, 4096, 3),
                                           (512, 64, 20000, 0)])
def test_fused_split_k(hb, fused_ids, variant, m, n, k, splits):
    import torch
    fused, _ = fused_ids
    P = PARTS[variant]
    bn = 64 if n <= 64 else 256
    A = _rand((m, k), k + 11)
    B = _rand((k, n), k + 12)
    ref = A.double() @ B.double()
    cfg = {"split_k": splits, "tile": fused[(P, bn)]}
    C1 = hb.gemm(A, B, variant=variant, config=cfg)
    C2 = hb.gemm(A, B, variant=variant, config=cfg)
    assert torch.equal(C1, C2)  # fixed reduction order
    e = _err(C1, ref)
    if P == 3:
        assert e <= _err(hb.gemm(A, B), ref), e  # no worse than FFMA
    else:
        assert e <= 2.0 ** -16


def test_fused_reference_fixture_exact(hb, fused_ids, oracle_mod, golden_dir):
    import hashlib
    import json
    import os

    import numpy as np
    import torch
    fused, _ = fused_ids
    fix = json.load(open(os.path.join(golden_dir, "sgemm_mod_N512_NITER2.json")))
    n, niter = fix["N"], fix["NITER"]
    m1, m2 = oracle_mod.fill_mod(niter * n * n)
    a = torch.from_numpy(m1).cuda().view(niter, n, n)
    b = torch.from_numpy(m2).cuda().view(niter, n, n)
    out = torch.empty_like(a)
    for i in range(niter):
        hb.gemm(a[i], b[i], out[i], variant="bf16x6", config={"tile": fused[(3, 256)]})
    got = out.cpu().numpy()
    assert hashlib.sha256(np.ascontiguousarray(got).tobytes()).hexdigest() == fix["sha256_result_f32"]


def test_fused_rejects_transposed(hb, fused_ids):
    fused, _ = fused_ids
    A = _rand((64, 96), 1)
    B = _rand((96, 64), 2)
    with pytest.raises(hb.HbsgError) as e:
        hb.gemm(A.t().contiguous(), B, variant="bf16x6", trans_a=True,
                config={"tile": fused[(3, 256)]})
    assert e.value.status == -2


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3", "bf16x6_scaled"])
@pytest.mark.parametrize("ragged", [False, True])
def test_grouped_fused_matches_single(hb, fused_ids, variant, ragged):
    # a grouped plan on the fused tiles computes every problem exactly as the
    # single-GEMM entry point on the unfused tile of the same width
    import numpy as np
    import torch
    fused, plain = fused_ids
    P = PARTS[variant]
    rng = np.random.Generator(np.random.PCG64(17 + ragged))
    As, Bs = [], []
    for i in range(20):
        if ragged:
            m, n, k = (int(x) for x in rng.integers(1, 700, 3))
        else:
            m, n, k = (int(x) for x in rng.integers(2, 21, 3) * 32)
        As.append(_rand((m, k), 100 + i, "scaled" in variant))
        Bs.append(_rand((k, n), 200 + i, "scaled" in variant))
    plan = hb.GroupedPlan(As, Bs, variant=variant, config={"tile": fused[(P, 256)]})
    Cs = plan.run()
    torch.cuda.synchronize()
    for a, b, c in zip(As, Bs, Cs):
        ref = hb.gemm(a, b, variant=variant, config={"tile": plain[(P, 256)], "split_k": 1})
        assert torch.equal(c, ref), (tuple(a.shape), tuple(b.shape))
    plan.close()
