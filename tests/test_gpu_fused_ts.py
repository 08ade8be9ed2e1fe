"""Fused-split tiles that keep A's BF16 parts in tensor memory (single CTA,
128 x 64 output tiles, tcgen05.mma with A from TMEM) on the GPU, through the
C ABI.

The A converters write the same split values into tensor memory that the
split pass writes to HBM, the B converters write B's parts in the unfused
operand layout, and products, product order and TMEM drains are those of the
unfused kernels, so each result is bit-identical to the unfused single-CTA
tile of the same product count and width. Bars otherwise as in
test_gpu_bf16.py.
"""
import pytest

pytestmark = pytest.mark.gpu

PARTS = {"bf16x6": 3, "bf16x3": 2, "bf16x6_scaled": 3, "bf16x3_scaled": 2}


@pytest.fixture(scope="module")
def hb():
    import hb_hammerbench_b200 as hb
    return hb


@pytest.fixture(scope="module")
def all_ids(hb):
    """({(parts, bn): A-in-TMEM tile id}, {(parts, bn): unfused single-CTA tile id})."""
    ts, plain = {}, {}
    for t in hb.tiles():
        if t["family"] != "bf16" or t["bm"] != 128:
            continue
        (ts if t["fused"] else plain)[(t["parts"], t["bn"])] = t["tile"]
    assert set(ts) == {(3, 64), (2, 64), (3, 128), (2, 128)}
    return ts, plain


@pytest.fixture(scope="module")
def ids(all_ids):
    """The 64-wide tiles: ({parts: A-in-TMEM id}, {parts: unfused id})."""
    ts, plain = all_ids
    return ({p: ts[(p, 64)] for p in (2, 3)}, {p: plain[(p, 64)] for p in (2, 3)})


def _rand(shape, seed, wide=False):
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


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3", "bf16x6_scaled", "bf16x3_scaled"])
@pytest.mark.parametrize("bn", [64, 128])
@pytest.mark.parametrize("m,n,k", [(128, 64, 32), (256, 64, 64), (300, 200, 100),
                                   (1000, 700, 1031), (64, 520, 7), (777, 64, 2048),
                                   (4099, 33, 4100)])
def test_ts_matches_unfused(hb, all_ids, variant, bn, m, n, k):
    import torch
    ts, plain = all_ids
    P = PARTS[variant]
    wide = "scaled" in variant
    A = _rand((m, k), m + 3 * k, wide)
    B = _rand((k, n), n + 7 * k, wide)
    cfg = {"split_k": 1, "chunk_k": 64}
    Ct = hb.gemm(A, B, variant=variant, config={**cfg, "tile": ts[(P, bn)]})
    Cu = hb.gemm(A, B, variant=variant, config={**cfg, "tile": plain[(P, bn)]})
    assert torch.equal(Ct, Cu)


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3"])
def test_ts128_split_k_and_fixture(hb, all_ids, oracle_mod, golden_dir, variant):
    """128-wide A-in-TMEM tiles: fixed-order split-K and the i % 7 / i % 3
    fixture's SHA-256 (X6)."""
    import hashlib
    import json
    import os

    import numpy as np
    import torch
    ts, _ = all_ids
    P = PARTS[variant]
    A = _rand((384, 20000), 31)
    B = _rand((20000, 200), 32)
    cfg = {"split_k": 0, "tile": ts[(P, 128)]}
    C1 = hb.gemm(A, B, variant=variant, config=cfg)
    assert torch.equal(C1, hb.gemm(A, B, variant=variant, config=cfg))
    ref = A.double() @ B.double()
    e = _err(C1, ref)
    assert e <= (_err(hb.gemm(A, B), ref) if P == 3 else 2.0 ** -16), e
    if P == 3:
        fix = json.load(open(os.path.join(golden_dir, "sgemm_mod_N512_NITER2.json")))
        n, niter = fix["N"], fix["NITER"]
        m1, m2 = oracle_mod.fill_mod(niter * n * n)
        a = torch.from_numpy(m1).cuda().view(niter, n, n)
        b = torch.from_numpy(m2).cuda().view(niter, n, n)
        out = torch.empty_like(a)
        for i in range(niter):
            hb.gemm(a[i], b[i], out[i], variant="bf16x6", config={"tile": ts[(3, 128)]})
        got = out.cpu().numpy()
        assert hashlib.sha256(np.ascontiguousarray(got).tobytes()).hexdigest() == \
            fix["sha256_result_f32"]


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3"])
@pytest.mark.parametrize("chunk_k", [32, 256])
def test_ts_drain_intervals(hb, ids, variant, chunk_k):
    import torch
    ts, plain = ids
    P = PARTS[variant]
    A = _rand((512, 3000), 41)
    B = _rand((3000, 64), 42)
    cfg = {"split_k": 1, "chunk_k": chunk_k}
    assert torch.equal(hb.gemm(A, B, variant=variant, config={**cfg, "tile": ts[P]}),
                       hb.gemm(A, B, variant=variant, config={**cfg, "tile": plain[P]}))


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3"])
@pytest.mark.parametrize("m,n,k,splits", [(256, 64, 65536, 0), (300, 50, 4096, 3),
                                           (512, 64, 20000, 0)])
def test_ts_split_k(hb, ids, variant, m, n, k, splits):
    import torch
    ts, plain = ids
    P = PARTS[variant]
    A = _rand((m, k), k + 11)
    B = _rand((k, n), k + 12)
    ref = A.double() @ B.double()
    cfg = {"split_k": splits, "tile": ts[P]}
    C1 = hb.gemm(A, B, variant=variant, config=cfg)
    C2 = hb.gemm(A, B, variant=variant, config=cfg)
    assert torch.equal(C1, C2)  # fixed reduction order
    e = _err(C1, ref)
    if P == 3:
        assert e <= _err(hb.gemm(A, B), ref), e  # no worse than FFMA
    else:
        assert e <= 2.0 ** -16


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3_scaled"])
def test_ts_zero_k_gives_zeros(hb, ids, variant):
    import torch
    ts, _ = ids
    A = torch.empty((300, 0), device="cuda")
    B = torch.empty((0, 200), device="cuda")
    C = torch.full((300, 200), 7.0, device="cuda")
    hb.gemm(A, B, C, variant=variant, config={"tile": ts[PARTS[variant]]})
    assert torch.count_nonzero(C).item() == 0


def test_ts_reference_fixture_exact(hb, ids, oracle_mod, golden_dir):
    import hashlib
    import json
    import os

    import numpy as np
    import torch
    ts, _ = ids
    fix = json.load(open(os.path.join(golden_dir, "sgemm_mod_N512_NITER2.json")))
    n, niter = fix["N"], fix["NITER"]
    m1, m2 = oracle_mod.fill_mod(niter * n * n)
    a = torch.from_numpy(m1).cuda().view(niter, n, n)
    b = torch.from_numpy(m2).cuda().view(niter, n, n)
    out = torch.empty_like(a)
    for i in range(niter):
        hb.gemm(a[i], b[i], out[i], variant="bf16x6", config={"tile": ts[3]})
    got = out.cpu().numpy()
    assert hashlib.sha256(np.ascontiguousarray(got).tobytes()).hexdigest() == fix["sha256_result_f32"]


def test_ts_rejected_where_unsupported(hb, ids):
    ts, _ = ids
    A = _rand((64, 96), 1)
    B = _rand((96, 64), 2)
    with pytest.raises(hb.HbsgError) as e:  # transposed operands
        hb.gemm(A.t().contiguous(), B, variant="bf16x6", trans_a=True, config={"tile": ts[3]})
    assert e.value.status == -2
    with pytest.raises(hb.HbsgError):  # grouped plans run the CTA-pair fused tiles only
        hb.GroupedPlan([A], [B], variant="bf16x6", config={"tile": ts[3]})


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3"])
def test_ts_tall_m_config(hb, ids, variant):
    """65536 x 64 x 4096 (the tall, narrow benchmark shape): bit-identical to
    the unfused tile, X6 no worse than FFMA against FP64."""
    import torch
    ts, plain = ids
    P = PARTS[variant]
    A = _rand((65536, 4096), 5)
    B = _rand((4096, 64), 6)
    Ct = hb.gemm(A, B, variant=variant, config={"tile": ts[P], "split_k": 1})
    Cu = hb.gemm(A, B, variant=variant, config={"tile": plain[P], "split_k": 1})
    assert torch.equal(Ct, Cu)
    ref = A.double() @ B.double()
    e = _err(Ct, ref)
    if P == 3:
        assert e <= _err(hb.gemm(A, B, variant="ffma"), ref)
    else:
        assert e <= 2.0 ** -16


def test_ts_workspace_holds_b_parts(hb, ids):
    """The A-in-TMEM tiles keep B's parts in the workspace (P x N x K padded to
    32, bf16); a workspace 256 bytes short is rejected through the C ABI
    (status -3) before any launch, and the full one gives the same result as
    the host interface's own allocation."""
    import ctypes

    import torch
    from hb_hammerbench_b200 import _lib
    ts, _ = ids
    m, n, k = 4096, 64, 4100
    for v, P in (("bf16x6", 3), ("bf16x3", 2)):
        cfg = {"tile": ts[P], "split_k": 1}
        need = hb.gemm_workspace_size(m, n, k, v, cfg)
        assert need >= P * n * ((k + 31) // 32 * 32) * 2
        A = _rand((m, k), 7)
        B = _rand((k, n), 8)
        C = torch.empty((m, n), device="cuda")
        ws = torch.empty(need, dtype=torch.uint8, device="cuda")
        c = ctypes.pointer(_lib.Config(**cfg))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        args = (0, 0, m, n, k, ctypes.c_void_p(A.data_ptr()), A.stride(0),
                ctypes.c_void_p(B.data_ptr()), B.stride(0), ctypes.c_void_p(C.data_ptr()),
                C.stride(0), _lib.VARIANTS[v], c, ctypes.c_void_p(ws.data_ptr()))
        assert _lib.lib().hbsg_gemm_ex(*args, need - 256, stream) == _lib.ERR_WORKSPACE
        assert _lib.lib().hbsg_gemm_ex(*args, need, stream) == _lib.OK
        assert torch.equal(C, hb.gemm(A, B, variant=v, config=cfg))
