"""Grouped GEMM (persistent kernel over the tiles of many uneven problems,
CUDA-graph replay) on the GPU. Every problem's result must be bit-identical
to the single-GEMM entry point with the same tile shape and no K slicing: a
tile's arithmetic does not depend on which CTA or launch computes it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hb():
    import hb_hammerbench_b200 as hb
    return hb


def _problems(seed, count, lo=64, hi=640, step=32, ragged=False):
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    g = torch.Generator(device="cuda").manual_seed(seed)
    As, Bs = [], []
    for _ in range(count):
        if ragged:
            m, n, k = (int(x) for x in rng.integers(1, hi, 3))
        else:
            m, n, k = (int(x) for x in rng.integers(lo // step, hi // step + 1, 3) * step)
        As.append(torch.rand((m, k), device="cuda", generator=g) * 2 - 1)
        Bs.append(torch.rand((k, n), device="cuda", generator=g) * 2 - 1)
    return As, Bs


TILE_FOR = {"ffma": 1, "bf16x6": 10, "bf16x3": 13, "bf16x6_scaled": 10, "bf16x3_scaled": 13}


@pytest.mark.parametrize("variant", ["ffma", "bf16x6", "bf16x3", "bf16x6_scaled"])
@pytest.mark.parametrize("ragged", [False, True])
def test_grouped_plan_matches_single(hb, variant, ragged):
    import torch
    As, Bs = _problems(7 + ragged, 24, ragged=ragged)
    plan = hb.GroupedPlan(As, Bs, variant=variant)
    Cs = plan.run()
    torch.cuda.synchronize()
    for a, b, c in zip(As, Bs, Cs):
        ref = hb.gemm(a, b, variant=variant, config={"tile": TILE_FOR[variant], "split_k": 1})
        assert torch.equal(c, ref), (tuple(a.shape), tuple(b.shape))
    plan.close()


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3", "bf16x6_scaled", "bf16x3_scaled"])
@pytest.mark.parametrize("ragged", [False, True])
def test_grouped_pair_tiles_match_single(hb, variant, ragged):
    # CTA-pair tiles (256 x 256, cta_group::2) in a grouped plan: each problem
    # bit-identical to the single-GEMM entry point on the same pair tile
    import torch
    P = 3 if "x6" in variant else 2
    tile = [t["tile"] for t in hb.tiles() if t["family"] == "bf16" and not t["fused"]
            and t["bm"] == 256 and t["parts"] == P][0]
    As, Bs = _problems(23 + ragged, 20, hi=700, ragged=ragged)
    plan = hb.GroupedPlan(As, Bs, variant=variant, config={"tile": tile})
    Cs = plan.run()
    torch.cuda.synchronize()
    for a, b, c in zip(As, Bs, Cs):
        ref = hb.gemm(a, b, variant=variant, config={"tile": tile, "split_k": 1})
        assert torch.equal(c, ref), (tuple(a.shape), tuple(b.shape))
    plan.close()


@pytest.mark.parametrize("variant", ["ffma", "bf16x6"])
def test_grouped_one_shot_matches_plan(hb, variant):
    import torch
    As, Bs = _problems(11, 16)
    Cs1 = hb.gemm_grouped(As, Bs, variant=variant)
    plan = hb.GroupedPlan(As, Bs, variant=variant)
    Cs2 = plan.run()
    torch.cuda.synchronize()
    for c1, c2 in zip(Cs1, Cs2):
        assert torch.equal(c1, c2)


def test_plan_rerun_sees_new_operand_values(hb):
    import torch
    As, Bs = _problems(13, 8)
    plan = hb.GroupedPlan(As, Bs, variant="bf16x6")
    first = [c.clone() for c in plan.run()]
    for a in As:
        a.mul_(-2.0)  # exact scaling: every product term scales exactly
    second = plan.run()
    torch.cuda.synchronize()
    for c1, c2 in zip(first, second):
        assert torch.equal(c2, -2.0 * c1)


def test_degenerate_problems(hb):
    import torch
    As = [torch.rand((64, 0), device="cuda"), torch.rand((0, 32), device="cuda"),
          torch.rand((33, 17), device="cuda")]
    Bs = [torch.rand((0, 40), device="cuda"), torch.rand((32, 8), device="cuda"),
          torch.rand((17, 5), device="cuda")]
    Cs = [torch.full((64, 40), 3.0, device="cuda"), torch.empty((0, 8), device="cuda"),
          torch.empty((33, 5), device="cuda")]
    for v in ("ffma", "bf16x6"):
        hb.gemm_grouped(As, Bs, Cs, variant=v)
        torch.cuda.synchronize()
        assert torch.count_nonzero(Cs[0]).item() == 0
        assert torch.equal(Cs[2], hb.gemm(As[2], Bs[2], variant=v,
                                          config={"tile": TILE_FOR[v], "split_k": 1}))


def test_errors(hb):
    import ctypes

    from hb_hammerbench_b200 import _lib
    L = _lib.lib()
    assert L.hbsg_gemm_grouped(-1, None, 0, None, None, 0, None) == _lib.ERR_INVALID_ARG
    arr = (_lib.Problem * 1)()
    arr[0] = _lib.Problem(8, 8, 8, 0, 8, 0, 8, 0, 8)  # null pointers
    assert L.hbsg_gemm_grouped(1, arr, 0, None, None, 0, None) == _lib.ERR_INVALID_ARG
    arr[0] = _lib.Problem(8, 8, 8, 0x1000, 4, 0x1000, 8, 0x1000, 8)  # lda < k
    assert L.hbsg_gemm_grouped(1, arr, 0, None, None, 0, None) == _lib.ERR_INVALID_ARG
    arr[0] = _lib.Problem(8, 8, 8, 0x1000, 8, 0x1000, 8, 0x1000, 8)
    assert L.hbsg_gemm_grouped(1, arr, 2, None, None, 0, None) == _lib.ERR_WORKSPACE
    plan = ctypes.c_void_p()
    assert L.hbsg_grouped_plan_create(ctypes.byref(plan), 1, arr, 9, None, None, 0) == _lib.ERR_UNSUPPORTED
    assert L.hbsg_grouped_run(None, None) == _lib.ERR_INVALID_ARG
