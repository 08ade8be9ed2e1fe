"""The autotuner measures schedules on the GPU; the chosen schedule computes
the same product as the default one: bit-identical for an FFMA schedule
without K slices (one FMA chain per element), within the FP64-relative
bound otherwise."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def cache(tmp_path, monkeypatch):
    from hb_hammerbench_b200 import autotune
    monkeypatch.setenv("HBSG_AUTOTUNE_CACHE", str(tmp_path / "t.json"))
    autotune.clear_memory_cache()
    yield
    autotune.clear_memory_cache()


@pytest.mark.parametrize("variant", ["ffma", "bf16x6"])
def test_tune_and_use(cache, variant):
    import torch

    import hb_hammerbench_b200 as hb
    from hb_hammerbench_b200 import autotune
    m, n, k = 1024, 768, 1024
    cfg = autotune.tune(m, n, k, variant, steps=2, max_candidates=6)
    assert autotune.lookup(m, n, k, variant) == cfg
    A = torch.rand((m, k), device="cuda") * 2 - 1
    B = torch.rand((k, n), device="cuda") * 2 - 1
    C1 = hb.gemm(A, B, variant=variant, config=cfg)
    C0 = hb.gemm(A, B, variant=variant)
    ref = A.double() @ B.double()
    if variant == "ffma" and cfg.get("split_k", 0) <= 1:
        assert torch.equal(C0, C1)  # same single FMA chain per element
    else:  # K slices change the summation order: FP64-relative bound instead
        assert (torch.linalg.norm(C1.double() - ref) / torch.linalg.norm(ref)).item() < 2e-6


def test_tune_grouped(cache):
    import torch

    import hb_hammerbench_b200 as hb
    from hb_hammerbench_b200 import autotune
    As = [torch.rand((m, k), device="cuda") for m, k in ((256, 320), (128, 96), (512, 64))]
    Bs = [torch.rand((k, n), device="cuda") for k, n in ((320, 192), (96, 640), (64, 256))]
    cfg = autotune.tune_grouped(As, Bs, "bf16x6", steps=1)
    x6_tiles = [t["tile"] for t in hb.tiles() if t["family"] == "bf16" and t["parts"] == 3]
    assert cfg["tile"] in x6_tiles
    dims = [(a.shape[0], b.shape[1], a.shape[1]) for a, b in zip(As, Bs)]
    assert autotune.lookup_grouped(dims, "bf16x6") == cfg
    Cs = hb.GroupedPlan(As, Bs, variant="bf16x6", config=cfg).run()
    torch.cuda.synchronize()
    for a, b, c in zip(As, Bs, Cs):
        ref = a.double() @ b.double()
        assert (torch.linalg.norm(c.double() - ref) / torch.linalg.norm(ref)).item() < 2e-6


def test_tuned_choice_is_the_default(cache, monkeypatch):
    # with the lookup on, a call without a schedule runs the cached choice for
    # its shape class: bit-identical to passing that schedule explicitly
    import torch

    import hb_hammerbench_b200 as hb
    from hb_hammerbench_b200 import autotune
    fused = [t["tile"] for t in hb.tiles() if t["fused"] and t["parts"] == 3 and t["bn"] == 256][0]
    m, n, k = 1000, 900, 1500
    cfg = {"tile": fused, "split_k": 0, "chunk_k": 32, "raster_group": 8}
    autotune._store(autotune.shape_key(m, n, k, "bf16x6"), {"config": cfg, "ms": 1.0})
    monkeypatch.setenv("HBSG_AUTOTUNE", "1")
    A = torch.rand((m, k), device="cuda") * 2 - 1
    B = torch.rand((k, n), device="cuda") * 2 - 1
    assert torch.equal(hb.gemm(A, B, variant="bf16x6"), hb.gemm(A, B, variant="bf16x6", config=cfg))
    monkeypatch.setenv("HBSG_AUTOTUNE", "0")
    C0 = hb.gemm(A, B, variant="bf16x6")  # library heuristic: chunk 64, not the cached 32
    ref = A.double() @ B.double()
    assert (torch.linalg.norm(C0.double() - ref) / torch.linalg.norm(ref)).item() < 2e-6
