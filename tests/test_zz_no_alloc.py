"""hbsg_gemm_noalloc: the split-BF16 GEMM with its scratch in a fixed array
inside the library, for callers that cannot allocate device memory when they
need a product (a memory pool that already holds the whole GPU, or a loop
that cannot afford the device synchronisation an allocation may cause).

Called through the C ABI and compared with the workspace entry point
(hbsg_gemm_ex with a caller-provided workspace) on two calls in a row. Both
run the same split and tensor-core kernels, so the tolerance is bit-for-bit
equality, the one the other same-kernel comparisons in this suite use.
This file is named to be collected last.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _rand(shape, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.rand(shape, device="cuda", generator=g) * 2 - 1


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x6_scaled", "bf16x3"])
def test_noalloc_matches_workspace_entry_point_twice(variant):
    import torch

    import hb_hammerbench_b200 as hb
    from hb_hammerbench_b200 import _lib
    L = _lib.lib()
    v = _lib.VARIANTS[variant]
    m, n, k = 640, 512, 1000
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, seed in enumerate((1, 2)):  # two calls in a row, different inputs
        A = _rand((m, k), seed)
        B = _rand((k, n), seed + 100)
        C = torch.full((m, n), float("nan"), device="cuda")
        st = L.hbsg_gemm_noalloc(0, 0, m, n, k, _p(A), k, _p(B), n, _p(C), n, v, stream)
        assert st == _lib.OK, (call, L.hbsg_strerror(st))
        need = hb.gemm_workspace_size(m, n, k, variant)
        ws = torch.empty(need, dtype=torch.uint8, device="cuda")
        C_ref = torch.empty((m, n), device="cuda")
        st = L.hbsg_gemm_ex(0, 0, m, n, k, _p(A), k, _p(B), n, _p(C_ref), n, v, None,
                            _p(ws), need, stream)
        assert st == _lib.OK
        torch.cuda.synchronize()
        assert torch.equal(C, C_ref), call
        # and it is a correct product
        ref = A.double() @ B.double()
        rel = (torch.linalg.norm(C.double() - ref) / torch.linalg.norm(ref)).item()
        assert rel < (2.0 ** -16 if variant == "bf16x3" else 2e-6)


@pytest.mark.parametrize("variant", ["bf16x6", "bf16x3"])
def test_noalloc_tall_narrow_product(variant):
    """A tall, narrow product, for which the library's own schedule splits B
    in a pass of its own into the scratch and A inside the product kernel."""
    import torch

    import hb_hammerbench_b200 as hb
    from hb_hammerbench_b200 import _lib
    L = _lib.lib()
    v = _lib.VARIANTS[variant]
    m, n, k = 16384, 64, 2048
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, seed in enumerate((3, 4)):
        A = _rand((m, k), seed)
        B = _rand((k, n), seed + 100)
        C = torch.full((m, n), float("nan"), device="cuda")
        st = L.hbsg_gemm_noalloc(0, 0, m, n, k, _p(A), k, _p(B), n, _p(C), n, v, stream)
        assert st == _lib.OK, (call, L.hbsg_strerror(st))
        need = hb.gemm_workspace_size(m, n, k, variant)
        ws = torch.empty(max(need, 256), dtype=torch.uint8, device="cuda")
        C_ref = torch.empty((m, n), device="cuda")
        st = L.hbsg_gemm_ex(0, 0, m, n, k, _p(A), k, _p(B), n, _p(C_ref), n, v, None,
                            _p(ws), need, stream)
        assert st == _lib.OK
        torch.cuda.synchronize()
        assert torch.equal(C, C_ref), call


def test_noalloc_transposed_operands():
    import torch

    from hb_hammerbench_b200 import _lib
    L = _lib.lib()
    m, n, k = 300, 260, 520
    A = _rand((m, k), 5)
    B = _rand((k, n), 6)
    at = A.t().contiguous()
    bt = B.t().contiguous()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    C1 = torch.empty((m, n), device="cuda")
    C2 = torch.empty((m, n), device="cuda")
    assert L.hbsg_gemm_noalloc(0, 0, m, n, k, _p(A), k, _p(B), n, _p(C1), n, _lib.BF16X6, stream) == 0
    assert L.hbsg_gemm_noalloc(1, 1, m, n, k, _p(at), m, _p(bt), k, _p(C2), n, _lib.BF16X6, stream) == 0
    torch.cuda.synchronize()
    assert torch.equal(C1, C2)


def test_noalloc_rejects_problems_beyond_the_scratch():
    import torch

    import hb_hammerbench_b200 as hb
    from hb_hammerbench_b200 import _lib
    L = _lib.lib()
    # BF16X6 at 2048^3 with transposed operands (always served by the kernels
    # whose split parts live in the scratch) needs 50 MB of parts > 16 MiB
    n = 2048
    assert hb.split_layout(n, n, n, "bf16x6")["total_bytes"] > _lib.NOALLOC_SCRATCH_BYTES
    A = torch.zeros((n, n), device="cuda")
    C = torch.full((n, n), 7.0, device="cuda")
    st = L.hbsg_gemm_noalloc(1, 1, n, n, n, _p(A), n, _p(A), n, _p(C), n, _lib.BF16X6, None)
    assert st == _lib.ERR_WORKSPACE
    torch.cuda.synchronize()
    assert bool((C == 7.0).all())  # nothing was launched
    # FFMA needs no scratch and is not served here
    assert L.hbsg_gemm_noalloc(0, 0, 8, 8, 8, _p(A), n, _p(A), n, _p(C), n, _lib.FFMA, None) == \
        _lib.ERR_UNSUPPORTED
