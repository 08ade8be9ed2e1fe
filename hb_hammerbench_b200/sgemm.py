"""Host-side interface of the SGEMM hot path (torch tensors in, C ABI under).

Mirrors the HammerBench sgemm benchmark's host flow (apps/sgemm/main.cpp):
  sgemm(mat1, mat2, result, n, niter)  ~ the enqueue of `kernel` with argv
                                         {mat1, mat2, result, pod}
                                         (main.cpp:86-98): NITER independent
                                         n x n row-major products, matrix i at
                                         element offset n*n*i.
  gemm(a, b, c, ...)                   ~ the legacy rectangular kernel_mm_opt
                                         (apps/legacy/gemm/sgemm_data_parallel/
                                         kernel.cpp:323-344) with strides.
Every call goes through libhbsg.so on the tensors' device and the current
torch stream; errors raise HbsgError with the library's status.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import Config, HbsgError, TileInfo, check, lib  # noqa: F401


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _variant(v) -> int:
    if isinstance(v, str):
        return _lib.VARIANTS[v.lower()]
    return int(v)


def _ptr(t: torch.Tensor | None) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _check_f32_cuda(name: str, t: torch.Tensor) -> None:
    if t.dtype != torch.float32 or not t.is_cuda:
        raise TypeError(f"{name} must be a float32 CUDA tensor")


def _config(cfg) -> ctypes.POINTER(Config) | None:
    if cfg is None:
        return None
    if isinstance(cfg, dict):
        cfg = Config(**cfg)
    return ctypes.pointer(cfg)


def sgemm_workspace_size(n: int, niter: int, variant="ffma") -> int:
    return int(lib().hbsg_sgemm_workspace_size(n, niter, _variant(variant)))


def gemm_workspace_size(m: int, n: int, k: int, variant="ffma", config=None) -> int:
    return int(lib().hbsg_gemm_workspace_size(m, n, k, _variant(variant), _config(config)))


def _workspace(nbytes: int, device, workspace: torch.Tensor | None):
    if nbytes == 0:
        return workspace
    if workspace is not None and workspace.numel() * workspace.element_size() >= nbytes:
        return workspace
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def sgemm(mat1: torch.Tensor, mat2: torch.Tensor, result: torch.Tensor | None = None,
          n: int | None = None, niter: int | None = None, variant="ffma",
          workspace: torch.Tensor | None = None) -> torch.Tensor:
    """result[i] = mat1[i] @ mat2[i] for i < niter (each n x n, contiguous)."""
    _check_f32_cuda("mat1", mat1)
    _check_f32_cuda("mat2", mat2)
    if not (mat1.is_contiguous() and mat2.is_contiguous()):
        raise ValueError("mat1 and mat2 must be contiguous")
    if n is None:
        n = mat1.shape[-1]
    if niter is None:
        niter = mat1.numel() // (n * n) if n else 0
    if mat1.numel() < niter * n * n or mat2.numel() < niter * n * n:
        raise ValueError("buffers smaller than niter*n*n")
    if result is None:
        result = torch.empty_like(mat1)
    _check_f32_cuda("result", result)
    v = _variant(variant)
    with torch.cuda.device(mat1.device):
        if v == _lib.FFMA and workspace is None:
            st = lib().hbsg_sgemm(_ptr(mat1), _ptr(mat2), _ptr(result), n, niter, _stream())
            check(st, "hbsg_sgemm")
        else:
            need = sgemm_workspace_size(n, niter, v)
            ws = _workspace(need, mat1.device, workspace)
            st = lib().hbsg_sgemm_variant(_ptr(mat1), _ptr(mat2), _ptr(result), n, niter, v,
                                          _ptr(ws), need, _stream())
            check(st, "hbsg_sgemm_variant")
    return result


def resolve_config(m: int, n: int, k: int, variant, trans: bool, config):
    """The schedule a call runs: the caller's config when given, else the
    autotuner's measured choice for the shape class (row-major operands; the
    tuner measures those), else None (the library heuristic)."""
    if config is not None or trans:
        return config
    from . import autotune
    if not autotune.enabled():
        return None
    name = variant if isinstance(variant, str) else {v: k_ for k_, v in _lib.VARIANTS.items()}[int(variant)]
    return autotune.lookup(m, n, k, name.lower())


def gemm(a: torch.Tensor, b: torch.Tensor, c: torch.Tensor | None = None, variant="ffma",
         trans_a: bool = False, trans_b: bool = False, config=None,
         workspace: torch.Tensor | None = None) -> torch.Tensor:
    """c = op(a) @ op(b) for 2-D float32 CUDA tensors with unit inner stride.
    With trans_a, `a` holds A^T (k x m); with trans_b, `b` holds B^T (n x k).
    Without a config the autotuner's choice for the shape class is used when
    one is known (resolve_config)."""
    _check_f32_cuda("a", a)
    _check_f32_cuda("b", b)
    if a.dim() != 2 or b.dim() != 2 or a.stride(1) != 1 or b.stride(1) != 1:
        raise ValueError("a and b must be 2-D with unit inner stride")
    m, k = (a.shape[1], a.shape[0]) if trans_a else (a.shape[0], a.shape[1])
    kb, n = (b.shape[1], b.shape[0]) if trans_b else (b.shape[0], b.shape[1])
    if k != kb:
        raise ValueError(f"inner dimensions differ: {k} vs {kb}")
    if c is None:
        c = torch.empty((m, n), dtype=torch.float32, device=a.device)
    _check_f32_cuda("c", c)
    if c.dim() != 2 or c.stride(1) != 1 or tuple(c.shape) != (m, n):
        raise ValueError("c must be m x n with unit inner stride")
    v = _variant(variant)
    cfgp = _config(resolve_config(m, n, k, variant, trans_a or trans_b, config))
    with torch.cuda.device(a.device):
        need = int(lib().hbsg_gemm_workspace_size_for(int(trans_a), int(trans_b), m, n, k,
                                                      _ptr(a), a.stride(0), _ptr(b), b.stride(0),
                                                      v, cfgp))
        ws = _workspace(need, a.device, workspace)
        st = lib().hbsg_gemm_ex(int(trans_a), int(trans_b), m, n, k, _ptr(a), a.stride(0),
                                _ptr(b), b.stride(0), _ptr(c), c.stride(0), v, cfgp,
                                _ptr(ws), need, _stream())
        check(st, "hbsg_gemm_ex")
    return c


def _problems(As, Bs, Cs):
    arr = (_lib.Problem * len(As))()
    for i, (a, b, c) in enumerate(zip(As, Bs, Cs)):
        for name, t in (("a", a), ("b", b), ("c", c)):
            _check_f32_cuda(name, t)
            if t.dim() != 2 or (t.numel() and t.stride(1) != 1):
                raise ValueError(f"problem {i}: {name} must be 2-D with unit inner stride")
        m, k = a.shape
        k2, n = b.shape
        if k != k2 or tuple(c.shape) != (m, n):
            raise ValueError(f"problem {i}: shapes {tuple(a.shape)} x {tuple(b.shape)} -> {tuple(c.shape)}")
        arr[i] = _lib.Problem(m, n, k, a.data_ptr(), max(a.stride(0), k, 1), b.data_ptr(),
                              max(b.stride(0), n, 1), c.data_ptr(), max(c.stride(0), n, 1))
    return arr


class GroupedPlan:
    """A grouped product C_i = A_i @ B_i over many problems of uneven sizes,
    planned once (tables in a workspace, launches captured in a CUDA graph)
    and replayed with run(). The plan reads the tensors' current contents on
    every run; keep them (and the plan) alive while it is used."""

    def __init__(self, As, Bs, Cs=None, variant="ffma", config=None):
        if Cs is None:
            Cs = [torch.empty((a.shape[0], b.shape[1]), device=a.device) for a, b in zip(As, Bs)]
        self.As, self.Bs, self.Cs = list(As), list(Bs), list(Cs)
        self.variant = _variant(variant)
        self._arr = _problems(self.As, self.Bs, self.Cs)
        if config is None and self.As:
            from . import autotune
            if autotune.enabled():
                name = {v: k_ for k_, v in _lib.VARIANTS.items()}[self.variant]
                dims = [(a.shape[0], b.shape[1], a.shape[1]) for a, b in zip(self.As, self.Bs)]
                config = autotune.lookup_grouped(dims, name)
        self.config = config
        self._cfg = _config(config)
        dev = self.As[0].device if self.As else torch.device("cuda")
        with torch.cuda.device(dev):
            need = int(lib().hbsg_grouped_workspace_size(len(self.As), self._arr, self.variant,
                                                          self._cfg))
            self.workspace = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
            torch.cuda.current_stream().synchronize()
            self._plan = ctypes.c_void_p()
            check(lib().hbsg_grouped_plan_create(ctypes.byref(self._plan), len(self.As), self._arr,
                                                 self.variant, self._cfg,
                                                 _ptr(self.workspace), need),
                  "hbsg_grouped_plan_create")
        self.device = dev

    def run(self):
        with torch.cuda.device(self.device):
            check(lib().hbsg_grouped_run(self._plan, _stream()), "hbsg_grouped_run")
        return self.Cs

    def close(self):
        if self._plan:
            lib().hbsg_grouped_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gemm_grouped(As, Bs, Cs=None, variant="ffma", config=None, workspace=None):
    """One-shot grouped product (tables built and uploaded per call, no graph)."""
    if Cs is None:
        Cs = [torch.empty((a.shape[0], b.shape[1]), device=a.device) for a, b in zip(As, Bs)]
    arr = _problems(As, Bs, Cs)
    v = _variant(variant)
    cfgp = _config(config)
    dev = As[0].device if len(As) else torch.device("cuda")
    with torch.cuda.device(dev):
        need = int(lib().hbsg_grouped_workspace_size(len(As), arr, v, cfgp))
        ws = _workspace(max(need, 256), dev, workspace)
        check(lib().hbsg_gemm_grouped(len(As), arr, v, cfgp, _ptr(ws), need, _stream()),
              "hbsg_gemm_grouped")
    return Cs


def split_layout(m: int, n: int, k: int, variant="bf16x6") -> dict:
    """Byte offsets of the BF16 operand parts inside a split-BF16 workspace."""
    lay = _lib.SplitLayout()
    check(lib().hbsg_get_split_layout(m, n, k, _variant(variant), ctypes.byref(lay)),
          "hbsg_get_split_layout")
    return {f: getattr(lay, f) for f, _ in _lib.SplitLayout._fields_}


def tiles() -> list[dict]:
    """The tile-shape table (1-based ids) the autotuner searches."""
    out = []
    for t in range(1, lib().hbsg_num_tiles() + 1):
        info = TileInfo()
        check(lib().hbsg_tile_describe(t, ctypes.byref(info)), "hbsg_tile_describe")
        out.append({"tile": t, "family": "ffma" if info.variant_class == 0 else "bf16",
                    "bm": info.bm, "bn": info.bn, "bk": info.bk,
                    "threads": info.threads, "smem_bytes": info.smem_bytes,
                    "parts": info.parts, "fused": bool(info.fused)})
    return out


def check_device() -> None:
    check(lib().hbsg_check_device(_stream()), "device check")


def fp32_peak(packed: bool = True, iters: int = 4096, repeats: int = 5) -> dict:
    """Measured FP32 SIMT roof of the current device: the probe kernel of
    independent FMA chains (hbsg_fp32_peak_probe) timed with CUDA events on
    the current stream, best of `repeats` launches after one warm-up launch.
    Returns {"tflops": ..., "ms": ..., "flops": ...}."""
    sink = torch.zeros(1, device="cuda")
    flops = ctypes.c_double()
    stream = torch.cuda.current_stream()

    def launch():
        check(lib().hbsg_fp32_peak_probe(int(packed), iters, _ptr(sink), ctypes.byref(flops),
                                         _stream()), "hbsg_fp32_peak_probe")
    launch()
    best = None
    for _ in range(repeats):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return {"tflops": flops.value / (best * 1e-3) / 1e12, "ms": best, "flops": flops.value}


def jacobi(a0: torch.Tensor, nx: int, ny: int, nz: int, c0: int = 2, c1: int = 4,
           out: torch.Tensor | None = None) -> torch.Tensor:
    """One 7-point Jacobi step (the suite's apps/jacobi kernel) on a flat
    float32 CUDA grid of nx*ny*nz elements, element (x, y, z) at
    ((y*nx)+x)*nz + z: out = c1 * (sum of six neighbours) - c0 * a0."""
    _check_f32_cuda("a0", a0)
    if not a0.is_contiguous() or a0.numel() != nx * ny * nz:
        raise ValueError("a0 must be a contiguous grid of nx*ny*nz floats")
    if out is None:
        out = torch.empty_like(a0)
    _check_f32_cuda("out", out)
    if not out.is_contiguous() or out.numel() != a0.numel():
        raise ValueError("out must be a contiguous grid of nx*ny*nz floats")
    with torch.cuda.device(a0.device):
        check(lib().hbsg_jacobi(c0, c1, _ptr(a0), _ptr(out), nx, ny, nz, _stream()),
              "hbsg_jacobi")
    return out
