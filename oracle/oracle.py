"""ctypes access to the CPU oracle (oracle.c) and, when it was built, to the
reference testbench's own host_mm compiled from the reference source.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py. The product package never imports it.

Function map (reference lines each one follows are in oracle.c):
  host_mm_rows / host_mm_rows_mt  apps/sgemm/main.cpp:15-26
  host_mm_batched                 apps/sgemm/main.cpp:54-56
  host_mm_fma                     apps/sgemm/kernel.cpp:24-32,186-275
  gemm_f64                        FP64 product (error measurement)
  split_bf16                      FP32 -> BF16 hi/mid/lo split
  host_jacobi                     apps/jacobi/main.cpp:19-48
  bs_host                         apps/blackscholes/bs.hpp:5-125
  bs_device                       apps/blackscholes/bs_kernel.hpp:33-198
  bs_validation_error             apps/blackscholes/main.cpp:119-141
  ref_host_mm                     the reference's host_mm itself (oracle/_ref)
  ref_host_jacobi                 the reference's host_jacobi itself (oracle/_ref)
  ref_bs_host                     the reference's BlkSchlsEqEuroNoDiv itself (oracle/_ref)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_REF_PATH = os.path.join(_HERE, "_ref", "libref_host_mm.so")

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
_L = ctypes.c_long
_I = ctypes.c_int

_lib = None
_ref = None


def build(reference_root: str | None = None) -> None:
    """Compile liboracle.so, and the reference host_mm library when a
    reference checkout is given (argument, else $HB_REFERENCE_ROOT) and holds
    apps/sgemm/main.cpp."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    root = reference_root or os.environ.get("HB_REFERENCE_ROOT")
    if root and os.path.isfile(os.path.join(root, "apps", "sgemm", "main.cpp")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={root}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        l = ctypes.CDLL(_LIB_PATH)
        l.oracle_host_mm_rows.argtypes = [_I, _I, _I, _f32p, _L, _f32p, _L, _f32p, _L, _I, _I]
        l.oracle_host_mm_rows.restype = None
        l.oracle_host_mm_rows_mt.argtypes = [_I, _I, _I, _f32p, _L, _f32p, _L, _f32p, _L, _I, _I, _I]
        l.oracle_host_mm_rows_mt.restype = _I
        l.oracle_host_mm_batched.argtypes = [_f32p, _f32p, _f32p, _I, _I]
        l.oracle_host_mm_batched.restype = None
        l.oracle_host_mm_fma.argtypes = [_I, _I, _I, _f32p, _L, _f32p, _L, _f32p, _L]
        l.oracle_host_mm_fma.restype = None
        l.oracle_gemm_f64.argtypes = [_I, _I, _I, _f32p, _L, _f32p, _L, _f64p, _L]
        l.oracle_gemm_f64.restype = None
        l.oracle_split_bf16.argtypes = [_f32p, _L, _I, _I, _u16p, _u16p, _u16p]
        l.oracle_split_bf16.restype = None
        l.oracle_pow2_exponent.argtypes = [_f32p, _L, _L]
        l.oracle_pow2_exponent.restype = _I
        l.oracle_fill_mod.argtypes = [_f32p, _f32p, _L]
        l.oracle_fill_ramp_identity.argtypes = [_f32p, _f32p, _I]
        l.oracle_fill_identity_ramp.argtypes = [_f32p, _I, _I, _f32p, _I]
        l.oracle_host_jacobi.argtypes = [_I, _I, _f32p, _f32p, _I, _I, _I]
        l.oracle_host_jacobi.restype = None
        l.oracle_fill_jacobi.argtypes = [_f32p, _L]
        l.oracle_fill_jacobi.restype = None
        l.oracle_bs_host.argtypes = [_f32p, _L]
        l.oracle_bs_host.restype = None
        l.oracle_bs_device.argtypes = [_f32p, _L]
        l.oracle_bs_device.restype = None
        _lib = l
    return _lib


_REF_JACOBI_PATH = os.path.join(_HERE, "_ref", "libref_jacobi.so")
_ref_jacobi = None


def ref_available() -> bool:
    return os.path.exists(_REF_PATH)


def ref_jacobi_available() -> bool:
    return os.path.exists(_REF_JACOBI_PATH)


_REF_BS_PATH = os.path.join(_HERE, "_ref", "libref_bs.so")
_ref_bs = None


def ref_bs_available() -> bool:
    return os.path.exists(_REF_BS_PATH)


def ref_bs_lib():
    global _ref_bs
    if _ref_bs is None:
        if not os.path.exists(_REF_BS_PATH):
            raise FileNotFoundError("reference Black-Scholes host library not built (oracle/_ref)")
        _ref_bs = ctypes.CDLL(_REF_BS_PATH)
    return _ref_bs


def ref_jacobi_lib():
    global _ref_jacobi
    if _ref_jacobi is None:
        if not os.path.exists(_REF_JACOBI_PATH):
            raise FileNotFoundError("reference host_jacobi library not built (oracle/_ref)")
        _ref_jacobi = ctypes.CDLL(_REF_JACOBI_PATH)
    return _ref_jacobi


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(_REF_PATH):
            raise FileNotFoundError("reference host_mm library not built (oracle/_ref)")
        _ref = ctypes.CDLL(_REF_PATH)
    return _ref


def ref_host_mm(mat1: np.ndarray, mat2: np.ndarray, n: int, opt: str = "O3") -> np.ndarray:
    """Run the reference's own host_mm (compiled with N = n) on one n x n pair."""
    fn = getattr(ref_lib(), f"hbref_host_mm_{opt}_{n}")
    fn.argtypes = [_f32p, _f32p, _f32p]
    fn.restype = None
    a = np.ascontiguousarray(mat1, dtype=np.float32).reshape(n, n)
    b = np.ascontiguousarray(mat2, dtype=np.float32).reshape(n, n)
    out = np.empty((n, n), dtype=np.float32)
    fn(out, a, b)
    return out


def _c32(x):
    return np.ascontiguousarray(x, dtype=np.float32)


def host_mm(A: np.ndarray, B: np.ndarray, rows: tuple[int, int] | None = None,
            threads: int = 1) -> np.ndarray:
    """host_mm arithmetic (two roundings per step) for general M x K by K x N.
    `rows` restricts the computation to a row range; the returned array then
    holds only those rows."""
    A = _c32(A)
    B = _c32(B)
    M, K = A.shape
    K2, N = B.shape
    assert K == K2
    r0, r1 = rows if rows is not None else (0, M)
    out = np.zeros((r1 - r0, N), dtype=np.float32)
    # C pointer offset so that row r0 lands in out[0].
    Ash = _c32(A[r0:r1])
    if threads == 1:
        lib().oracle_host_mm_rows(r1 - r0, N, K, Ash, K, B, N, out, N, 0, r1 - r0)
    else:
        lib().oracle_host_mm_rows_mt(r1 - r0, N, K, Ash, K, B, N, out, N, 0, r1 - r0, threads)
    return out


def host_mm_batched(mat1: np.ndarray, mat2: np.ndarray, n: int, niter: int) -> np.ndarray:
    out = np.empty(niter * n * n, dtype=np.float32)
    lib().oracle_host_mm_batched(_c32(mat1).ravel(), _c32(mat2).ravel(), out, n, niter)
    return out


def host_mm_fma(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    A = _c32(A)
    B = _c32(B)
    M, K = A.shape
    _, N = B.shape
    out = np.empty((M, N), dtype=np.float32)
    lib().oracle_host_mm_fma(M, N, K, A, K, B, N, out, N)
    return out


def gemm_f64(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    A = _c32(A)
    B = _c32(B)
    M, K = A.shape
    _, N = B.shape
    out = np.empty((M, N), dtype=np.float64)
    lib().oracle_gemm_f64(M, N, K, A, K, B, N, out, N)
    return out


def pow2_exponent(x: np.ndarray) -> int:
    x = _c32(x).ravel()
    return lib().oracle_pow2_exponent(x, x.size, 1)


def split_bf16(v: np.ndarray, exp: int = 0, parts: int = 3):
    """Return (hi, mid, lo) uint16 bf16 bit patterns (lo None for 2 parts)."""
    v = _c32(v).ravel()
    n = v.size
    hi = np.empty(n, np.uint16)
    mid = np.empty(n, np.uint16)
    lo = np.empty(n if parts == 3 else 1, np.uint16)
    lib().oracle_split_bf16(v, n, exp, parts, hi, mid, lo)
    return hi, mid, (lo if parts == 3 else None)


def bf16_to_f32(h: np.ndarray) -> np.ndarray:
    return (np.asarray(h, np.uint16).astype(np.uint32) << 16).view(np.float32)


def fill_mod(count: int):
    a = np.empty(count, np.float32)
    b = np.empty(count, np.float32)
    lib().oracle_fill_mod(a, b, count)
    return a, b


def fill_ramp_identity(n: int):
    a = np.empty(n * n, np.float32)
    b = np.empty(n * n, np.float32)
    lib().oracle_fill_ramp_identity(a, b, n)
    return a.reshape(n, n), b.reshape(n, n)


def fill_identity_ramp(M: int, K: int, N: int):
    a = np.empty(M * K, np.float32)
    b = np.empty(K * N, np.float32)
    lib().oracle_fill_identity_ramp(a, M, K, b, N)
    return a.reshape(M, K), b.reshape(K, N)


def host_jacobi(A0: np.ndarray, nx: int, ny: int, nz: int, c0: int = 2, c1: int = 4) -> np.ndarray:
    """host_jacobi arithmetic (apps/jacobi/main.cpp:19-48) on a flat grid of
    nx*ny*nz floats, element (x, y, z) at ((y*nx)+x)*nz + z."""
    a = _c32(A0).ravel()
    assert a.size == nx * ny * nz
    out = np.empty_like(a)
    lib().oracle_host_jacobi(c0, c1, a, out, nx, ny, nz)
    return out


def fill_jacobi(count: int) -> np.ndarray:
    a = np.empty(count, np.float32)
    lib().oracle_fill_jacobi(a, count)
    return a


def ref_host_jacobi(A0: np.ndarray, nx: int, ny: int, nz: int, c0: int = 2,
                    c1: int = 4) -> np.ndarray:
    """Run the reference's own host_jacobi (apps/jacobi/main.cpp, oracle/_ref)."""
    fn = getattr(ref_jacobi_lib(), "hbref_host_jacobi")
    fn.argtypes = [_I, _I, _f32p, _f32p, _I, _I, _I]
    fn.restype = None
    a = _c32(A0).ravel().copy()
    out = np.zeros_like(a)
    fn(c0, c1, a, out, nx, ny, nz)
    return out


def _bs_records(records: np.ndarray) -> np.ndarray:
    r = np.array(records, dtype=np.float32, copy=True, order="C")
    assert r.ndim == 2 and r.shape[1] == 8, "option records are (n, 8) float32"
    return r


def bs_host(records: np.ndarray) -> np.ndarray:
    """The testbench's host reference (BlkSchlsEqEuroNoDiv, bs.hpp) on (n, 8)
    option records; returns a copy with call and put (columns 5, 6) set."""
    r = _bs_records(records)
    lib().oracle_bs_host(r.ravel(), r.shape[0])
    return r


def bs_device(records: np.ndarray) -> np.ndarray:
    """The device kernel's arithmetic (BlkSchlsEqEuroNoDiv_kernel,
    bs_kernel.hpp) on (n, 8) option records; returns a copy with call and put
    set."""
    r = _bs_records(records)
    lib().oracle_bs_device(r.ravel(), r.shape[0])
    return r


def ref_bs_host(records: np.ndarray) -> np.ndarray:
    """Run the reference's own BlkSchlsEqEuroNoDiv (bs.hpp, oracle/_ref)."""
    fn = getattr(ref_bs_lib(), "hbref_bs_host")
    fn.argtypes = [_f32p, _L]
    fn.restype = None
    r = _bs_records(records)
    fn(r.ravel(), r.shape[0])
    return r


def bs_validation_error(actual: np.ndarray, expected: np.ndarray) -> float:
    """The testbench's check (main.cpp:119-141): the float sum over options of
    the squared call and put differences, accumulated in option order; the
    testbench fails when it exceeds 0.01."""
    a = np.asarray(actual, np.float32)
    e = np.asarray(expected, np.float32)
    err = np.float32(0.0)
    dc = (a[:, 5] - e[:, 5]).astype(np.float32)
    dp = (a[:, 6] - e[:, 6]).astype(np.float32)
    for c, p in zip((dc * dc).astype(np.float32), (dp * dp).astype(np.float32)):
        err = np.float32(err + c)
        err = np.float32(err + p)
    return float(err)


def error_vs_f64(C: np.ndarray, ref64: np.ndarray) -> dict:
    """max-abs error and relative Frobenius error of C against the FP64 product."""
    d = C.astype(np.float64) - ref64
    fro = float(np.linalg.norm(ref64))
    return {
        "max_abs": float(np.max(np.abs(d))) if d.size else 0.0,
        "rel_fro": float(np.linalg.norm(d) / fro) if fro > 0 else float(np.linalg.norm(d)),
    }


def uniform_inputs(shape_a, shape_b, seed: int):
    """Seeded i.i.d. U[-1,1) float32 inputs (numpy PCG64)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    top = np.nextafter(np.float32(1.0), np.float32(0.0))
    a = np.minimum(rng.uniform(-1.0, 1.0, size=shape_a).astype(np.float32), top)
    b = np.minimum(rng.uniform(-1.0, 1.0, size=shape_b).astype(np.float32), top)
    return a, b
