"""The C-ABI library: loads on a CPU host, exports every function declared in
include/hbsg.h, and rejects bad arguments before touching a device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(hbsg_[a-z_0-9]+)\s*\(", text, re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def L():
    from hb_hammerbench_b200 import _lib
    return _lib


def test_library_loads(L):
    assert L.lib().hbsg_version() == 101


def test_exports_every_declared_symbol(L):
    names = _declared_functions()
    assert len(names) >= 10
    lib = L.lib()
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"


def test_python_signatures_cover_header(L):
    assert set(_declared_functions()) == set(L.SIGNATURES)


def test_strerror(L):
    lib = L.lib()
    assert lib.hbsg_strerror(0) == b"success"
    for st in range(-7, 0):
        s = lib.hbsg_strerror(st)
        assert s and s != b"unknown status"
    assert lib.hbsg_strerror(-99) == b"unknown status"


def test_argument_errors_before_any_launch(L):
    lib = L.lib()
    P = ctypes.c_void_p
    fake = P(0x10000)
    # null operands
    assert lib.hbsg_sgemm(None, fake, fake, 16, 1, None) == L.ERR_INVALID_ARG
    assert lib.hbsg_sgemm(fake, fake, None, 16, 1, None) == L.ERR_INVALID_ARG
    # negative sizes
    assert lib.hbsg_sgemm(fake, fake, fake, -1, 1, None) == L.ERR_INVALID_ARG
    assert lib.hbsg_sgemm(fake, fake, fake, 16, -2, None) == L.ERR_INVALID_ARG
    # empty problems are a no-op success
    assert lib.hbsg_sgemm(None, None, None, 0, 3, None) == L.OK
    assert lib.hbsg_sgemm(None, None, None, 8, 0, None) == L.OK
    # bad variant
    assert lib.hbsg_sgemm_variant(fake, fake, fake, 16, 1, 99, None, 0, None) == L.ERR_UNSUPPORTED
    # leading dimensions smaller than the row length
    assert lib.hbsg_gemm(0, 0, 4, 8, 16, fake, 8, fake, 8, fake, 8, 0, None, 0, None) == L.ERR_INVALID_ARG
    assert lib.hbsg_gemm(0, 0, 4, 8, 16, fake, 16, fake, 4, fake, 8, 0, None, 0, None) == L.ERR_INVALID_ARG
    # Black-Scholes: negative counts, null records, overlapping outputs
    assert lib.hbsg_blackscholes(fake, -1, None) == L.ERR_INVALID_ARG
    assert lib.hbsg_blackscholes(None, 4, None) == L.ERR_INVALID_ARG
    assert lib.hbsg_blackscholes(None, 0, None) == L.OK
    ins = [P(0x10000 + 0x1000 * i) for i in range(5)]
    assert lib.hbsg_blackscholes_arrays(*ins, P(0x20000), P(0x20000 + 16), 8, None) == \
        L.ERR_INVALID_ARG
    assert lib.hbsg_blackscholes_arrays(*ins, ins[2], P(0x30000), 8, None) == L.ERR_INVALID_ARG
    assert lib.hbsg_blackscholes_arrays(*ins, None, P(0x30000), 8, None) == L.ERR_INVALID_ARG
    assert lib.hbsg_blackscholes_arrays(*ins, P(0x20000), P(0x30000), -2, None) == \
        L.ERR_INVALID_ARG


def test_no_device_is_reported_not_crashed(L):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    fake = ctypes.c_void_p(0x10000)
    assert L.lib().hbsg_sgemm(fake, fake, fake, 16, 1, None) == L.ERR_NO_DEVICE
    assert L.lib().hbsg_blackscholes(fake, 4, None) == L.ERR_NO_DEVICE


def test_tile_table(L):
    from hb_hammerbench_b200 import tiles
    t = tiles()
    assert len(t) == L.lib().hbsg_num_tiles() >= 4
    for e in t:
        assert e["bm"] > 0 and e["bn"] > 0 and e["threads"] % 32 == 0
        assert e["smem_bytes"] <= 227 * 1024
    info = L.TileInfo()
    assert L.lib().hbsg_tile_describe(0, ctypes.byref(info)) == L.ERR_INVALID_ARG
    assert L.lib().hbsg_tile_describe(len(t) + 1, ctypes.byref(info)) == L.ERR_INVALID_ARG
