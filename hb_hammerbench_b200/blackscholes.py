"""Host-side interface of the Black-Scholes kernel (the suite's
apps/blackscholes benchmark) over libhbsg.so.

Mirrors the benchmark's host flow (apps/blackscholes/main.cpp:50-141): an
array of option records (OptionData, option_data.hpp:2-13: s, strike, r, v,
t, call, put, unused as float32) is priced in place on the device, one call
per launch of `kernel(data, num_option, pod)`.

  price(records)              (n, 8) float32 CUDA tensor, call and put set in place
  price_arrays(s, k, r, v, t) separate float32 CUDA arrays -> (call, put)
  option_records(n, seed)     seeded synthetic records (numpy)

Synthetic records stand in for the benchmark's input file (in_10M.txt, the
PARSEC option set). Their ranges are that file's: spot 40-100, spot / strike
0.82-1.22 (one record in eight at the money, spot == strike), rate
0.0275-0.1, volatility 0.05-0.65, maturity 0.05-1 year.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import check, lib
from .sgemm import _check_f32_cuda, _ptr, _stream

FIELDS = ("s", "strike", "r", "v", "t", "call", "put", "unused")
RECORD_FLOATS = 8


def option_records(n: int, seed: int = 0) -> np.ndarray:
    """(n, 8) float32 option records with call, put and unused zero."""
    rng = np.random.Generator(np.random.PCG64(seed))
    rec = np.zeros((n, RECORD_FLOATS), np.float32)
    s = rng.uniform(40.0, 100.0, n).astype(np.float32)
    ratio = rng.uniform(0.82, 1.22, n)
    strike = (s / ratio).astype(np.float32)
    atm = rng.integers(0, 8, n) == 0
    strike[atm] = s[atm]
    rec[:, 0] = s
    rec[:, 1] = strike
    rec[:, 2] = rng.uniform(0.0275, 0.1, n).astype(np.float32)
    rec[:, 3] = rng.uniform(0.05, 0.65, n).astype(np.float32)
    rec[:, 4] = rng.uniform(0.05, 1.0, n).astype(np.float32)
    return rec


def price(records: torch.Tensor) -> torch.Tensor:
    """Price (n, 8) float32 option records on their CUDA device in place
    (hbsg_blackscholes); returns `records`."""
    _check_f32_cuda("records", records)
    if records.dim() != 2 or records.shape[1] != RECORD_FLOATS or not records.is_contiguous():
        raise ValueError("records must be a contiguous (n, 8) float32 tensor")
    with torch.cuda.device(records.device):
        check(lib().hbsg_blackscholes(_ptr(records), records.shape[0], _stream()),
              "hbsg_blackscholes")
    return records


def price_arrays(s: torch.Tensor, strike: torch.Tensor, r: torch.Tensor, v: torch.Tensor,
                 t: torch.Tensor, call: torch.Tensor | None = None,
                 put: torch.Tensor | None = None):
    """Price options held as separate float32 CUDA arrays
    (hbsg_blackscholes_arrays); returns (call, put)."""
    ins = (s, strike, r, v, t)
    n = s.numel()
    for name, x in zip(FIELDS, ins):
        _check_f32_cuda(name, x)
        if not x.is_contiguous() or x.numel() != n:
            raise ValueError(f"{name} must be a contiguous array of {n} floats")
    call = torch.empty_like(s) if call is None else call
    put = torch.empty_like(s) if put is None else put
    for name, x in (("call", call), ("put", put)):
        _check_f32_cuda(name, x)
        if not x.is_contiguous() or x.numel() != n:
            raise ValueError(f"{name} must be a contiguous array of {n} floats")
    with torch.cuda.device(s.device):
        check(lib().hbsg_blackscholes_arrays(*[_ptr(x) for x in ins], _ptr(call), _ptr(put), n,
                                             _stream()),
              "hbsg_blackscholes_arrays")
    return call, put
