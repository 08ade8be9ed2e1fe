"""B200 (sm_100a) SGEMM hot path of the HammerBench sgemm benchmark.

The kernels live in libhbsg.so behind the C ABI of include/hbsg.h; this
package is the host-side interface over it (see sgemm.py).
"""
from ._lib import (BF16X3, BF16X3_SCALED, BF16X6, BF16X6_SCALED, FFMA, VARIANTS,  # noqa: F401
                   HbsgError, LIB_PATH, lib)
from .sgemm import (GroupedPlan, fp32_peak, gemm, gemm_grouped,  # noqa: F401
                    gemm_workspace_size, jacobi, resolve_config, sgemm, sgemm_workspace_size,
                    split_layout, tiles)
from . import blackscholes  # noqa: F401

__version__ = "1.0"
