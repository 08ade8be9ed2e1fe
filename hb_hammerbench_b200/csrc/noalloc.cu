// Allocation-free entry point of the split-BF16 GEMM (hbsg_gemm_noalloc).
//
// Some callers cannot allocate device memory when they need a product: an
// application whose memory pool has already reserved (nearly) the whole GPU
// would see a workspace allocation fail or force its pool to give memory
// back, and a latency-critical loop cannot afford cudaMalloc/cudaFree, which
// may synchronise the device. For them the split parts go into the fixed
// array below instead of a caller-provided workspace.
//
// The array is HBSG_NOALLOC_SCRATCH_BYTES of device memory that every GPU
// which loads this library keeps until the process exits. Host code cannot
// use the array's name as a device address (on the host it names a host-side
// stand-in), so the device address is looked up once per device with
// cudaGetSymbolAddress while that device is current, on the first call made
// on it; that first call should happen before any stream capture begins.
// Every call on a device shares the array, so calls that can overlap on the
// GPU race on it. Nothing has to be cleared between calls: the split pass
// writes every scratch byte the product later reads (zero padding along K
// included) and clears the column-maximum words before it accumulates them.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

namespace hbsg {

static __device__ __align__(256) unsigned char g_noalloc_scratch[HBSG_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[kMaxDevices];

static int lookup_scratch(void** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return HBSG_ERR_CUDA;
  }
  *out = p;
  return HBSG_OK;
}

// Device address of the scratch array on the current device: looked up on the
// first call made on each device and kept for the life of the process. The
// cached address belongs to the device's primary context, so it does not
// survive cudaDeviceReset (the module is loaded again, possibly elsewhere);
// callers that reset a device must not use this entry point afterwards.
// Device ordinals beyond the table are looked up on every call.
static int noalloc_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return HBSG_ERR_NO_DEVICE;
  }
  if (dev >= kMaxDevices) return lookup_scratch(out);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    const int st = lookup_scratch(&g_noalloc_addr[dev]);
    if (st != HBSG_OK) return st;
  }
  *out = g_noalloc_addr[dev];
  return HBSG_OK;
}

}  // namespace hbsg

extern "C" int hbsg_gemm_noalloc(int trans_a, int trans_b, int m, int n, int k, const float* a,
                                 int64_t lda, const float* b, int64_t ldb, float* c, int64_t ldc,
                                 int variant, hbsg_stream_t stream) {
  if (variant == HBSG_FFMA) return HBSG_ERR_UNSUPPORTED;
  if (variant < HBSG_BF16X3 || variant > HBSG_BF16X6_SCALED) return HBSG_ERR_UNSUPPORTED;
  if (m < 0 || n < 0 || k < 0) return HBSG_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return HBSG_OK;
  // A fused-split schedule of an unscaled form may need no scratch at all
  // (need == 0); argument and device errors are reported by hbsg_gemm_ex.
  const size_t need = hbsg::gemm_workspace_exact(trans_a, trans_b, m, n, k, a, lda, b, ldb, variant,
                                                 nullptr);
  if (need > HBSG_NOALLOC_SCRATCH_BYTES) return HBSG_ERR_WORKSPACE;
  void* scratch = nullptr;
  const int s2 = hbsg::noalloc_scratch(&scratch);
  if (s2 != HBSG_OK) return s2;
  return hbsg_gemm_ex(trans_a, trans_b, m, n, k, a, lda, b, ldb, c, ldc, variant, nullptr, scratch,
                      HBSG_NOALLOC_SCRATCH_BYTES, stream);
}
