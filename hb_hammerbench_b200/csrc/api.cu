// C-ABI layer: argument validation, variant dispatch, status codes.
// Entry points are declared (with the reference interfaces they replace) in
// include/hbsg.h.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

namespace hbsg {

static std::mutex g_dev_mu;
static int g_sms[64];
static int g_ok[64];  // 0 unknown, 1 sm_100, -1 other

int current_device_sms(int* device_out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return -1;
  }
  if (device_out) *device_out = dev;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (g_ok[dev] == 0) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    g_ok[dev] = (prop.major == 10 && prop.minor == 0) ? 1 : -1;
    g_sms[dev] = prop.multiProcessorCount;
  }
  return g_ok[dev] == 1 ? g_sms[dev] : -1;
}

bool set_smem_once(const void* func, int bytes, uint32_t* device_mask) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 32) return false;
  if (__atomic_load_n(device_mask, __ATOMIC_ACQUIRE) & (1u << dev)) return true;
  if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
    return false;
  __atomic_fetch_or(device_mask, 1u << dev, __ATOMIC_ACQ_REL);
  return true;
}

static int status_from(cudaError_t e) {
  if (e == cudaSuccess) return HBSG_OK;
  cudaGetLastError();
  if (e == cudaErrorInvalidConfiguration || e == cudaErrorLaunchOutOfResources ||
      e == cudaErrorInvalidValue)
    return HBSG_ERR_LAUNCH;
  return HBSG_ERR_CUDA;
}

static bool variant_valid(int v) { return v >= HBSG_FFMA && v <= HBSG_BF16X6_SCALED; }

// Core dispatcher for one (possibly batched) GEMM.
static int gemm_dispatch(int trans_a, int trans_b, int M, int N, int K, const float* A, long lda,
                         long strideA, const float* B, long ldb, long strideB, float* C, long ldc,
                         long strideC, int batch, int variant, const hbsg_config* cfg, void* ws,
                         size_t ws_bytes, cudaStream_t st) {
  if (M < 0 || N < 0 || K < 0 || batch < 0) return HBSG_ERR_INVALID_ARG;
  if (!variant_valid(variant)) return HBSG_ERR_UNSUPPORTED;
  if (M == 0 || N == 0 || batch == 0) return HBSG_OK;
  if (!C) return HBSG_ERR_INVALID_ARG;
  if (K > 0 && (!A || !B)) return HBSG_ERR_INVALID_ARG;
  if (trans_a || trans_b) return HBSG_ERR_UNSUPPORTED;  // row-major only in this build
  if (lda < (K > 0 ? K : 1) || ldb < N || ldc < N) return HBSG_ERR_INVALID_ARG;
  int dev = 0;
  const int sms = current_device_sms(&dev);
  if (sms < 0) return HBSG_ERR_NO_DEVICE;
  if (variant != HBSG_FFMA) return HBSG_ERR_UNSUPPORTED;

  int tile = cfg && cfg->tile > 0 ? cfg->tile - 1 : -1;
  if (tile >= ffma_num_tiles()) return HBSG_ERR_UNSUPPORTED;
  if (tile < 0) tile = ffma_pick_tile(M, N, K, batch, sms);
  int splits = cfg && cfg->split_k > 1 ? cfg->split_k : 1;
  if (splits > 1 && K == 0) splits = 1;
  const size_t need = ffma_workspace_bytes(M, N, batch, splits);
  if (need > 0 && (!ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(ws) & 255)))
    return HBSG_ERR_WORKSPACE;

  FfmaParams p{};
  p.A = A;
  p.B = B;
  p.C = C;
  p.partial = static_cast<float*>(ws);
  p.lda = lda;
  p.ldb = ldb;
  p.ldc = ldc;
  p.strideA = strideA;
  p.strideB = strideB;
  p.strideC = strideC;
  p.M = M;
  p.N = N;
  p.K = K;
  p.splits = splits;
  p.raster = cfg && cfg->raster_group > 0 ? cfg->raster_group : 8;
  return status_from(ffma_launch(tile, p, batch, st));
}

}  // namespace hbsg

using namespace hbsg;

extern "C" {

int hbsg_sgemm(const float* mat1, const float* mat2, float* result, int n, int niter,
               hbsg_stream_t stream) {
  if (n < 0 || niter < 0) return HBSG_ERR_INVALID_ARG;
  if (n > 0 && niter > 0 && (!mat1 || !mat2 || !result)) return HBSG_ERR_INVALID_ARG;
  const long nn = (long)n * n;
  return gemm_dispatch(0, 0, n, n, n, mat1, n, nn, mat2, n, nn, result, n, nn, niter, HBSG_FFMA,
                       nullptr, nullptr, 0, reinterpret_cast<cudaStream_t>(stream));
}

int hbsg_sgemm_variant(const float* mat1, const float* mat2, float* result, int n, int niter,
                       int variant, void* workspace, size_t workspace_bytes,
                       hbsg_stream_t stream) {
  if (n < 0 || niter < 0) return HBSG_ERR_INVALID_ARG;
  if (n > 0 && niter > 0 && (!mat1 || !mat2 || !result)) return HBSG_ERR_INVALID_ARG;
  const long nn = (long)n * n;
  return gemm_dispatch(0, 0, n, n, n, mat1, n, nn, mat2, n, nn, result, n, nn, niter, variant,
                       nullptr, workspace, workspace_bytes,
                       reinterpret_cast<cudaStream_t>(stream));
}

size_t hbsg_sgemm_workspace_size(int n, int niter, int variant) {
  (void)n;
  (void)niter;
  (void)variant;
  return 0;
}

int hbsg_gemm(int trans_a, int trans_b, int m, int n, int k, const float* a, int64_t lda,
              const float* b, int64_t ldb, float* c, int64_t ldc, int variant, void* workspace,
              size_t workspace_bytes, hbsg_stream_t stream) {
  return gemm_dispatch(trans_a, trans_b, m, n, k, a, lda, 0, b, ldb, 0, c, ldc, 0, 1, variant,
                       nullptr, workspace, workspace_bytes,
                       reinterpret_cast<cudaStream_t>(stream));
}

int hbsg_gemm_ex(int trans_a, int trans_b, int m, int n, int k, const float* a, int64_t lda,
                 const float* b, int64_t ldb, float* c, int64_t ldc, int variant,
                 const hbsg_config* cfg, void* workspace, size_t workspace_bytes,
                 hbsg_stream_t stream) {
  return gemm_dispatch(trans_a, trans_b, m, n, k, a, lda, 0, b, ldb, 0, c, ldc, 0, 1, variant, cfg,
                       workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}

size_t hbsg_gemm_workspace_size(int m, int n, int k, int variant, const hbsg_config* cfg) {
  (void)k;
  if (m <= 0 || n <= 0 || !variant_valid(variant)) return 0;
  const int splits = cfg && cfg->split_k > 1 ? cfg->split_k : 1;
  return ffma_workspace_bytes(m, n, 1, splits);
}

int hbsg_num_tiles(void) { return ffma_num_tiles(); }

int hbsg_tile_describe(int tile, hbsg_tile_info* out) {
  if (!out) return HBSG_ERR_INVALID_ARG;
  if (tile < 1 || tile > ffma_num_tiles()) return HBSG_ERR_INVALID_ARG;
  return ffma_tile_info(tile - 1, out) ? HBSG_OK : HBSG_ERR_INVALID_ARG;
}

const char* hbsg_strerror(int status) {
  switch (status) {
    case HBSG_OK: return "success";
    case HBSG_ERR_INVALID_ARG: return "invalid argument";
    case HBSG_ERR_UNSUPPORTED: return "unsupported variant, configuration or layout";
    case HBSG_ERR_WORKSPACE: return "workspace missing, misaligned or too small";
    case HBSG_ERR_LAUNCH: return "kernel launch failed";
    case HBSG_ERR_DEVICE_TIMEOUT: return "a bounded device-side wait expired";
    case HBSG_ERR_NO_DEVICE: return "no sm_100 device is current";
    case HBSG_ERR_CUDA: return "CUDA runtime error";
    default: return "unknown status";
  }
}

int hbsg_check_device(hbsg_stream_t stream) {
  cudaError_t e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return status_from(e);
  return HBSG_OK;
}

int hbsg_version(void) { return 100; }

}  // extern "C"
