// FP32 SIMT throughput probe: the roof the FFMA SGEMM kernel is reported
// against, measured on the device it runs on instead of derived from the
// SM count and clock.
//
// Every thread runs kChains independent accumulator chains (no dependency
// between chains, none on memory), each step one fused multiply-add per lane
// (or one packed two-lane __ffma2_rn, two FMAs, when `packed`), for `iters`
// steps. The grid is kBlocksPerSm CTAs of 256 threads per SM, so every
// scheduler has several warps to issue from and the FMA latency is covered.
// The sums are folded into one float that is stored only when it equals a
// value the arithmetic never produces, so the compiler keeps the work and the
// kernel writes nothing in practice.
#include <cuda_runtime.h>

#include "internal.h"

namespace hbsg {

static constexpr int kPeakThreads = 256;
static constexpr int kBlocksPerSm = 4;
static constexpr int kChains = 8;

template <bool PACKED>
__global__ void __launch_bounds__(kPeakThreads) fp32_peak_kernel(int iters, float* sink) {
  const float t = 1.0f + 1e-7f * (float)(threadIdx.x & 7);
  const float2 a2 = make_float2(t, t);
  const float2 b2 = make_float2(-1e-7f, 1e-7f);
  float2 acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = make_float2((float)c, (float)(c + 1));
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      if constexpr (PACKED) {
        acc[c] = __ffma2_rn(acc[c], a2, b2);
      } else {
        acc[c].x = __fmaf_rn(acc[c].x, t, -1e-7f);
        acc[c].y = __fmaf_rn(acc[c].y, t, 1e-7f);
      }
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c].x + acc[c].y;
  if (s == -12345.678f) sink[0] = s;
}

}  // namespace hbsg

using namespace hbsg;

extern "C" int hbsg_fp32_peak_probe(int packed, int iters, float* sink, double* flops_out,
                                    hbsg_stream_t stream) {
  if (iters <= 0 || !sink || !flops_out) return HBSG_ERR_INVALID_ARG;
  const int sms = current_device_sms(nullptr);
  if (sms < 0) return HBSG_ERR_NO_DEVICE;
  const int grid = sms * kBlocksPerSm;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (packed) fp32_peak_kernel<true><<<grid, kPeakThreads, 0, st>>>(iters, sink);
  else fp32_peak_kernel<false><<<grid, kPeakThreads, 0, st>>>(iters, sink);
  if (cudaGetLastError() != cudaSuccess) return HBSG_ERR_LAUNCH;
  // 2 FMAs (one per float2 lane) of 2 flops per chain and step, both forms
  *flops_out = 4.0 * kChains * (double)iters * grid * kPeakThreads;
  return HBSG_OK;
}
