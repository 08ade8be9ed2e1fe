// Black-Scholes European option pricing for sm_100a: the suite's
// apps/blackscholes benchmark on the same host interface as the SGEMM path.
//
// Reference: the device kernel `kernel(OptionData* data, int num_option,
// int pod_id)` (apps/blackscholes/kernel.cpp:27-113) prices each option
// record in place with BlkSchlsEqEuroNoDiv_kernel (bs_kernel.hpp:163-198);
// the testbench checks call and put against the host BlkSchlsEqEuroNoDiv
// (bs.hpp:60-125) by the sum of squared differences <= 0.01
// (main.cpp:119-141).
//
// Arithmetic: the device kernel's own approximations, each step the same IEEE
// operation, so results are bit-identical to that kernel:
//   - ln(s / strike) by its 5-term Taylor series around 1 in Horner form
//     (bs_kernel.hpp:33-49), 0 when s == strike;
//   - exp of a non-positive argument by whole steps of e^-1, one optional
//     e^-0.5 step and a 5-term Taylor polynomial of the remainder, 0 below -15
//     (bs_kernel.hpp:52-91);
//   - the cumulative normal by Hull's polynomial (bs_kernel.hpp:95-160);
// each `fmadd.s` / `fnmsub.s` of the reference is one fused multiply-add
// (__fmaf_rn); every other product, sum, quotient and square root is rounded
// on its own (the explicit __f*_rn intrinsics keep nvcc from contracting
// them); no library math function is called.
//
// B200 form: pricing reads 5 floats and writes 2 per option, a few hundred
// instructions, so the kernel is HBM-bound on both layouts:
//   - records (the reference's OptionData, 8 floats = 32 bytes, call and put
//     updated in place): one thread per record loads it as two 16-byte
//     vectors and stores both back with call and put replaced, so each
//     record moves as one 32-byte sector each way (64 bytes per option);
//   - separate arrays (s, strike, r, v, t in; call, put out): 28 bytes per
//     option, four options per thread as 16-byte vectors.
// Loads and stores use the streaming (evict-first) cache hint: nothing is
// reused. Grid-stride loops over one wave of resident CTAs.
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"

namespace hbsg {

static constexpr int kBsThreads = 256;
static constexpr int kBsCtasPerSm = 8;

// my_logf (bs_kernel.hpp:33-49)
HBSG_DEV float bs_logf(float x) {
  const float diff = __fsub_rn(x, 1.0f);
  float r = __fmaf_rn(diff, 0.20000000f, -0.25000000f);
  r = __fmaf_rn(r, diff, 0.33333333f);
  r = __fmaf_rn(r, diff, -0.50000000f);
  r = __fmaf_rn(r, diff, 1.00000000f);
  return __fmul_rn(r, diff);
}

// expf_0 (bs_kernel.hpp:52-65)
HBSG_DEV float bs_exp0(float x) {
  float r = __fmaf_rn(x, 0.0083333338f, 0.04166667f);
  r = __fmaf_rn(r, x, 0.16666666f);
  r = __fmaf_rn(r, x, 0.5f);
  r = __fmaf_rn(r, x, 1.0f);
  return __fmaf_rn(r, x, 1.0f);
}

// fast_expf (bs_kernel.hpp:69-91), x <= 0, without its loop. The loop
// multiplies part1 by e^-1 and adds 1 to x while x <= -1. For -15 <= x <= -1
// every x + 1 is exact (1 is a multiple of x's ulp and |x + 1| < |x|), so the
// loop runs n = floor(-x) times, leaves x + n (exact, for the same reason) and
// part1 = the n-fold rounded product, which `pow_tab` (lane k of the warp
// holds the k-fold product, bs_pow_table) supplies by a shuffle: bit for bit
// the loop's result. Every lane of the warp must call this together.
HBSG_DEV float bs_fast_expf(float x, float pow_tab) {
  const bool zero = x < -15.0f;
  const int n = (x <= -1.0f && !zero) ? (int)floorf(-x) : 0;  // 0..15
  float part1 = __shfl_sync(0xffffffffu, pow_tab, n);
  x = __fadd_rn(x, (float)n);
  if (x <= -0.5f) {
    part1 = __fmul_rn(part1, 0.60653066f);
    x = __fadd_rn(x, 0.5f);
  }
  return zero ? 0.0f : __fmul_rn(part1, bs_exp0(x));
}

// Lane k (< 16) of a warp: e^-1 multiplied into 1.0f k times, each product
// rounded, as fast_expf's loop forms it.
HBSG_DEV float bs_pow_table() {
  const int k = threadIdx.x & 15;
  float p = 1.0f;
  for (int i = 0; i < k; ++i) p = __fmul_rn(p, 0.36787945f);
  return p;
}

// one lane of dual_CNDF (bs_kernel.hpp:95-160); 1 / (1 + 0.2316419 |x|) as
// the correctly rounded reciprocal, the same value as the reference's divide
HBSG_DEV float bs_cndf(float x, float pow_tab) {
  const bool neg = x < 0.0f;
  const float xa = fabsf(x);
  const float e = __fmul_rn(bs_fast_expf(__fmul_rn(__fmul_rn(-0.5f, xa), xa), pow_tab),
                            0.39894228040143270286f);
  const float k = __frcp_rn(__fmaf_rn(0.2316419f, xa, 1.0f));
  float f = __fmaf_rn(k, 1.330274429f, -1.821255978f);
  f = __fmaf_rn(f, k, 1.781477937f);
  f = __fmaf_rn(f, k, -0.356563782f);
  f = __fmaf_rn(f, k, 0.319381530f);
  f = __fmul_rn(f, k);
  const float out = __fmaf_rn(-f, e, 1.0f);  // fnmsub.s: -(f * e) + 1
  return neg ? __fsub_rn(1.0f, out) : out;
}

// BlkSchlsEqEuroNoDiv_kernel (bs_kernel.hpp:163-198)
HBSG_DEV void bs_price(float s, float strike, float r, float v, float t, float& call,
                       float& put, float pow_tab) {
  const float sqrt_t = __fsqrt_rn(t);
  const float logv = (s == strike) ? 0.0f : bs_logf(__fdiv_rn(s, strike));
  float d1 = __fmaf_rn(__fmul_rn(v, v), 0.5f, r);
  d1 = __fmaf_rn(d1, t, logv);
  const float den = __fmul_rn(v, sqrt_t);
  d1 = __fdiv_rn(d1, den);
  const float d2 = __fsub_rn(d1, den);
  const float c1 = bs_cndf(d1, pow_tab);
  const float c2 = bs_cndf(d2, pow_tab);
  const float fv = __fmul_rn(strike, bs_exp0(__fmul_rn(-r, t)));
  call = __fsub_rn(__fmul_rn(s, c1), __fmul_rn(fv, c2));
  put = __fsub_rn(__fmul_rn(fv, __fsub_rn(1.0f, c2)), __fmul_rn(s, __fsub_rn(1.0f, c1)));
}

// The grid-stride loops below step whole warps (the loop bound depends on the
// warp's first index only), because bs_fast_expf shuffles across the warp;
// lanes past the end price a dummy option and store nothing.

// Records in place, 16-byte aligned: two records per thread per step, all
// four loads issued before the arithmetic; the whole 32-byte record is stored
// back (its input fields unchanged), so each record's sector is written whole
// and never needs a fill from DRAM after the streaming load evicted it.
__global__ void __launch_bounds__(kBsThreads) bs_records_kernel(float* __restrict__ data,
                                                                long n) {
  float4* rec = reinterpret_cast<float4*>(data);
  const float pow_tab = bs_pow_table();
  const long stride = (long)gridDim.x * kBsThreads;
  const long lane = threadIdx.x & 31;
  const float4 dummy_a = make_float4(1.f, 1.f, 0.f, 1.f), dummy_b = make_float4(1.f, 0.f, 0.f, 0.f);
  for (long base = (long)blockIdx.x * kBsThreads + (threadIdx.x & ~31); base < n;
       base += 2 * stride) {
    const long i = base + lane, j = i + stride;
    const bool has0 = i < n, has1 = j < n;
    float4 a0 = dummy_a, b0 = dummy_b, a1 = dummy_a, b1 = dummy_b;
    if (has0) {
      a0 = __ldcs(rec + 2 * i);
      b0 = __ldcs(rec + 2 * i + 1);
    }
    if (has1) {
      a1 = __ldcs(rec + 2 * j);
      b1 = __ldcs(rec + 2 * j + 1);
    }
    bs_price(a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, pow_tab);
    bs_price(a1.x, a1.y, a1.z, a1.w, b1.x, b1.y, b1.z, pow_tab);
    if (has0) {
      __stcs(rec + 2 * i, a0);
      __stcs(rec + 2 * i + 1, b0);
    }
    if (has1) {
      __stcs(rec + 2 * j, a1);
      __stcs(rec + 2 * j + 1, b1);
    }
  }
}

// Records at any 4-byte alignment: scalar loads, call and put stored alone.
__global__ void __launch_bounds__(kBsThreads) bs_records_scalar_kernel(float* __restrict__ data,
                                                                       long n) {
  const float pow_tab = bs_pow_table();
  const long stride = (long)gridDim.x * kBsThreads;
  for (long base = (long)blockIdx.x * kBsThreads + (threadIdx.x & ~31); base < n;
       base += stride) {
    const long i = base + (threadIdx.x & 31);
    const bool has = i < n;
    float* o = data + 8 * (has ? i : 0);
    float call, put;
    bs_price(has ? o[0] : 1.f, has ? o[1] : 1.f, has ? o[2] : 0.f, has ? o[3] : 1.f,
             has ? o[4] : 1.f, call, put, pow_tab);
    if (has) {
      o[5] = call;
      o[6] = put;
    }
  }
}

// Separate arrays. VEC: all seven arrays 16-byte aligned, four options per
// thread per step; the last n % 4 options (and every option without VEC) are
// priced one per thread.
template <bool VEC>
__global__ void __launch_bounds__(kBsThreads)
    bs_arrays_kernel(const float* __restrict__ s, const float* __restrict__ strike,
                     const float* __restrict__ r, const float* __restrict__ v,
                     const float* __restrict__ t, float* __restrict__ call,
                     float* __restrict__ put, long n) {
  const float pow_tab = bs_pow_table();
  const long stride = (long)gridDim.x * kBsThreads;
  const long wbase = (long)blockIdx.x * kBsThreads + (threadIdx.x & ~31);
  const long lane = threadIdx.x & 31;
  long done = 0;
  if constexpr (VEC) {
    const long n4 = n / 4;
    const float4 one = make_float4(1.f, 1.f, 1.f, 1.f);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (long base = wbase; base < n4; base += stride) {
      const long q = base + lane;
      const bool has = q < n4;
      float4 S = one, K = one, R = zero, V = one, T = one;
      if (has) {
        S = __ldcs(reinterpret_cast<const float4*>(s) + q);
        K = __ldcs(reinterpret_cast<const float4*>(strike) + q);
        R = __ldcs(reinterpret_cast<const float4*>(r) + q);
        V = __ldcs(reinterpret_cast<const float4*>(v) + q);
        T = __ldcs(reinterpret_cast<const float4*>(t) + q);
      }
      float4 C, P;
      bs_price(S.x, K.x, R.x, V.x, T.x, C.x, P.x, pow_tab);
      bs_price(S.y, K.y, R.y, V.y, T.y, C.y, P.y, pow_tab);
      bs_price(S.z, K.z, R.z, V.z, T.z, C.z, P.z, pow_tab);
      bs_price(S.w, K.w, R.w, V.w, T.w, C.w, P.w, pow_tab);
      if (has) {
        __stcs(reinterpret_cast<float4*>(call) + q, C);
        __stcs(reinterpret_cast<float4*>(put) + q, P);
      }
    }
    done = n4 * 4;
  }
  for (long base = done + wbase; base < n; base += stride) {
    const long i = base + lane;
    const bool has = i < n;
    const long ii = has ? i : n - 1;  // lanes past the end read the last option
    float c, p;
    bs_price(__ldcs(s + ii), __ldcs(strike + ii), __ldcs(r + ii), __ldcs(v + ii),
             __ldcs(t + ii), c, p, pow_tab);
    if (has) {
      __stcs(call + i, c);
      __stcs(put + i, p);
    }
  }
}

// One wave of resident CTAs (the occupancy of the kernel, looked up once per
// kernel; at most kBsCtasPerSm per SM), fewer when the work is smaller: the
// grid-stride loops then give every CTA the same share.
static int bs_grid(const void* kernel, int* cache, long work, int sms) {
  int per_sm = __atomic_load_n(cache, __ATOMIC_ACQUIRE);
  if (per_sm <= 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBsThreads, 0) !=
            cudaSuccess ||
        per_sm <= 0) {
      cudaGetLastError();
      per_sm = 1;
    }
    per_sm = per_sm < kBsCtasPerSm ? per_sm : kBsCtasPerSm;
    __atomic_store_n(cache, per_sm, __ATOMIC_RELEASE);
  }
  const long want = (work + kBsThreads - 1) / kBsThreads;
  const long cap = (long)sms * per_sm;
  return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

static int g_occ_records = 0, g_occ_scalar = 0, g_occ_arrays_vec = 0, g_occ_arrays = 0;

static bool overlaps(const void* a, long abytes, const void* b, long bbytes) {
  const char* x = static_cast<const char*>(a);
  const char* y = static_cast<const char*>(b);
  return x < y + bbytes && y < x + abytes;
}

}  // namespace hbsg

using namespace hbsg;

extern "C" int hbsg_blackscholes(hbsg_option* options, int64_t num_option, hbsg_stream_t stream) {
  if (num_option < 0) return HBSG_ERR_INVALID_ARG;
  if (num_option == 0) return HBSG_OK;
  if (!options) return HBSG_ERR_INVALID_ARG;
  const int sms = current_device_sms(nullptr);
  if (sms < 0) return HBSG_ERR_NO_DEVICE;
  float* data = reinterpret_cast<float*>(options);
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if ((reinterpret_cast<uintptr_t>(data) & 15) == 0)
    bs_records_kernel<<<bs_grid((const void*)bs_records_kernel, &g_occ_records,
                                (num_option + 1) / 2, sms),
                        kBsThreads, 0, st>>>(data, num_option);
  else
    bs_records_scalar_kernel<<<bs_grid((const void*)bs_records_scalar_kernel, &g_occ_scalar,
                                       num_option, sms),
                               kBsThreads, 0, st>>>(data, num_option);
  return cudaGetLastError() == cudaSuccess ? HBSG_OK : HBSG_ERR_LAUNCH;
}

extern "C" int hbsg_blackscholes_arrays(const float* s, const float* strike, const float* r,
                                        const float* v, const float* t, float* call, float* put,
                                        int64_t n, hbsg_stream_t stream) {
  if (n < 0) return HBSG_ERR_INVALID_ARG;
  if (n == 0) return HBSG_OK;
  if (!s || !strike || !r || !v || !t || !call || !put) return HBSG_ERR_INVALID_ARG;
  const long nb = (long)n * 4;
  const float* ins[5] = {s, strike, r, v, t};
  if (overlaps(call, nb, put, nb)) return HBSG_ERR_INVALID_ARG;
  for (const float* in : ins)
    if (overlaps(in, nb, call, nb) || overlaps(in, nb, put, nb)) return HBSG_ERR_INVALID_ARG;
  const int sms = current_device_sms(nullptr);
  if (sms < 0) return HBSG_ERR_NO_DEVICE;
  uintptr_t bits = reinterpret_cast<uintptr_t>(call) | reinterpret_cast<uintptr_t>(put);
  for (const float* in : ins) bits |= reinterpret_cast<uintptr_t>(in);
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if ((bits & 15) == 0)
    bs_arrays_kernel<true><<<bs_grid((const void*)bs_arrays_kernel<true>, &g_occ_arrays_vec,
                                     (n + 3) / 4, sms),
                             kBsThreads, 0, st>>>(s, strike, r, v, t, call, put, n);
  else
    bs_arrays_kernel<false><<<bs_grid((const void*)bs_arrays_kernel<false>, &g_occ_arrays, n,
                                      sms),
                              kBsThreads, 0, st>>>(s, strike, r, v, t, call, put, n);
  return cudaGetLastError() == cudaSuccess ? HBSG_OK : HBSG_ERR_LAUNCH;
}
