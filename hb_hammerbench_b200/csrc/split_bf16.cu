// Split pre-pass for the split-BF16 tensor-core SGEMM (sm_100a).
//
// Every FP32 operand element x becomes BF16 parts (round to nearest even):
//   x' = x * 2^-e            (e = 0, or the row/column exponent when scaled)
//   hi  = bf16(x'),  r1 = x' - hi          (exact in FP32)
//   mid = bf16(r1),  r2 = r1 - mid         (exact in FP32)
//   lo  = bf16(r2)                          (3-part form only)
// With three parts hi + mid + lo == x' exactly for every normal FP32 value.
//
// Output layout (the K-major operand layout the tensor-core kernel's TMA reads):
//   Ap[p][m][k]  p < parts, m < M, k < Kp   (Kp = K rounded up to 32, zero-filled)
//   Bp[p][n][k]  B transposed: the K x N row-major input becomes N rows of Kp
// The scaled forms first reduce max|x| per row of A / per column of B into
// FP32 bit patterns (non-negative floats order like their bit patterns, so an
// integer atomicMax is an exact, order-independent max), then derive
// e = frexp exponent of that max: the row's largest |x'| lies in [0.5, 1).
#include <cuda_bf16.h>

#include "common.cuh"
#include "internal.h"

namespace hbsg {

HBSG_DEV int exp_from_maxbits(uint32_t bits) {
  const float mx = __uint_as_float(bits);
  if (!(mx > 0.0f) || !isfinite(mx)) return 0;
  int e;
  frexpf(mx, &e);
  return e;
}

template <int P>
HBSG_DEV void split_value(float x, int e, __nv_bfloat16* out) {
  if (e != 0) x = ldexpf(x, -e);
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h);
  const __nv_bfloat16 m = __float2bfloat16_rn(r1);
  out[0] = h;
  out[1] = m;
  if constexpr (P == 3) {
    const float r2 = r1 - __bfloat162float(m);
    out[2] = __float2bfloat16_rn(r2);
  }
}

// max|A[m][k]| over k per row, one warp per row.
__global__ void row_maxabs_kernel(const float* __restrict__ A, long lda, int M, int K,
                                  uint32_t* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= M) return;
  const float* row = A + (long)warp * lda;
  float mx = 0.0f;
  for (int k = lane; k < K; k += 32) {
    const float a = fabsf(row[k]);
    if (isfinite(a)) mx = fmaxf(mx, a);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) out[warp] = __float_as_uint(mx);
}

// max|B[k][n]| over k per column: threads along n, blocks along k slices.
__global__ void col_maxabs_kernel(const float* __restrict__ B, long ldb, int K, int N,
                                  int k_per_block, uint32_t* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int k0 = blockIdx.y * k_per_block;
  const int k1 = min(K, k0 + k_per_block);
  float mx = 0.0f;
  for (int k = k0; k < k1; ++k) {
    const float b = fabsf(B[(long)k * ldb + n]);
    if (isfinite(b)) mx = fmaxf(mx, b);
  }
  if (mx > 0.0f) atomicMax(out + n, __float_as_uint(mx));
}

// A (M x K, row stride lda) -> Ap[p][m][0..Kp). One thread per 8 consecutive k.
template <int P, bool SCALED>
__global__ void split_a_kernel(const float* __restrict__ A, long lda, int M, int K, int Kp,
                               __nv_bfloat16* __restrict__ Ap, const uint32_t* __restrict__ rowmax) {
  const long groups_per_row = Kp / 8;
  const long total = (long)M * groups_per_row;
  const long plane = (long)M * Kp;
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < total;
       g += (long)gridDim.x * blockDim.x) {
    const int m = (int)(g / groups_per_row);
    const int k0 = (int)(g - (long)m * groups_per_row) * 8;
    const int e = SCALED ? exp_from_maxbits(rowmax[m]) : 0;
    const float* src = A + (long)m * lda + k0;
    float v[8];
    if (k0 + 8 <= K && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
      const float4 x0 = *reinterpret_cast<const float4*>(src);
      const float4 x1 = *reinterpret_cast<const float4*>(src + 4);
      v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w;
      v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = (k0 + i < K) ? src[i] : 0.0f;
    }
    __align__(16) __nv_bfloat16 parts[P][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      __nv_bfloat16 o[3];
      split_value<P>(v[i], e, o);
#pragma unroll
      for (int p = 0; p < P; ++p) parts[p][i] = o[p];
    }
    __nv_bfloat16* dst = Ap + (long)m * Kp + k0;
#pragma unroll
    for (int p = 0; p < P; ++p)
      *reinterpret_cast<uint4*>(dst + p * plane) = *reinterpret_cast<const uint4*>(parts[p]);
  }
}

// B (K x N, row stride ldb) -> Bp[p][n][0..Kp) through a 64 x 64 shared tile.
template <int P, bool SCALED>
__global__ void __launch_bounds__(256) split_b_kernel(const float* __restrict__ B, long ldb, int K,
                                                      int N, int Kp, __nv_bfloat16* __restrict__ Bp,
                                                      const uint32_t* __restrict__ colmax) {
  __shared__ float tile[64][65];
  const int k0 = blockIdx.y * 64;
  const int n0 = blockIdx.x * 64;
  const int tid = threadIdx.x;
  // load: 64 rows (k) x 64 columns (n), coalesced along n
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int idx = tid + i * 256;
    const int r = idx >> 6;
    const int c = idx & 63;
    const int k = k0 + r;
    const int n = n0 + c;
    tile[r][c] = (k < K && n < N) ? B[(long)k * ldb + n] : 0.0f;
  }
  __syncthreads();
  const long plane = (long)N * Kp;
  // store: 8 threads per output row n, each 8 consecutive k
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    const int j = pass * 32 + (tid >> 3);  // n offset
    const int kk = (tid & 7) * 8;          // k offset
    const int n = n0 + j;
    if (n >= N || k0 + kk >= Kp) continue;
    const int e = SCALED ? exp_from_maxbits(colmax[n]) : 0;
    __align__(16) __nv_bfloat16 parts[P][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      __nv_bfloat16 o[3];
      split_value<P>(tile[kk + i][j], e, o);
#pragma unroll
      for (int p = 0; p < P; ++p) parts[p][i] = o[p];
    }
    __nv_bfloat16* dst = Bp + (long)n * Kp + k0 + kk;
#pragma unroll
    for (int p = 0; p < P; ++p)
      *reinterpret_cast<uint4*>(dst + p * plane) = *reinterpret_cast<const uint4*>(parts[p]);
  }
}

static int grid_for(long work, int per_block, int sms) {
  long b = (work + per_block - 1) / per_block;
  const long cap = (long)sms * 8;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

cudaError_t split_operand_a(const float* A, long lda, int M, int K, int Kp, int parts, bool scaled,
                            void* Ap, uint32_t* rowmax, int sms, cudaStream_t st) {
  if (scaled) {
    row_maxabs_kernel<<<(M + 7) / 8, 256, 0, st>>>(A, lda, M, K, rowmax);
  }
  const long work = (long)M * (Kp / 8);
  const int grid = grid_for(work, 256, sms);
  auto* ap = static_cast<__nv_bfloat16*>(Ap);
  if (parts == 3) {
    if (scaled) split_a_kernel<3, true><<<grid, 256, 0, st>>>(A, lda, M, K, Kp, ap, rowmax);
    else split_a_kernel<3, false><<<grid, 256, 0, st>>>(A, lda, M, K, Kp, ap, rowmax);
  } else {
    if (scaled) split_a_kernel<2, true><<<grid, 256, 0, st>>>(A, lda, M, K, Kp, ap, rowmax);
    else split_a_kernel<2, false><<<grid, 256, 0, st>>>(A, lda, M, K, Kp, ap, rowmax);
  }
  return cudaGetLastError();
}

cudaError_t split_operand_b(const float* B, long ldb, int K, int N, int Kp, int parts, bool scaled,
                            void* Bp, uint32_t* colmax, int sms, cudaStream_t st) {
  if (scaled) {
    cudaError_t e = cudaMemsetAsync(colmax, 0, sizeof(uint32_t) * N, st);
    if (e != cudaSuccess) return e;
    const int kpb = 256;
    dim3 g((N + 255) / 256, (K + kpb - 1) / kpb);
    if (K > 0) col_maxabs_kernel<<<g, 256, 0, st>>>(B, ldb, K, N, kpb, colmax);
  }
  dim3 grid((N + 63) / 64, (Kp + 63) / 64);
  auto* bp = static_cast<__nv_bfloat16*>(Bp);
  (void)sms;
  if (parts == 3) {
    if (scaled) split_b_kernel<3, true><<<grid, 256, 0, st>>>(B, ldb, K, N, Kp, bp, colmax);
    else split_b_kernel<3, false><<<grid, 256, 0, st>>>(B, ldb, K, N, Kp, bp, colmax);
  } else {
    if (scaled) split_b_kernel<2, true><<<grid, 256, 0, st>>>(B, ldb, K, N, Kp, bp, colmax);
    else split_b_kernel<2, false><<<grid, 256, 0, st>>>(B, ldb, K, N, Kp, bp, colmax);
  }
  return cudaGetLastError();
}

}  // namespace hbsg
