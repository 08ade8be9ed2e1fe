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
#include "internal.h"
#include "split_kernel.cuh"

namespace hbsg {

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

// B (K x N, row stride ldb) -> Bp[p][n][0..Kp) through 64 x 64 shared tiles.
template <int P, bool SCALED>
__global__ void __launch_bounds__(256) split_b_kernel(const float* __restrict__ B, long ldb, int K,
                                                      int N, int Kp, __nv_bfloat16* __restrict__ Bp,
                                                      const uint32_t* __restrict__ colmax) {
  __shared__ float tile[64][65];
  split_b_block<P, SCALED>(B, ldb, K, N, Kp, Bp, colmax, blockIdx.y * 64, blockIdx.x * 64, tile);
}

cudaError_t maxabs_rows(const float* A, long lda, int M, int K, uint32_t* rowmax, cudaStream_t st) {
  if (M > 0) row_maxabs_kernel<<<(M + 7) / 8, 256, 0, st>>>(A, lda, M, K, rowmax);
  return cudaGetLastError();
}

cudaError_t maxabs_cols(const float* B, long ldb, int K, int N, uint32_t* colmax, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(colmax, 0, sizeof(uint32_t) * N, st);
  if (e != cudaSuccess) return e;
  const int kpb = 256;
  dim3 g((N + 255) / 256, (K + kpb - 1) / kpb);
  if (K > 0 && N > 0) col_maxabs_kernel<<<g, 256, 0, st>>>(B, ldb, K, N, kpb, colmax);
  return cudaGetLastError();
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
