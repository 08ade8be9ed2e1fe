// Split helpers (FP32 -> BF16 parts) shared by the single and grouped split
// passes. The split itself is described in split_bf16.cu.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

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

// One 64 (k) x 64 (n) block of B (K x N, row stride ldb) split into
// Bp[p][n][k0 .. k0+63], in three steps that callers may interleave with
// other blocks: split_b_load (16 values per thread into registers, coalesced
// along n), split_b_to_tile (into the shared tile), split_b_from_tile (split
// and store, 8 threads per 128-byte output row segment). 256 threads.
HBSG_DEV void split_b_load(const float* __restrict__ B, long ldb, int K, int N, int k0, int n0,
                           float* v) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int idx = tid + i * 256;
    const int k = k0 + (idx >> 6);
    const int n = n0 + (idx & 63);
    v[i] = (k < K && n < N) ? B[(long)k * ldb + n] : 0.0f;
  }
}

HBSG_DEV void split_b_to_tile(const float* v, float (*tile)[65]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int idx = tid + i * 256;
    tile[idx >> 6][idx & 63] = v[i];
  }
}

template <int P, bool SCALED>
HBSG_DEV void split_b_from_tile(int N, int Kp, __nv_bfloat16* __restrict__ Bp,
                                const uint32_t* __restrict__ colmax, int k0, int n0,
                                const float (*tile)[65]) {
  const int tid = threadIdx.x;
  const long plane = (long)N * Kp;
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

template <int P, bool SCALED>
HBSG_DEV void split_b_block(const float* __restrict__ B, long ldb, int K, int N, int Kp,
                            __nv_bfloat16* __restrict__ Bp, const uint32_t* __restrict__ colmax,
                            int k0, int n0, float (*tile)[65]) {
  float v[16];
  split_b_load(B, ldb, K, N, k0, n0, v);
  split_b_to_tile(v, tile);
  __syncthreads();
  split_b_from_tile<P, SCALED>(N, Kp, Bp, colmax, k0, n0, tile);
}

}  // namespace hbsg
