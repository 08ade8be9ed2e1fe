// FP32 SIMT (FFMA) SGEMM tile body for sm_100a, shared by the single and
// batched launch (ffma_sgemm.cu) and the grouped launch (grouped.cu). The
// design and the reference lines it follows are described in ffma_sgemm.cu.
#pragma once

#include "common.cuh"
#include "internal.h"

namespace hbsg {

template <int BM, int BN, int BK, int WM, int WN, int STAGES>
struct FfmaShape {
  static constexpr int kWarpsM = BM / WM;
  static constexpr int kWarpsN = BN / WN;
  static constexpr int kThreads = kWarpsM * kWarpsN * 32;
  static constexpr int TM = WM / 8;
  static constexpr int TN = WN / 4;
  static constexpr int AS = BK + 4;
  static constexpr int kAStage = BM * AS;
  static constexpr int kBStage = BK * BN;
  static constexpr int kSmemBytes = STAGES * (kAStage + kBStage) * 4;
  // resident CTAs per SM the register budget is sized for: small register
  // blocks (<= 64 accumulators) leave room for two 256-thread CTAs
  static constexpr int kMinBlocks = (kThreads <= 128 || TM * TN <= 64) ? 2 : 1;
  static_assert(WM % 8 == 0 && WN % 16 == 0, "warp tile");
  static_assert(BK % 4 == 0, "BK");
  static_assert(((AS / 4) & 1) == 1, "A pad keeps 8 rows in distinct bank groups");
};

// One BM x BN output tile over k in [k_begin, k_end): C tile = A rows x B
// columns, written to C (row stride ldc). `smem` is the dynamic shared
// memory ring; callers that process several tiles must __syncthreads()
// between calls.
// PAIR selects the packed two-lane FMA (__ffma2_rn, sm_100): each instruction
// performs two independent IEEE fused multiply-adds, so the per-element
// arithmetic is unchanged while half as many FMA instructions are issued.
// TA / TB: A stored k x m (element (m, k) at A[k*lda + m]) / B stored n x k
// (element (k, n) at B[n*ldb + k]). Transposed operands use the 4-byte copy
// path with the thread order chosen for coalesced global reads; the shared
// memory layouts, and so the arithmetic, are the same as for row-major.
template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool VEC, bool PAIR,
          bool TA = false, bool TB = false>
__device__ __forceinline__ void ffma_tile(const float* __restrict__ A, long lda,
                                          const float* __restrict__ B, long ldb, int M, int N,
                                          int k_begin, int k_end, int m0, int n0, float* C,
                                          long ldc, bool vec_store, float* smem) {
  using S = FfmaShape<BM, BN, BK, WM, WN, STAGES>;
  constexpr int NT = S::kThreads;
  constexpr int TM = S::TM;
  constexpr int TN = S::TN;
  constexpr int AS = S::AS;

  float* As = smem;
  float* Bs = smem + STAGES * S::kAStage;
  const int KT = k_end > k_begin ? (k_end - k_begin + BK - 1) / BK : 0;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = warp / S::kWarpsN;
  const int wn = warp % S::kWarpsN;
  const int tm = lane & 7;
  const int tn = lane >> 3;

  auto load_tile = [&](int slot, int kt) {
    const int k0 = k_begin + kt * BK;
    float* as = As + slot * S::kAStage;
    float* bs = Bs + slot * S::kBStage;
    if constexpr (VEC) {
      constexpr int ACH = BM * BK / 4;
#pragma unroll
      for (int c = tid; c < ACH; c += NT) {
        const int r = c / (BK / 4);
        const int kc = (c % (BK / 4)) * 4;
        const int gr = m0 + r;
        const int gk = k0 + kc;
        int bytes = 0;
        const float* src = A;
        if (gr < M && gk < k_end) {
          bytes = min(4, k_end - gk) * 4;
          src = A + (long)gr * lda + gk;
        }
        cp_async16(as + r * AS + kc, src, bytes);
      }
      constexpr int BCH = BK * BN / 4;
#pragma unroll
      for (int c = tid; c < BCH; c += NT) {
        const int r = c / (BN / 4);
        const int nc = (c % (BN / 4)) * 4;
        const int gk = k0 + r;
        const int gn = n0 + nc;
        int bytes = 0;
        const float* src = B;
        if (gk < k_end && gn < N) {
          bytes = min(4, N - gn) * 4;
          src = B + (long)gk * ldb + gn;
        }
        cp_async16(bs + r * BN + nc, src, bytes);
      }
    } else {
      static_assert(!(VEC && (TA || TB)), "transposed operands use the 4-byte path");
#pragma unroll 4
      for (int c = tid; c < BM * BK; c += NT) {
        const int r = TA ? c % BM : c / BK;   // transposed: m fastest (contiguous)
        const int kc = TA ? c / BM : c % BK;  // row-major: k fastest (contiguous)
        const int gr = m0 + r;
        const int gk = k0 + kc;
        const bool ok = gr < M && gk < k_end;
        const long off = TA ? (long)gk * lda + gr : (long)gr * lda + gk;
        cp_async4(as + r * AS + kc, ok ? A + off : A, ok ? 4 : 0);
      }
#pragma unroll 4
      for (int c = tid; c < BK * BN; c += NT) {
        const int r = c / BN;  // n fastest: conflict-free shared stores; for a
        const int nc = c % BN; // transposed B the row reads are absorbed by L1
        const int gk = k0 + r;
        const int gn = n0 + nc;
        const bool ok = gk < k_end && gn < N;
        const long off = TB ? (long)gn * ldb + gk : (long)gk * ldb + gn;
        cp_async4(bs + r * BN + nc, ok ? B + off : B, ok ? 4 : 0);
      }
    }
  };

  float acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.0f;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_tile(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < KT) load_tile(nk % STAGES, nk);
      cp_async_commit();
    }
    const int slot = kt % STAGES;
    const float* a_s = As + slot * S::kAStage + (wm * WM + tm) * AS;
    const float* b_s = Bs + slot * S::kBStage + wn * WN + 4 * tn;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      float4 a4[TM];
#pragma unroll
      for (int i = 0; i < TM; ++i) a4[i] = *reinterpret_cast<const float4*>(a_s + i * 8 * AS + kk);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float4 b4[TN / 4];
#pragma unroll
        for (int j = 0; j < TN / 4; ++j)
          b4[j] = *reinterpret_cast<const float4*>(b_s + (kk + k) * BN + 16 * j);
        // the (a, a) operand pairs of the packed FMA are built for all rows
        // before the step's FMAs, off their dependency chains (measured +1 %)
        float2 a2s[TM];
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          const float av = k == 0 ? a4[i].x : k == 1 ? a4[i].y : k == 2 ? a4[i].z : a4[i].w;
          a2s[i] = make_float2(av, av);
        }
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          const float av = k == 0 ? a4[i].x : k == 1 ? a4[i].y : k == 2 ? a4[i].z : a4[i].w;
          if constexpr (PAIR) {
            const float2 a2 = a2s[i];
#pragma unroll
            for (int j = 0; j < TN / 4; ++j) {
              float2 lo = __ffma2_rn(a2, make_float2(b4[j].x, b4[j].y),
                                     make_float2(acc[i][4 * j + 0], acc[i][4 * j + 1]));
              float2 hi = __ffma2_rn(a2, make_float2(b4[j].z, b4[j].w),
                                     make_float2(acc[i][4 * j + 2], acc[i][4 * j + 3]));
              acc[i][4 * j + 0] = lo.x;
              acc[i][4 * j + 1] = lo.y;
              acc[i][4 * j + 2] = hi.x;
              acc[i][4 * j + 3] = hi.y;
            }
          } else {
#pragma unroll
            for (int j = 0; j < TN / 4; ++j) {
              acc[i][4 * j + 0] = __fmaf_rn(av, b4[j].x, acc[i][4 * j + 0]);
              acc[i][4 * j + 1] = __fmaf_rn(av, b4[j].y, acc[i][4 * j + 1]);
              acc[i][4 * j + 2] = __fmaf_rn(av, b4[j].z, acc[i][4 * j + 2]);
              acc[i][4 * j + 3] = __fmaf_rn(av, b4[j].w, acc[i][4 * j + 3]);
            }
          }
        }
      }
    }
  }
  cp_async_wait<0>();

  // Epilogue: direct stores.
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int r = m0 + wm * WM + tm + 8 * i;
    if (r >= M) continue;
    float* crow = C + (long)r * ldc;
#pragma unroll
    for (int j = 0; j < TN / 4; ++j) {
      const int c = n0 + wn * WN + 16 * j + 4 * tn;
      if (vec_store && c + 3 < N) {
        *reinterpret_cast<float4*>(crow + c) =
            make_float4(acc[i][4 * j], acc[i][4 * j + 1], acc[i][4 * j + 2], acc[i][4 * j + 3]);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (c + e < N) crow[c + e] = acc[i][4 * j + e];
      }
    }
  }
}

}  // namespace hbsg
