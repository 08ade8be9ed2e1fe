// Split-BF16 tensor-core GEMM kernel body for sm_100a (tcgen05 + TMEM + TMA),
// shared by the single-GEMM launch (tc_gemm.cu) and the grouped launch
// (grouped.cu). See tc_gemm.cu for the design.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "internal.h"

namespace hbsg {

// Device-side error flag of this translation unit (read by the host through
// the TU's *_read_and_clear_device_error function).
static __device__ int g_device_error = 0;

// Tensor-core tile table (parts, BN, stages), shared by the single-GEMM and
// grouped launches so that tile ids mean the same shape in both. Entries with
// 3 parts serve the 6-product forms, 2 parts the 3-product forms. BN = 192
// fills the last wave better where 256-wide tiles leave it part empty (4096^2:
// 704 tiles = 4.76 waves on 148 SMs instead of 512 = 3.46).
#define HBSG_TC_TILE_LIST(X) \
  X(3, 256, 3)               \
  X(3, 128, 4)               \
  X(3, 64, 6)                \
  X(2, 256, 4)               \
  X(2, 128, 6)               \
  X(2, 64, 8)                \
  X(3, 192, 3)               \
  X(2, 192, 5)

static constexpr int kBM = 128;
static constexpr int kTileQueue = 8;  // entries of the tile queue ring in shared memory
static constexpr int kBK = 32;  // bf16 elements per k-tile row = 64 bytes = one swizzle row
static constexpr unsigned long long kWaitLimitNs = 4000000000ull;  // default bound: 4 s

HBSG_DEV unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait on an mbarrier phase. Returns false (and raises the flags) on
// timeout or when another role already aborted.
HBSG_DEV bool wait_bounded(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                          unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63) == 0) {
      if (*abort_flag) return false;
      if (globaltimer() - t0 > limit_ns) {
        *abort_flag = 1;
        atomicExch(&g_device_error, (int)HBSG_ERR_DEVICE_TIMEOUT);
        return false;
      }
    }
  }
}

HBSG_DEV void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// Same load with an L2 cache policy (from createpolicy).
HBSG_DEV void tma_load_3d_hint(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                               uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3, %4}], [%5], %6;\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar)),
      "l"(policy)
      : "memory");
}

HBSG_DEV uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// L2 prefetch of one 3-D tensor box (no shared-memory destination, no
// completion): keeps operand tiles warm in L2 ahead of the smem ring.
HBSG_DEV void tma_prefetch_3d(const CUtensorMap* map, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}

HBSG_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
HBSG_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Issue forms for a whole converged warp: elect.sync picks the one lane that
// issues, and the loop around them runs on all lanes with warp-uniform
// operands (TMEM addresses, descriptors). The same loop run inside a branch
// taken by lane 0 alone measured ~70 cycles per MMA issued, against the ~32
// an M = 128, N = 64, K = 16 MMA takes on the tensor core.
HBSG_DEV void tc_mma_elect(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                           uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p, e;\n\t.reg .b32 l;\n\t"
      "elect.sync l|e, 0xffffffff;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

HBSG_DEV void tc_commit_elect(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .pred e;\n\t.reg .b32 l;\n\t"
      "elect.sync l|e, 0xffffffff;\n\t"
      "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}\n" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 32 lanes x 32 columns of 32-bit TMEM into 32 registers per thread.
HBSG_DEV void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor: K-major, 64-byte swizzle, rows of 64 bytes,
// 8-row core groups 512 bytes apart (SBO), LBO unused for swizzled K-major
// (encoded 1), descriptor version 1 (bits 46-47), layout type 4 = SWIZZLE_64B.
HBSG_DEV uint64_t sw64_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

// Instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28.
__host__ __device__ constexpr uint32_t f16_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Product q of the P-part form as (A part, B part), smallest term first.
// P = 2: (hi,mid) (mid,hi) (hi,hi)
// P = 3: (mid,mid) (hi,lo) (lo,hi) (hi,mid) (mid,hi) (hi,hi)
template <int P>
struct Products {
  static constexpr int n = P == 3 ? 6 : 3;
  __host__ __device__ static constexpr int a(int q) {
    return P == 3 ? (q == 0 ? 1 : q == 2 ? 2 : q == 4 ? 1 : 0) : (q == 1 ? 1 : 0);
  }
  __host__ __device__ static constexpr int b(int q) {
    return P == 3 ? (q == 0 ? 1 : q == 1 ? 2 : q == 3 ? 1 : 0) : (q == 0 ? 1 : 0);
  }
};
static_assert(Products<3>::a(0) == 1 && Products<3>::b(0) == 1, "mid*mid");
static_assert(Products<3>::a(1) == 0 && Products<3>::b(1) == 2, "hi*lo");
static_assert(Products<3>::a(2) == 2 && Products<3>::b(2) == 0, "lo*hi");
static_assert(Products<3>::a(3) == 0 && Products<3>::b(3) == 1, "hi*mid");
static_assert(Products<3>::a(4) == 1 && Products<3>::b(4) == 0, "mid*hi");
static_assert(Products<3>::a(5) == 0 && Products<3>::b(5) == 0, "hi*hi");
static_assert(Products<2>::a(0) == 0 && Products<2>::b(0) == 1, "hi*mid");
static_assert(Products<2>::a(1) == 1 && Products<2>::b(1) == 0, "mid*hi");
static_assert(Products<2>::a(2) == 0 && Products<2>::b(2) == 0, "hi*hi");

template <int P, int BN, int STAGES>
struct TcShape {
  static constexpr int kABytes = kBM * kBK * 2;  // one part
  static constexpr int kBBytes = BN * kBK * 2;
  static constexpr int kStageBytes = P * (kABytes + kBBytes);
  static constexpr int kTmemCols = 2 * BN;  // two accumulator buffers
  static constexpr int kAllocCols = kTmemCols <= 32 ? 32 : kTmemCols <= 64 ? 64 : kTmemCols <= 128 ? 128 : kTmemCols <= 256 ? 256 : 512;
  static constexpr int kBarBytes = 8 * (2 * STAGES + 4) + 16;
  static constexpr int kColExpBytes = 8 * 4 * (BN / 2);  // scaled epilogue: per-warp column exponents
  // tile queue (grouped launches): kTileQueue barrier pairs, then the entries
  static constexpr int kQueueOff = STAGES * kStageBytes + kBarBytes + kColExpBytes;
  static constexpr int kQueueBytes = kTileQueue * (2 * 8 + 16);
  static constexpr int kSmemBytes = 1024 + kQueueOff + kQueueBytes;
  static constexpr int kThreads = 320;
  static_assert(kSmemBytes <= 232448, "shared memory");
  static_assert(BN % 16 == 0 && BN >= 64 && BN <= 256, "UMMA N");
};

// frexp exponent of max|x| from its FP32 bit pattern: the scale 2^-e the
// split applied to that row or column (0 for zero, non-finite or absent).
HBSG_DEV int pow2_exp_of_bits(uint32_t bits) {
  const int E = (int)((bits >> 23) & 0xffu);
  if (E == 0xff || bits == 0u) return 0;
  if (E != 0) return E - 126;
  int e;
  frexpf(__uint_as_float(bits), &e);  // subnormal maximum
  return e;
}

// x * 2^s, exact when 2^s is a normal float (one rounding otherwise, as ldexpf).
// Out of line: the rare out-of-range case stays one call instruction at each
// of the epilogue's many unrolled call sites, which keeps the kernel's code
// (and so the MMA issuer's instruction-cache footprint) small.
static __device__ __noinline__ float scale_pow2_slow(float x, int s) { return ldexpf(x, s); }

HBSG_DEV float scale_pow2(float x, int s) {
  if (s == 0) return x;
  if (s >= -126 && s <= 127) return x * __uint_as_float((uint32_t)(s + 127) << 23);
  return scale_pow2_slow(x, s);
}

// One output tile of work for the kernel body.
struct TileWork {
  int prob;               // problem index (grouped launches; 0 otherwise)
  int ready_target;       // inline split: jobs that must be done before loading (0 = none)
  const CUtensorMap* ma;  // A parts map (box {32, 128, P})
  const CUtensorMap* mb;  // B parts map (box {32, BN, P})
  float* C;
  long ldc;
  int M, N;
  int m0, n0;
  int kt0;  // first k-tile (of 32) of this work item
  int KT;   // k-tiles in this work item
  const uint32_t* rowmax;  // scaled forms only
  const uint32_t* colmax;
  // FP32 operands, read by the fused-split body only (tc_fused.cuh): A is
  // M x K (row stride lda), B is K x N (row stride ldb)
  const float* A = nullptr;
  const float* B = nullptr;
  long lda = 0, ldb = 0;
  int K = 0;
};

// Settings shared by every tile of a launch.
struct TcRun {
  int chunk_ktiles;                  // k-tiles accumulated in TMEM before draining
  int l2_keep;                       // 1: operand loads carry an L2 evict-last policy
  int l2_ahead;                      // k-tiles prefetched into L2 ahead of the loads (0 = off)
  unsigned long long wait_limit_ns;  // bound of every mbarrier wait
  int debug_skip_loads;              // test hook: producer never loads (forces the timeout path)
};

// Writes one warp's 32 x COLS block of C, held one row per lane (lane l: row
// row0 + l, columns col0 .. col0 + COLS - 1 in sum[]). Inside each group of
// 32 / VW lanes the VW-float column chunks of every 32-column block are
// transposed by xor-butterfly shuffle stages, after which lane i of a group
// holds columns VW*i .. VW*i + VW-1 of the group's rows. Each store
// instruction then writes whole 128-byte row segments instead of 32 rows of
// VW*4 bytes: scattered stores crowd the load/store path that the MMA issue
// shares, which cost the grouped product (tiles of K ~ 1000, so much more C
// per FLOP) about 10 % of its time; with VW = 4 this measured 7.3 -> 6.6 ms
// on 512 products of ~1000^3 (32-byte chunks over 4-lane groups: 6.7 ms).
// Scaled forms apply 2^(row exponent + column exponent) first.
template <int COLS, bool SCALED, int VW = 4>
HBSG_DEV void store_rows_transposed(float* sum, const TileWork& w, int row0, int col0, int lane,
                                    const int* wexp, int row_end = 0x7fffffff) {
  static_assert(VW == 4, "16-byte chunks (float4 stores)");
  constexpr int NCH = 32 / VW;  // chunks per 32-column block = lanes per group
  if constexpr (SCALED) {
    const int row = row0 + lane;
    const int er = row < w.M ? pow2_exp_of_bits(w.rowmax[row]) : 0;
#pragma unroll
    for (int j = 0; j < COLS; ++j) sum[j] = scale_pow2(sum[j], er + wexp[j]);
  }
  const int gi = lane & (NCH - 1);
  const int rb = row0 + (lane & ~(NCH - 1));
  const bool vec = ((w.ldc & (VW - 1)) == 0) &&
                   ((reinterpret_cast<uintptr_t>(w.C) & (4 * VW - 1)) == 0);
#pragma unroll
  for (int b = 0; b < COLS / 32; ++b) {
    float* x = sum + 32 * b;
#pragma unroll
    for (int s = NCH / 2; s >= 1; s >>= 1) {
      const bool up = (gi & s) != 0;
#pragma unroll
      for (int c = 0; c < NCH; ++c) {
        if (c & s) continue;
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          const float send = up ? x[VW * c + e] : x[VW * (c ^ s) + e];
          const float got = __shfl_xor_sync(0xffffffffu, send, s);
          if (up) x[VW * c + e] = got;
          else x[VW * (c ^ s) + e] = got;
        }
      }
    }
    const int c = col0 + 32 * b + VW * gi;
#pragma unroll
    for (int rho = 0; rho < NCH; ++rho) {
      const int r = rb + rho;
      if (r >= w.M || r >= row_end) continue;
      float* p = w.C + (long)r * w.ldc + c;
      const float* v = x + VW * rho;
      if (vec && c + VW - 1 < w.N) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
      } else {
#pragma unroll
        for (int e = 0; e < VW; ++e)
          if (c + e < w.N) p[e] = v[e];
      }
    }
  }
}

// Kernel body shared by the single-GEMM and grouped launches. `Tiles` gives
// count() and get(t). Tiles are dealt in one of two ways:
//   - Tiles::kQueue false: CTA b processes tiles b, b + gridDim.x, ...
//   - Tiles::kQueue true (grouped launches): the producer thread claims the
//     next tile from a global counter (tiles.queue, zeroed before the launch)
//     one tile ahead, and hands each claimed tile (index, k-tiles, MMA width)
//     to the MMA issuer and the epilogue through a ring of kTileQueue entries
//     in shared memory (full / empty mbarrier pairs, every wait bounded); an
//     index of -1 ends the sequence. A CTA that drew long tiles then takes
//     fewer, so the persistent grid ends together however uneven the tiles.
// When Tiles::kInlineSplit is true the CTA has two more warps (10, 11) that
// produce the BF16 operand parts while the tensor cores work
// (Tiles::split_worker), and the producer waits for a problem's parts to be
// complete (Tiles::wait_ready) before loading its first tile.
template <int P, int BN, int STAGES, bool SCALED, class Tiles>
__device__ __forceinline__ void tc_body(const Tiles& tiles, const TcRun& run) {
  using S = TcShape<P, BN, STAGES>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* smem = smem_raw + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * S::kStageBytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* tfull = bars + 2 * STAGES;
  uint64_t* tempty = bars + 2 * STAGES + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* col_exp = reinterpret_cast<int*>(smem + STAGES * S::kStageBytes + S::kBarBytes);
  uint64_t* qfull = reinterpret_cast<uint64_t*>(smem + S::kQueueOff);  // producer published
  uint64_t* qempty = qfull + kTileQueue;  // the MMA issuer and the 8 epilogue warps read it
  volatile int* qent = reinterpret_cast<volatile int*>(qempty + kTileQueue);  // 4 ints an entry

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int num_tiles = tiles.count();

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 8);
    }
    for (int j = 0; j < kTileQueue; ++j) {
      mbar_init(&qfull[j], 1);
      mbar_init(&qempty[j], 9);
    }
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(S::kAllocCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const unsigned long long lim = run.wait_limit_ns;

  // Next entry of the tile queue for a consumer (the MMA issuer, or lane 0 of
  // an epilogue warp): {tile or -1, k-tiles, MMA width, valid rows}; false on
  // abort.
  auto queue_take = [&](uint32_t& q, int4& e) -> bool {
    const int j = (int)(q % kTileQueue);
    if (!wait_bounded(&qfull[j], (q / kTileQueue) & 1, abort_flag, lim)) return false;
    e = make_int4(qent[4 * j], qent[4 * j + 1], qent[4 * j + 2], qent[4 * j + 3]);
    mbar_arrive(&qempty[j]);
    ++q;
    return true;
  };

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      uint32_t it = 0, q = 0;
      bool ok = true;
      const CUtensorMap* last_ma = nullptr;
      int ready_prob = -1;
      const uint64_t keep = l2_policy_evict_last();
      // the current tile t and the next tn are known (claimed) one tile
      // ahead, so the description loads and the claim's atomic never sit on
      // the critical path at a tile switch
      int t, tn;
      if constexpr (Tiles::kQueue) {
        t = atomicAdd(tiles.queue, 1);
        tn = t < num_tiles ? atomicAdd(tiles.queue, 1) : num_tiles;
      } else {
        t = blockIdx.x;
        tn = t + (int)gridDim.x;
      }
      TileWork w;
      if (t < num_tiles) w = tiles.get(t);
      for (;;) {
        if constexpr (Tiles::kQueue) {
          // publish t (or the end of the sequence) to the consumers
          const int j = (int)(q % kTileQueue);
          if (!wait_bounded(&qempty[j], ((q / kTileQueue) & 1) ^ 1, abort_flag, lim)) {
            ok = false;
            break;
          }
          const int nv = t < num_tiles ? min(BN, w.N - w.n0) : 0;
          qent[4 * j] = t < num_tiles ? t : -1;
          qent[4 * j + 1] = t < num_tiles ? w.KT : 0;
          qent[4 * j + 2] = nv;
          qent[4 * j + 3] = t < num_tiles ? min(kBM, w.M - w.m0) : 0;
          mbar_arrive(&qfull[j]);
          ++q;
        }
        if (t >= num_tiles || !ok) break;
        TileWork nx = w;
        const bool has_next = tn < num_tiles;
        if (has_next) nx = tiles.get(tn);
        if constexpr (Tiles::kInlineSplit) {
          if (w.ready_target > 0 && w.prob != ready_prob) {
            if (!tiles.wait_ready(w.prob, w.ready_target, abort_flag, lim)) {
              ok = false;
              break;
            }
            ready_prob = w.prob;
          }
        }
        if (w.ma != last_ma) {
          asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(w.ma)) : "memory");
          asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(w.mb)) : "memory");
          last_ma = w.ma;
        }
        for (int kt = 0; kt < w.KT; ++kt, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!wait_bounded(&empty[s], ph ^ 1, abort_flag, lim)) {
            ok = false;
            break;
          }
          if (run.debug_skip_loads) continue;
          const uint32_t sa = base + s * S::kStageBytes;
          const uint32_t sb = sa + P * S::kABytes;
          mbar_arrive_expect_tx(&full[s], S::kStageBytes);
          if (run.l2_keep) {
            tma_load_3d_hint(sa, w.ma, (w.kt0 + kt) * kBK, w.m0, 0, &full[s], keep);
            tma_load_3d_hint(sb, w.mb, (w.kt0 + kt) * kBK, w.n0, 0, &full[s], keep);
          } else {
            tma_load_3d(sa, w.ma, (w.kt0 + kt) * kBK, w.m0, 0, &full[s]);
            tma_load_3d(sb, w.mb, (w.kt0 + kt) * kBK, w.n0, 0, &full[s]);
          }
          if (run.l2_ahead > 0) {  // the k-tile l2_ahead steps further, possibly of the next tile
            const int ka = kt + (kt == 0 ? 1 : run.l2_ahead);
            const int kend = kt == 0 ? min(w.KT, 1 + run.l2_ahead) : ka + 1;
            for (int kp = ka; kp < kend; ++kp) {  // at kt == 0: warm the whole lookahead window
              if (kp < w.KT) {
                tma_prefetch_3d(w.ma, (w.kt0 + kp) * kBK, w.m0, 0);
                tma_prefetch_3d(w.mb, (w.kt0 + kp) * kBK, w.n0, 0);
              } else if (has_next && kp - w.KT < nx.KT) {
                tma_prefetch_3d(nx.ma, (nx.kt0 + kp - w.KT) * kBK, nx.m0, 0);
                tma_prefetch_3d(nx.mb, (nx.kt0 + kp - w.KT) * kBK, nx.n0, 0);
              }
            }
          }
          if (kt == 0 && has_next && nx.ma != w.ma) {  // warm the next problem's maps
            asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(nx.ma)) : "memory");
            asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(nx.mb)) : "memory");
          }
        }
        if (!ok) break;
        w = nx;
        t = tn;
        if constexpr (Tiles::kQueue) {
          if (tn < num_tiles) tn = atomicAdd(tiles.queue, 1);
        } else {
          tn += (int)gridDim.x;
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    // The whole warp runs the loop converged and one elected lane issues
    // (tc_mma_elect); lane 0 takes the tile queue's entries for the warp, and
    // a wait passes only when it passed on every lane.
    {
      uint32_t it = 0, ch = 0, q = 0;
      bool ok = true;
      int t = blockIdx.x;
      TileWork w;  // static deal: fetched one tile ahead (see the producer)
      if constexpr (!Tiles::kQueue) {
        if (t < num_tiles) w = tiles.get(t);
      }
      for (;;) {
        int KT, nv, mv;
        if constexpr (Tiles::kQueue) {
          int4 e = make_int4(-1, 0, 0, 0);
          int got = 1;
          if (lane == 0) got = queue_take(q, e);
          const int tile = __shfl_sync(0xffffffffu, got ? e.x : -2, 0);
          if (tile < 0) break;  // -1: end of the sequence; -2: abort
          KT = __shfl_sync(0xffffffffu, e.y, 0);
          nv = __shfl_sync(0xffffffffu, e.z, 0);
          mv = __shfl_sync(0xffffffffu, e.w, 0);
        } else {
          if (t >= num_tiles) break;
          TileWork nx = w;
          if (t + (int)gridDim.x < num_tiles) nx = tiles.get(t + gridDim.x);
          KT = w.KT;
          nv = min(BN, w.N - w.n0);
          mv = min(kBM, w.M - w.m0);
          w = nx;
          t += gridDim.x;
        }
        // MMA width trimmed to the tile's valid columns (multiple of 16), and
        // its height to 64 when the tile holds at most 64 valid rows: the
        // last row and column tiles of a problem do less tensor work on
        // padding. (An M = 64 accumulator holds row r in lane
        // 32 (r / 16) + r % 16; the epilogue reads it so.)
        const uint32_t idesc =
            f16_idesc(mv <= 64 ? 64 : kBM, nv >= BN ? BN : ((nv + 15) & ~15));
        const int nchunks = (KT + run.chunk_ktiles - 1) / run.chunk_ktiles;
        int kt = 0;
        for (int c = 0; c < nchunks && ok; ++c, ++ch) {
          const int buf = ch & 1;
          if (!__all_sync(0xffffffffu,
                          wait_bounded(&tempty[buf], ((ch >> 1) & 1) ^ 1, abort_flag, lim))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem_base + buf * BN;
          const int kend = min(KT, kt + run.chunk_ktiles);
          bool first = true;
          for (; kt < kend; ++kt, ++it) {
            const int s = it % STAGES;
            if (!__all_sync(0xffffffffu,
                            wait_bounded(&full[s], (it / STAGES) & 1, abort_flag, lim))) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t sa = base + s * S::kStageBytes;
            const uint32_t sb = sa + P * S::kABytes;
#pragma unroll
            for (int ks = 0; ks < kBK / 16; ++ks) {
#pragma unroll
              for (int q2 = 0; q2 < Products<P>::n; ++q2) {
                const uint64_t ad = sw64_desc(sa + Products<P>::a(q2) * S::kABytes + ks * 32);
                const uint64_t bd = sw64_desc(sb + Products<P>::b(q2) * S::kBBytes + ks * 32);
                tc_mma_elect(d, ad, bd, idesc, first ? 0u : 1u);
                first = false;
              }
            }
            tc_commit_elect(&empty[s]);
          }
          if (ok) tc_commit_elect(&tfull[buf]);
        }
        if (!ok) break;
      }
    }
  } else if (warp >= 10) {
    // ---------------- operand splitters (inline-split launches) ----------------
    if constexpr (Tiles::kInlineSplit) tiles.template split_worker<P, SCALED>(lane, abort_flag);
  } else {
    // ---------------- epilogue (warps 2..9) ----------------
    const int q = warp & 3;         // TMEM lane quadrant this warp may access
    const int h = (warp - 2) >> 2;  // column half
    constexpr int COLS = BN / 2;
    uint32_t ch = 0, qs = 0;
    bool ok = true;
    int t = blockIdx.x;
    for (;;) {
      if constexpr (Tiles::kQueue) {
        int4 e = make_int4(-1, 0, 0, 0);
        int got = 1;
        if (lane == 0) got = queue_take(qs, e);
        t = __shfl_sync(0xffffffffu, got ? e.x : -2, 0);
        if (t < 0) break;  // -1: end of the sequence; -2: abort
      } else {
        if (t >= num_tiles) break;
      }
      const TileWork w = tiles.get(t);
      if constexpr (!Tiles::kQueue) t += gridDim.x;
      const int nchunks = (w.KT + run.chunk_ktiles - 1) / run.chunk_ktiles;
      float sum[COLS];
#pragma unroll
      for (int i = 0; i < COLS; ++i) sum[i] = 0.0f;
      for (int c = 0; c < nchunks; ++c, ++ch) {
        const int buf = ch & 1;
        int got = 0;
        if (lane == 0) got = wait_bounded(&tfull[buf], (ch >> 1) & 1, abort_flag, lim);
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!got) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem_base + ((uint32_t)(32 * q) << 16) + buf * BN + h * COLS;
#pragma unroll
        for (int j = 0; j < COLS / 32; ++j) {
          float v[32];
          tmem_ld32(taddr + 32 * j, v);
#pragma unroll
          for (int i = 0; i < 32; ++i) sum[32 * j + i] += v[i];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[buf]);
      }
      if (!ok) break;
      const int col0 = w.n0 + h * COLS;
      int* wexp = col_exp + (warp - 2) * COLS;  // this warp's column exponents
      if constexpr (SCALED) {
        // each warp stages the exponents of its own COLS columns (no barrier
        // across warps, so a warp that unwinds early can never strand others)
        __syncwarp();
#pragma unroll
        for (int i = lane; i < COLS; i += 32)
          wexp[i] = pow2_exp_of_bits(w.colmax[min(col0 + i, w.N - 1)]);
        __syncwarp();
      }
      // an M = 64 accumulator (tiles with at most 64 valid rows) holds rows
      // 16 q .. 16 q + 15 in lanes 32 q .. 32 q + 15 of the warp's quadrant
      if (w.M - w.m0 <= 64)
        store_rows_transposed<COLS, SCALED>(sum, w, w.m0 + 16 * q, col0, lane, wexp,
                                            w.m0 + 16 * q + 16);
      else
        store_rows_transposed<COLS, SCALED>(sum, w, w.m0 + 32 * q, col0, lane, wexp);
    }
  }

  // All roles leave their loops (normally or through a bounded abort); MMAs
  // the epilogue waited for are complete. On abort, give in-flight tensor-core
  // work a bounded moment before the TMEM is released.
  __syncthreads();
  if (*abort_flag) {
    const unsigned long long t0 = globaltimer();
    while (globaltimer() - t0 < 2000000ull) {
    }
  }
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base),
                 "r"(S::kAllocCols));
  }
}

}  // namespace hbsg
