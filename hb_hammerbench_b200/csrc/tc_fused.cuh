// Split-BF16 tensor-core GEMM body with the FP32 -> BF16 split fused in
// (tcgen05 cta_group::2, CTA pairs, sm_100a).
//
// The unfused path writes the BF16 parts of both operands to HBM in a split
// pass and the product kernel reads them back: for an operand element that is
// 4 bytes read + 2*P written + 2*P read again, against the 4 bytes the
// product needs. Here the product kernel reads the FP32 operands itself:
//   - a loader thread streams this CTA's FP32 A rows and B columns of each
//     k-tile into a shared-memory staging ring with TMA (no registers held in
//     flight, so the ring can run several k-tiles ahead of DRAM latency);
//   - converter warps read a staged k-tile, split every value into P parts
//     (exactly the split pass's arithmetic: hi = bf16(x), mid = bf16(x - hi),
//     lo = bf16(x - hi - mid)) and write them into the operand stage in the
//     layout the TMA produced for the unfused kernel (K-major rows of 32 bf16
//     = 64 bytes, 64-byte swizzle: the 16-byte chunk c of row r lands at chunk
//     c ^ ((r >> 1) & 3));
//   - the MMA issuer and the epilogue are those of the pair kernel
//     (tc_kernel2.cuh): same products, same order, same TMEM drains, so the
//     result is bit-identical to the unfused kernels with the same drain
//     interval.
//
// Why CTA pairs: the tensor core's shared-memory operand reads per MMA flop
// are lowest for the 256 x 256 pair tile (each SM holds 128 A rows and 128 B
// columns). Staging and converting add shared-memory traffic (FP32 written by
// the TMA, read by the converters, parts written), which a single-CTA
// 128 x 256 tile, whose MMA alone reads ~3/4 of an SM's shared-memory
// bandwidth, has no room for.
//
// CTA (512 threads, 16 warps, one CTA per SM, clusters of two):
//   warp 0       TMEM allocation; the leader CTA's warp issues the MMAs
//                (one elected lane)
//   warp 1       lane 0: TMA loads of the FP32 staging ring
//   warps 2-7    converters (this CTA's 128 A rows and BN/2 B columns)
//   warps 8-15   epilogue (TMEM lane quadrant warp % 4, column half)
// Register split (setmaxnreg): warpgroups 0-1 (issuer, loader, converters)
// 96 registers per thread, enough for the converters to keep about two 8-value
// units in flight; warpgroups 2-3 (epilogue, BN/2 FP32 sums per thread) 160:
// 2 x 128 x 96 + 2 x 128 x 160 = 65536, the block's launch allotment
// (512 threads x 128).
// Every wait is bounded as in the other tensor-core bodies. The TMA loads use
// no cluster multicast: each CTA loads its own rows into its own memory.
#pragma once

#include "split_kernel.cuh"
#include "tc_kernel2.cuh"

namespace hbsg {

// Fused tile table (parts, BN, part stages, FP32 staging stages), shared by
// the single-GEMM and grouped launches so that fused tile ids mean the same
// shape in both: 6-product then 3-product forms, 256 then 64 columns wide.
#define HBSG_FUSED_TILE_LIST(X) \
  X(3, 256, 2, 3)               \
  X(2, 256, 2, 4)               \
  X(3, 64, 3, 5)                \
  X(2, 64, 3, 6)

static constexpr int kFusedThreads = 512;
static constexpr int kConvWarps = 6;
static constexpr int kConvThreads = kConvWarps * 32;
static constexpr int kRegsLow = 96;    // warpgroups 0-1
static constexpr int kRegsHigh = 160;  // warpgroups 2-3
static_assert(2 * 128 * kRegsLow + 2 * 128 * kRegsHigh == 65536, "register split");

// mbarrier probe with cluster-scope acquire: the converters of the peer CTA
// arrive on the leader's stage barrier with release at cluster scope.
HBSG_DEV bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

HBSG_DEV bool wait_bounded_cluster(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                   unsigned long long limit_ns) {
  if (mbar_try_wait_cluster(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait_cluster(bar, parity)) return true;
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

// mbarrier probe that lets the hardware suspend the thread until the phase
// completes or `ns` nanoseconds pass, so waiting warps do not spin on the
// issue slots the converter warps need.
HBSG_DEV bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}

HBSG_DEV bool wait_bounded_hint(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                unsigned long long limit_ns) {
  if (mbar_try_wait_hint(bar, parity, 20000)) return true;
  const unsigned long long t0 = globaltimer();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait_hint(bar, parity, 20000)) return true;
    if (*abort_flag) return false;
    if (globaltimer() - t0 > limit_ns) {
      *abort_flag = 1;
      atomicExch(&g_device_error, (int)HBSG_ERR_DEVICE_TIMEOUT);
      return false;
    }
  }
}

// Bounded wait for roles that wait long (the epilogue waits a whole TMEM
// drain interval): between probes the thread sleeps, so its warp does not
// take issue slots from the converter warps sharing its scheduler.
HBSG_DEV bool wait_bounded_sleep(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                 unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  for (uint32_t i = 0;; ++i) {
    __nanosleep(128);
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 15) == 0) {
      if (*abort_flag) return false;
      if (globaltimer() - t0 > limit_ns) {
        *abort_flag = 1;
        atomicExch(&g_device_error, (int)HBSG_ERR_DEVICE_TIMEOUT);
        return false;
      }
    }
  }
}

// Generic-proxy shared-memory writes -> visible to the tensor core (async proxy).
HBSG_DEV void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

template <int N>
HBSG_DEV void regs_dec() {
  asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(N));
}
template <int N>
HBSG_DEV void regs_inc() {
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(N));
}

HBSG_DEV void st_shared16(uint32_t addr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(v.x), "r"(v.y),
               "r"(v.z), "r"(v.w)
               : "memory");
}

// The body's setmaxnreg split hands out exactly kFusedThreads x 128
// registers; a kernel built with another register count would wait forever in
// setmaxnreg.inc, so launchers check the count once (cache: 0 unchecked,
// 1 ok, -1 wrong) and refuse to launch otherwise.
static inline bool fused_regs_ok(const void* kernel, int* cache) {
  int st = __atomic_load_n(cache, __ATOMIC_ACQUIRE);
  if (st == 0) {
    cudaFuncAttributes fa;
    st = (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess &&
          fa.numRegs * kFusedThreads == 65536)
             ? 1
             : -1;
    __atomic_store_n(cache, st, __ATOMIC_RELEASE);
  }
  return st == 1;
}

// Co-resident clusters of two CTAs of a fused kernel (0 if unknown).
static inline int fused_resident_clusters(const void* kernel, int smem) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(kFusedThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = 2;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

HBSG_DEV uint32_t bf162_bits(__nv_bfloat162 h) { return *reinterpret_cast<uint32_t*>(&h); }

// 32 lanes x 16 columns of 32-bit TMEM into 16 registers per thread.
HBSG_DEV void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Splits 8 consecutive-k values of one row (A) or column (B) into P packed
// 16-byte chunks, part 0 = hi: the split pass's arithmetic (split_value in
// split_kernel.cuh), two values per conversion instruction.
template <int P, bool SCALED>
HBSG_DEV void split8(float (&x)[8], int e, uint4 (&out)[P]) {
  if constexpr (SCALED) {
    if (e != 0) {
#pragma unroll
      for (int i = 0; i < 8; ++i) x[i] = ldexpf(x[i], -e);
    }
  }
  uint32_t h[4], m[4], l[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * j], x[2 * j + 1]);
    const float2 hf = __bfloat1622float2(hb);
    const float r0 = x[2 * j] - hf.x;
    const float r1 = x[2 * j + 1] - hf.y;
    const __nv_bfloat162 mb = __floats2bfloat162_rn(r0, r1);
    h[j] = bf162_bits(hb);
    m[j] = bf162_bits(mb);
    if constexpr (P == 3) {
      const float2 mf = __bfloat1622float2(mb);
      l[j] = bf162_bits(__floats2bfloat162_rn(r0 - mf.x, r1 - mf.y));
    }
  }
  out[0] = make_uint4(h[0], h[1], h[2], h[3]);
  out[1] = make_uint4(m[0], m[1], m[2], m[3]);
  if constexpr (P == 3) out[2] = make_uint4(l[0], l[1], l[2], l[3]);
}

template <int P, int BN, int STAGES, int SSTAGES>
struct TcFusedShape {
  static constexpr int kHalf = BN / 2;                  // B columns per CTA
  static constexpr int kABytes = kBM * kBK * 2;         // 128 rows of one part
  static constexpr int kBBytes = kHalf * kBK * 2;       // this CTA's B columns, one part
  static constexpr int kStageBytes = P * (kABytes + kBBytes);
  static constexpr int kSABytes = kBM * kBK * 4;        // FP32 A staging: 128 rows x 32 k
  static constexpr int kSBBytes = kBK * kHalf * 4;      // FP32 B staging: 32 k x BN/2 columns
  static constexpr int kSStageBytes = kSABytes + kSBBytes;
  static constexpr int kAllocCols = 2 * BN <= 32 ? 32 : 2 * BN <= 64 ? 64 : 2 * BN <= 128 ? 128 : 2 * BN <= 256 ? 256 : 512;
  static constexpr int kBarBytes = 8 * (2 * STAGES + 4 + 2 * SSTAGES) + 16;
  static constexpr int kColExpBytes = 8 * 4 * (BN / 2);
  static constexpr int kStagingOff = STAGES * kStageBytes;
  static constexpr int kBarOff = kStagingOff + SSTAGES * kSStageBytes;
  static constexpr int kSmemBytes = 1024 + kBarOff + kBarBytes + kColExpBytes;
  // converter work per k-tile: 8-element units (one row of A or column of B,
  // 8 consecutive k); A units first: unit u < kAUnits is row u / 4, chunk u % 4
  static constexpr int kAUnits = kBM * 4;
  static constexpr int kBUnits = kHalf * 4;
  static constexpr int kUnits = kAUnits + kBUnits;
  // converter warps split by operand, in proportion to the units (a B unit,
  // eight strided loads, costs more than an A unit)
  static constexpr int kAWarps = BN >= 128 ? kConvWarps / 2 : kConvWarps - 1;
  static constexpr int kBWarps = kConvWarps - kAWarps;
  static constexpr int kAThreads = 32 * kAWarps;
  static constexpr int kBThreads = 32 * kBWarps;
  static constexpr int kUnitsA = (kAUnits + kAThreads - 1) / kAThreads;
  static constexpr int kUnitsB = (kBUnits + kBThreads - 1) / kBThreads;
  static constexpr int kFullA = kAUnits / kAThreads;  // slots every A thread fills
  static constexpr int kFullB = kBUnits / kBThreads;
  static_assert(kSmemBytes <= 232448, "shared memory");
  static_assert(BN % 32 == 0 && BN >= 64 && BN <= 256, "pair UMMA N");
  static_assert(kBBytes % 512 == 0, "B part base keeps the 512-byte swizzle alignment");
  static_assert(kStageBytes % 1024 == 0 && kSStageBytes % 1024 == 0 && kSABytes % 1024 == 0,
                "FP32 A staging keeps the 1024-byte alignment of the 128-byte swizzle");
  static_assert(kAUnits % 32 == 0 && kHalf % 32 == 0, "a warp's units lie in 8 whole rows / 32 columns");
};

// Byte offset of the 16-byte chunk c (8 bf16) of row r in a part tile of
// 64-byte rows with the 64-byte swizzle (address bits 4-5 ^= bits 7-8).
HBSG_DEV uint32_t sw64_offset(int r, int c) {
  return (uint32_t)(r * 64 + ((c ^ ((r >> 1) & 3)) << 4));
}

// Byte offset of the 16-byte chunk c (4 floats) of row r in the FP32 A
// staging tile (128-byte rows, 128-byte swizzle: address bits 4-6 ^= bits 7-9).
HBSG_DEV uint32_t sw128_offset(int r, int c) {
  return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4));
}

HBSG_DEV void tma_prefetch_2d(const CUtensorMap* map, int c0, int c1) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1)
               : "memory");
}

HBSG_DEV void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

template <int P, int BN, int STAGES, int SSTAGES, bool SCALED, class Tiles>
__device__ __forceinline__ void tc_fused_body(const Tiles& tiles, const TcRun& run) {
  using S = TcFusedShape<P, BN, STAGES, SSTAGES>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* smem = smem_raw + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::kBarOff);
  uint64_t* full = bars;                     // leader: both CTAs' converters filled the stage
  uint64_t* empty = bars + STAGES;           // each CTA: the stage is free again
  uint64_t* tfull = bars + 2 * STAGES;       // each CTA: accumulator buffer ready
  uint64_t* tempty = bars + 2 * STAGES + 2;  // leader: both CTAs drained the buffer
  uint64_t* sfull = bars + 2 * STAGES + 4;   // each CTA: FP32 staging loaded (TMA)
  uint64_t* sempty = sfull + SSTAGES;        // each CTA: FP32 staging read by the converters
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sempty + SSTAGES);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* col_exp = reinterpret_cast<int*>(smem + S::kBarOff + S::kBarBytes);
  const uint32_t staging = base + S::kStagingOff;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1;
  const int pairs = gridDim.x >> 1;
  const int num_tiles = tiles.count();

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 2 * kConvWarps);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 16);
    }
    for (int s = 0; s < SSTAGES; ++s) {
      mbar_init(&sfull[s], 1);
      mbar_init(&sempty[s], kConvWarps);
    }
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(S::kAllocCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n");
  }
  tc_fence_before();
  cluster_sync();  // barriers of both CTAs initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const unsigned long long lim = run.wait_limit_ns;

  // Each role's code sits inside the branch that set its register count, so
  // the compiler allocates the epilogue's sums under the larger limit.
  if (warp < 8) regs_dec<kRegsLow>();
  if (warp == 0) {
    // ---------------- MMA issuer (leader CTA only) ----------------
    // The whole warp runs the loop converged and one elected lane issues
    // (tc_mma_elect); a wait passes only when it passed on every lane.
    if (leader) {
      // full-width MMAs: each CTA holds a fixed half of the BN columns, so the
      // instruction's N cannot be trimmed (padding columns are zeros)
      constexpr uint32_t idesc = f16_idesc(2 * kBM, BN);
      uint32_t it = 0, ch = 0;
      bool ok = true;
      for (int t = pair; t < num_tiles && ok; t += pairs) {
        const TileWork w = tiles.get(t);
        const int KT = w.KT;
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
            if (!__all_sync(0xffffffffu, wait_bounded_cluster(&full[s], (it / STAGES) & 1,
                                                              abort_flag, lim))) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t sa = base + s * S::kStageBytes;
            const uint32_t sb = sa + P * S::kABytes;
#pragma unroll
            for (int ks = 0; ks < kBK / 16; ++ks) {
#pragma unroll
              for (int q = 0; q < Products<P>::n; ++q) {
                const uint64_t ad = sw64_desc(sa + Products<P>::a(q) * S::kABytes + ks * 32);
                const uint64_t bd = sw64_desc(sb + Products<P>::b(q) * S::kBBytes + ks * 32);
                tc_mma_pair_elect(d, ad, bd, idesc, first ? 0u : 1u);
                first = false;
              }
            }
            tc_commit_pair_elect(&empty[s]);
          }
          if (ok) tc_commit_pair_elect(&tfull[buf]);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- TMA loader of the FP32 staging ring (both CTAs) ----------------
    // This CTA's 128 A rows x 32 k (box {32, 128}, 128-byte swizzle) and its
    // 32 k x BN/2 B columns (box {BN/2, 32}); rows and columns beyond the
    // matrix and k beyond K arrive as zeros (out-of-bounds fill).
    if (lane == 0) {
      uint32_t it = 0;
      bool ok = true;
      const CUtensorMap* last = nullptr;
      for (int t = pair; t < num_tiles && ok; t += pairs) {
        const TileWork w = tiles.get(t);
        if (w.ma != last) {
          asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(w.ma)) : "memory");
          asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(w.mb)) : "memory");
          last = w.ma;
        }
        const int arow = w.m0 + kBM * (int)rank;
        const int bcol = w.n0 + S::kHalf * (int)rank;
        for (int kp = SSTAGES; kp < min(w.KT, run.l2_ahead); ++kp) {
          tma_prefetch_2d(w.ma, (w.kt0 + kp) * kBK, arow);
          tma_prefetch_2d(w.mb, bcol, (w.kt0 + kp) * kBK);
        }
        for (int kt = 0; kt < w.KT; ++kt, ++it) {
          const int ss = it % SSTAGES;
          if (!wait_bounded_hint(&sempty[ss], ((it / SSTAGES) & 1) ^ 1, abort_flag, lim)) {
            ok = false;
            break;
          }
          const uint32_t dst = staging + ss * S::kSStageBytes;
          const int k0 = (w.kt0 + kt) * kBK;
          mbar_arrive_expect_tx(&sfull[ss], S::kSStageBytes);
          tma_load_2d(dst, w.ma, k0, arow, &sfull[ss]);
          tma_load_2d(dst + S::kSABytes, w.mb, bcol, k0, &sfull[ss]);
          // the k-tile l2_ahead further on, into L2 only, so that the load
          // issued for it later finds it there (inside this work item)
          if (run.l2_ahead > 0 && kt + run.l2_ahead < w.KT) {
            const int kp = k0 + run.l2_ahead * kBK;
            tma_prefetch_2d(w.ma, kp, arow);
            tma_prefetch_2d(w.mb, bcol, kp);
          }
        }
      }
    }
  } else if (warp < 8) {
    // ---------------- converters (both CTAs) ----------------
    // Warps 2 .. 2+kAWarps-1 convert A rows, the others B columns, so each
    // warp's unit loop is branch-free: all of a k-tile's loads are issued
    // first and the units' independent split chains overlap.
    const uint32_t full_leader0 = map_to_rank(smem_u32(&full[0]), 0);
    const bool a_role = warp < 2 + S::kAWarps;
    const int tr = a_role ? threadIdx.x - 64 : threadIdx.x - 64 - 32 * S::kAWarps;
    constexpr int NA = S::kUnitsA;   // unit slots per A thread (the last may be partial)
    constexpr int NB = S::kUnitsB;
    constexpr int NMAX = NA > NB ? NA : NB;
    int ex[NMAX];
#pragma unroll
    for (int i = 0; i < NMAX; ++i) ex[i] = 0;
    uint32_t it = 0;
    bool ok = true;
    for (int t = pair; t < num_tiles && ok; t += pairs) {
      const TileWork w = tiles.get(t);
      if constexpr (SCALED) {
        // the split exponent of each unit's row or column, fixed for the tile
#pragma unroll
        for (int i = 0; i < NMAX; ++i) {
          ex[i] = 0;
          if (a_role) {
            const int u = tr + i * S::kAThreads;
            const int m = w.m0 + kBM * (int)rank + (u >> 2);
            if (i < NA && u < S::kAUnits && m < w.M) ex[i] = exp_from_maxbits(w.rowmax[m]);
          } else {
            const int u = tr + i * S::kBThreads;
            const int n = w.n0 + S::kHalf * (int)rank + u % S::kHalf;
            if (i < NB && u < S::kBUnits && n < w.N) ex[i] = exp_from_maxbits(w.colmax[n]);
          }
        }
      }
      for (int kt = 0; kt < w.KT; ++kt, ++it) {
        const int s = it % STAGES;
        const int ss = it % SSTAGES;
        if (!wait_bounded_hint(&sfull[ss], (it / SSTAGES) & 1, abort_flag, lim) ||
            !wait_bounded_hint(&empty[s], ((it / STAGES) & 1) ^ 1, abort_flag, lim)) {
          ok = false;
          break;
        }
        // plain (non-volatile) shared-memory accesses, so the compiler can
        // schedule them freely; the barrier waits above and the proxy fence
        // below order them against the TMA writes and the tensor-core reads
        const uint8_t* f_p = smem + S::kStagingOff + ss * S::kSStageBytes;
        uint8_t* s_p = smem + s * S::kStageBytes;
        if (a_role) {
          float v[NA][8];
#pragma unroll
          for (int i = 0; i < NA; ++i) {
            const int u = tr + i * S::kAThreads;
            if (i < S::kFullA || u < S::kAUnits) {
              const int r = u >> 2, c = u & 3;
              const float4 a0 = *reinterpret_cast<const float4*>(f_p + sw128_offset(r, 2 * c));
              const float4 a1 = *reinterpret_cast<const float4*>(f_p + sw128_offset(r, 2 * c + 1));
              v[i][0] = a0.x; v[i][1] = a0.y; v[i][2] = a0.z; v[i][3] = a0.w;
              v[i][4] = a1.x; v[i][5] = a1.y; v[i][6] = a1.z; v[i][7] = a1.w;
            }
          }
#pragma unroll
          for (int i = 0; i < NA; ++i) {
            const int u = tr + i * S::kAThreads;
            if (i < S::kFullA || u < S::kAUnits) {
              uint4 o[P];
              split8<P, SCALED>(v[i], ex[i], o);
              const uint32_t off = sw64_offset(u >> 2, u & 3);
#pragma unroll
              for (int p = 0; p < P; ++p)
                *reinterpret_cast<uint4*>(s_p + p * S::kABytes + off) = o[p];
            }
          }
        } else {
          const uint8_t* fb_p = f_p + S::kSABytes;
          uint8_t* sb_p = s_p + P * S::kABytes;
          float v[NB][8];
#pragma unroll
          for (int i = 0; i < NB; ++i) {
            const int u = tr + i * S::kBThreads;
            if (i < S::kFullB || u < S::kBUnits) {
              const int col = u % S::kHalf, c = u / S::kHalf;
              const float* src = reinterpret_cast<const float*>(fb_p) + 8 * c * S::kHalf + col;
#pragma unroll
              for (int j = 0; j < 8; ++j) v[i][j] = src[j * S::kHalf];
            }
          }
#pragma unroll
          for (int i = 0; i < NB; ++i) {
            const int u = tr + i * S::kBThreads;
            if (i < S::kFullB || u < S::kBUnits) {
              uint4 o[P];
              split8<P, SCALED>(v[i], ex[i], o);
              const uint32_t off = sw64_offset(u % S::kHalf, u / S::kHalf);
#pragma unroll
              for (int p = 0; p < P; ++p)
                *reinterpret_cast<uint4*>(sb_p + p * S::kBBytes + off) = o[p];
            }
          }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&sempty[ss]);  // the staging slot may be reloaded
          if (leader) mbar_arrive(&full[s]);
          else mbar_arrive_remote(full_leader0 + 8u * s);
        }
      }
    }
  } else {
    // ---------------- epilogue (warps 8..15, both CTAs) ----------------
    regs_inc<kRegsHigh>();
    const int q = warp & 3;
    const int h = (warp - 8) >> 2;
    constexpr int COLS = BN / 2;
    uint32_t ch = 0;
    bool ok = true;
    const uint32_t tempty_leader0 = map_to_rank(smem_u32(&tempty[0]), 0);
    for (int t = pair; t < num_tiles && ok; t += pairs) {
      const TileWork w = tiles.get(t);
      const int nchunks = (w.KT + run.chunk_ktiles - 1) / run.chunk_ktiles;
      float sum[COLS];
#pragma unroll
      for (int i = 0; i < COLS; ++i) sum[i] = 0.0f;
      for (int c = 0; c < nchunks; ++c, ++ch) {
        const int buf = ch & 1;
        int got = 0;
        if (lane == 0) got = wait_bounded_sleep(&tfull[buf], (ch >> 1) & 1, abort_flag, lim);
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!got) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem_base + ((uint32_t)(32 * q) << 16) + buf * BN + h * COLS;
#pragma unroll
        for (int j = 0; j < COLS / 16; ++j) {
          float vv[16];
          tmem_ld16(taddr + 16 * j, vv);
#pragma unroll
          for (int i = 0; i < 16; ++i) sum[16 * j + i] += vv[i];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_remote(tempty_leader0 + 8u * buf);
      }
      if (!ok) break;
      const int col0 = w.n0 + h * COLS;
      int* wexp = col_exp + (warp - 8) * COLS;
      if constexpr (SCALED) {
        __syncwarp();
#pragma unroll
        for (int i = lane; i < COLS; i += 32)
          wexp[i] = pow2_exp_of_bits(w.colmax[min(col0 + i, w.N - 1)]);
        __syncwarp();
      }
      store_rows_transposed<COLS, SCALED>(sum, w, w.m0 + kBM * (int)rank + 32 * q, col0, lane,
                                          wexp);
    }
  }

  // Every role leaves its loop (normally or through bounded aborts). After an
  // abort, give in-flight tensor-core work a bounded moment; then the pair
  // synchronises and releases its tensor memory together.
  __syncthreads();
  if (*abort_flag) {
    const unsigned long long t0 = globaltimer();
    while (globaltimer() - t0 < 2000000ull) {
    }
  }
  tc_fence_before();
  cluster_sync();
  if (warp == 0) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base),
                 "r"(S::kAllocCols));
  }
}

}  // namespace hbsg
