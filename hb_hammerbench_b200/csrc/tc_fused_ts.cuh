// Fused-split tensor-core GEMM body with the A operand's BF16 parts in tensor
// memory (tcgen05.mma with A from TMEM, single CTA, sm_100a): the tile for
// narrow outputs (64- or 128-column tiles, e.g. 65536 x 64 x 4096).
//
// Why: with a narrow B tile the shared-memory traffic per MMA flop of the
// CTA-pair fused tiles (tc_fused.cuh) is dominated by A: for 128 rows x 32 k
// of A per k-tile the TMA writes 16 KB of FP32, the converters read it and
// write 24 KB of parts, and the tensor core reads the parts back once per
// product (6 x 8 KB for the 6-product form). Here the A converters split each
// row in registers and store the parts straight into tensor memory
// (tcgen05.st); the MMA reads A from there, so A's shared-memory traffic is
// the TMA write and one read (32 KB per k-tile instead of 88 KB), and the
// tile can run at the HBM rate of streaming A, which is its roofline.
// B (K x N with N small, the same columns for every row tile) is split once
// by the split pass into the workspace (parts[P][N][Kp], 1.5 MB for
// 4096 x 64 in 3 parts) and TMA-loaded in the unfused kernels' layout, rather
// than split again inside every CTA for every row tile it computes.
//
// Pipeline: only B's parts and the TMEM slot must wait for the MMAs that read
// them to complete; the FP32 A staging is free as soon as the converters have
// read it. The two operands therefore have rings of their own, each with its
// own loader thread, so the A loads run ahead of the MMAs in flight. The MMA
// issuer is a whole converged warp with one elected lane issuing (a loop on a
// single lane spent ~70 cycles per N = 64 MMA issued, measured per role, about
// twice the tensor core's time for one: 87 against 122 TFLOP/s for the
// 6-product 65536 x 64 x 4096).
//
// Layouts:
//   - shared memory: the FP32 A staging ring (SA stages of 128 rows x 32 k,
//     128-byte swizzle, TMA) and the B parts ring (SB stages of P x BN rows
//     of 32 bf16 = 64 bytes, 64-byte swizzle, K-major, one 3-D TMA box);
//   - tensor memory: columns [0, 2*BN) the two FP32 accumulator buffers (row
//     m in lane m), then TSTAGES slots of A parts, each P parts x 16 columns:
//     row m in lane m, k-pair (2j, 2j+1) in column j, element 2j in the low
//     half (the kind::f16 A-from-TMEM layout for M = 128).
//
// Arithmetic: the same split (split8), products, product order and TMEM
// drains as every other split-BF16 tile, so results are bit-identical to them
// at the same drain interval.
//
// CTA (512 threads, 16 warps, one CTA per SM):
//   warp 0       lane 0: TMA loads of the FP32 A staging
//   warp 1       TMEM allocation; the MMA issue (one elected lane issues)
//   warp 2       lane 0: TMA loads of the B parts
//   warp 3       no role
//   warps 4-11   A converters: thread = row 32 (warp % 4) + lane; warps 4-7
//                convert the even k-tiles, warps 8-11 the odd ones, so one
//                group's loads overlap the other's stores
//   warps 12-15  epilogue (TMEM lane quadrant warp % 4, all BN columns)
// Every wait is bounded as in the other tensor-core bodies. The TMA loads use
// no cluster multicast.
#pragma once

#include "tc_fused.cuh"

namespace hbsg {

// (parts, BN, A staging stages, B parts stages, TMEM A slots)
#define HBSG_FUSED_TS_TILE_LIST(X) \
  X(3, 64, 6, 8, 8)                \
  X(2, 64, 8, 8, 12)               \
  X(3, 128, 4, 5, 4)               \
  X(2, 128, 6, 6, 8)

static constexpr int kTsThreads = 512;
static constexpr int kTsAGroups = 2;  // A converter groups of 4 warps, alternating k-tiles
// Tiles wider than 64 columns: the epilogue warpgroup holds BN FP32 sums per
// thread, so setmaxnreg moves registers to it from the other three
// warpgroups (3 x 128 x 112 + 128 x 176 = 65536, the block's launch
// allotment of 512 threads x 128).
static constexpr int kTsRegsLow = 112;
static constexpr int kTsRegsHigh = 176;
static_assert(3 * 128 * kTsRegsLow + 128 * kTsRegsHigh == 65536, "register split");

template <int P, int BN, int SA, int SB, int TSTAGES>
struct TcTsShape {
  static constexpr int kSABytes = kBM * kBK * 4;  // one FP32 A staging stage
  static constexpr int kBPart = BN * kBK * 2;     // one B part of one k-tile
  static constexpr int kSBBytes = P * kBPart;     // one B parts stage
  static constexpr int kBRingOff = SA * kSABytes;
  static constexpr int kACols = P * (kBK / 2);  // TMEM columns of one slot
  static constexpr int kAColBase = 2 * BN;
  static constexpr int kTmemCols = kAColBase + TSTAGES * kACols;
  static constexpr int kAllocCols = kTmemCols <= 32 ? 32 : kTmemCols <= 64 ? 64 : kTmemCols <= 128 ? 128 : kTmemCols <= 256 ? 256 : 512;
  static constexpr int kBarBytes = 8 * (2 * SA + 2 * SB + 2 * TSTAGES + 4) + 16;
  static constexpr int kColExpBytes = 4 * 4 * BN;  // 4 epilogue warps x BN column exponents
  static constexpr int kBarOff = kBRingOff + SB * kSBBytes;
  static constexpr int kSmemBytes = 1024 + kBarOff + kBarBytes + kColExpBytes;
  static_assert(kSmemBytes <= 232448, "shared memory");
  static_assert(kTmemCols <= 512, "tensor memory");
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "UMMA N (M = 128) and 32-column stores");
  static_assert(TSTAGES % kTsAGroups == 0 && SA % kTsAGroups == 0,
                "each converter group owns whole TMEM slots and staging stages");
  static_assert(kSABytes % 1024 == 0 && kBRingOff % 1024 == 0 && kBPart % 512 == 0,
                "staging keeps the 128-byte swizzle's 1024-byte and the parts' 512-byte alignment");
};

// 32 lanes x 8 columns of 32-bit TMEM from 8 registers per thread (thread i
// writes lane quadrant base + i).
HBSG_DEV void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
      : "memory");
}

HBSG_DEV void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// D (TMEM) (+)= A (TMEM, K-major) x B (shared memory descriptor), M = 128,
// called by a whole converged warp: elect.sync picks the one lane that
// issues it.
HBSG_DEV void tc_mma_ts_elect(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                              uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p, e;\n\t.reg .b32 l;\n\t"
      "elect.sync l|e, 0xffffffff;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

template <int P, int BN, int SA, int SB, int TSTAGES, bool SCALED, class Tiles>
__device__ __forceinline__ void tc_fused_ts_body(const Tiles& tiles, const TcRun& run) {
  using S = TcTsShape<P, BN, SA, SB, TSTAGES>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* smem = smem_raw + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::kBarOff);
  uint64_t* sfull = bars;              // TMA: the A staging stage has landed
  uint64_t* sempty = bars + SA;        // A converters: the A staging stage has been read
  uint64_t* bfull = sempty + SA;       // TMA: the B parts stage has landed
  uint64_t* bempty = bfull + SB;       // MMA: the B parts stage has been read
  uint64_t* afull = bempty + SB;       // A converters: the slot's A parts are in TMEM
  uint64_t* aempty = afull + TSTAGES;  // MMA: the slot's A parts have been read
  uint64_t* tfull = aempty + TSTAGES;  // MMA: accumulator buffer complete
  uint64_t* tempty = tfull + 2;        // epilogue: accumulator buffer drained
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* col_exp = reinterpret_cast<int*>(smem + S::kBarOff + S::kBarBytes);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int num_tiles = tiles.count();

  if (threadIdx.x == 0) {
    for (int s = 0; s < SA; ++s) {
      mbar_init(&sfull[s], 1);
      mbar_init(&sempty[s], 4);  // the 4 warps of the stage's converter group
    }
    for (int s = 0; s < SB; ++s) {
      mbar_init(&bfull[s], 1);
      mbar_init(&bempty[s], 1);
    }
    for (int j = 0; j < TSTAGES; ++j) {
      mbar_init(&afull[j], 4);
      mbar_init(&aempty[j], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
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

  // each role's code sits inside the branch that set its register count
  constexpr bool kSplitRegs = BN > 64;
  if constexpr (kSplitRegs) {
    if (warp < 12) regs_dec<kTsRegsLow>();
  }
  if (warp == 0 || warp == 2) {
    // ---------------- TMA loads: A staging (warp 0), B parts (warp 2) ----------------
    // A: 128 rows x 32 k of FP32 (rows and k beyond the matrix arrive as
    // zeros); B: the k-tile's 32 k of BN rows of every part
    if (lane == 0) {
      const bool a_role = warp == 0;
      uint32_t it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
        const TileWork w = tiles.get(t);
        const CUtensorMap* map = a_role ? w.ma : w.mb;
        if (t == (int)blockIdx.x)
          asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
        for (int kt = 0; kt < w.KT; ++kt, ++it) {
          const int k0 = (w.kt0 + kt) * kBK;
          if (a_role) {
            const int s = it % SA;
            if (!wait_bounded_hint(&sempty[s], ((it / SA) & 1) ^ 1, abort_flag, lim)) {
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&sfull[s], S::kSABytes);
            tma_load_2d(base + s * S::kSABytes, map, k0, w.m0, &sfull[s]);
          } else {
            const int s = it % SB;
            if (!wait_bounded_hint(&bempty[s], ((it / SB) & 1) ^ 1, abort_flag, lim)) {
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&bfull[s], S::kSBBytes);
            tma_load_3d(base + S::kBRingOff + s * S::kSBBytes, map, k0, w.n0, 0, &bfull[s]);
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    // The loop runs converged on all 32 lanes of the warp, so its operands
    // (TMEM addresses, descriptors) are warp-uniform, and one elected lane
    // issues each MMA and commit (a loop on a single lane measured ~70
    // cycles per N = 64 MMA issued, about twice the tensor core's time for
    // one). Every lane takes the bounded waits; a wait counts as passed only
    // when it passed on all lanes.
    constexpr uint32_t idesc = f16_idesc(kBM, BN);
    uint32_t it = 0, ch = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
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
          const int sb = it % SB;
          const int j = it % TSTAGES;
          const bool got = wait_bounded(&bfull[sb], (it / SB) & 1, abort_flag, lim) &&
                           wait_bounded(&afull[j], (it / TSTAGES) & 1, abort_flag, lim);
          if (!__all_sync(0xffffffffu, got)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t bs = base + S::kBRingOff + sb * S::kSBBytes;
          const uint32_t ta = tmem_base + S::kAColBase + j * S::kACols;
#pragma unroll
          for (int ks = 0; ks < kBK / 16; ++ks) {
#pragma unroll
            for (int q = 0; q < Products<P>::n; ++q) {
              const uint64_t bd = sw64_desc(bs + Products<P>::b(q) * S::kBPart + ks * 32);
              tc_mma_ts_elect(d, ta + Products<P>::a(q) * (kBK / 2) + ks * 8, bd, idesc,
                              first ? 0u : 1u);
              first = false;
            }
          }
          tc_commit_elect(&bempty[sb]);
          tc_commit_elect(&aempty[j]);
        }
        if (ok) tc_commit_elect(&tfull[buf]);
      }
    }
  } else if (warp >= 4 && warp < 4 + 4 * kTsAGroups) {
    // ---------------- A converters ----------------
    // thread = tile row 32 q + lane (its TMEM lane); group g converts the
    // k-tiles it with it % 2 == g: eight 16-byte staging loads (then the
    // staging stage is released), the split of 32 values, P x 16 TMEM columns
    const int q = warp & 3;
    const int g = (warp - 4) >> 2;
    const int r = 32 * q + lane;
    const uint32_t trow = tmem_base + ((uint32_t)(32 * q) << 16) + S::kAColBase;
    int ex = 0;
    uint32_t it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
      const TileWork w = tiles.get(t);
      if constexpr (SCALED) {
        const int m = w.m0 + r;
        ex = m < w.M ? exp_from_maxbits(w.rowmax[m]) : 0;
      }
      for (int kt = 0; kt < w.KT; ++kt, ++it) {
        if ((int)(it % kTsAGroups) != g) continue;
        const int s = it % SA;
        const int j = it % TSTAGES;
        if (!wait_bounded_hint(&sfull[s], (it / SA) & 1, abort_flag, lim)) {
          ok = false;
          break;
        }
        const uint8_t* fa = smem + s * S::kSABytes;
        float v[4][8];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float4 a0 = *reinterpret_cast<const float4*>(fa + sw128_offset(r, 2 * u));
          const float4 a1 = *reinterpret_cast<const float4*>(fa + sw128_offset(r, 2 * u + 1));
          v[u][0] = a0.x; v[u][1] = a0.y; v[u][2] = a0.z; v[u][3] = a0.w;
          v[u][4] = a1.x; v[u][5] = a1.y; v[u][6] = a1.z; v[u][7] = a1.w;
        }
        uint4 o[4][P];
#pragma unroll
        for (int u = 0; u < 4; ++u) split8<P, SCALED>(v[u], ex, o[u]);
        // the staging values are in registers (the split used them): the
        // stage may be reloaded by the TMA
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sempty[s]);
        // the slot is free once the MMAs that read it (k-tile it - TSTAGES)
        // completed
        if (!wait_bounded_hint(&aempty[j], ((it / TSTAGES) & 1) ^ 1, abort_flag, lim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t ta = trow + j * S::kACols;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
#pragma unroll
          for (int p = 0; p < P; ++p) {
            const uint32_t reg[8] = {o[2 * h][p].x,     o[2 * h][p].y,     o[2 * h][p].z,
                                     o[2 * h][p].w,     o[2 * h + 1][p].x, o[2 * h + 1][p].y,
                                     o[2 * h + 1][p].z, o[2 * h + 1][p].w};
            tmem_st8(ta + p * (kBK / 2) + h * (kBK / 4), reg);
          }
        }
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&afull[j]);
      }
    }
  } else if (warp >= 12) {
    // ---------------- epilogue (warps 12-15) ----------------
    if constexpr (kSplitRegs) regs_inc<kTsRegsHigh>();
    const int q = warp & 3;
    uint32_t ch = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
      const TileWork w = tiles.get(t);
      const int nchunks = (w.KT + run.chunk_ktiles - 1) / run.chunk_ktiles;
      float sum[BN];
#pragma unroll
      for (int i = 0; i < BN; ++i) sum[i] = 0.0f;
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
        const uint32_t taddr = tmem_base + ((uint32_t)(32 * q) << 16) + buf * BN;
#pragma unroll
        for (int jj = 0; jj < BN / 16; ++jj) {
          float vv[16];
          tmem_ld16(taddr + 16 * jj, vv);
#pragma unroll
          for (int i = 0; i < 16; ++i) sum[16 * jj + i] += vv[i];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[buf]);
      }
      if (!ok) break;
      int* wexp = col_exp + q * BN;
      if constexpr (SCALED) {
        __syncwarp();
#pragma unroll
        for (int i = lane; i < BN; i += 32) wexp[i] = pow2_exp_of_bits(w.colmax[min(w.n0 + i, w.N - 1)]);
        __syncwarp();
      }
      store_rows_transposed<BN, SCALED>(sum, w, w.m0 + 32 * q, w.n0, lane, wexp);
    }
  }

  // Every role leaves its loop (normally or through a bounded abort). After
  // an abort, give in-flight tensor-core work a bounded moment before the
  // tensor memory is released.
  tc_fence_before();
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
