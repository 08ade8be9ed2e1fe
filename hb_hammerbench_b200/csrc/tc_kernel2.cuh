// Split-BF16 tensor-core GEMM body for CTA pairs (tcgen05 cta_group::2).
//
// A cluster of two CTAs on neighbouring SMs computes a 256 x BN output tile
// with one tcgen05.mma.cta_group::2 per product and k-step (M = 256), issued
// by the pair's leader (cluster rank 0):
//   - CTA r holds rows [128r, 128r + 128) of the A tile and rows
//     [BN/2 * r, BN/2 * (r + 1)) of the B^T tile (its half of N) in its own
//     shared memory, at the same offsets in both CTAs; the instruction reads
//     both halves. Per SM this moves 128 + BN/2 operand rows per k-step
//     instead of 128 + BN for a single-CTA 128 x BN tile, which is what bounds
//     the single-CTA kernel (its shared-memory pipe runs ~84 % busy).
//   - Each CTA's TMA loads its own halves and signals the leader's stage
//     barrier (.cta_group::2 form, addressed through mapa); the leader's producer
//     expects the bytes of both CTAs.
//   - tcgen05.commit multicasts to both CTAs' barriers (smem stage free,
//     accumulator ready); the accumulator of CTA r (its 128 rows x BN
//     columns) lies in its own TMEM, so the epilogue is the single-CTA one.
//   - Epilogue warps of both CTAs release an accumulator buffer by arriving
//     on the leader's barrier (the peer through a cluster address).
// No TMA multicast is used. Every wait is bounded as in the single-CTA body.
#pragma once

#include "tc_kernel.cuh"

namespace hbsg {

HBSG_DEV uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %cluster_ctarank;" : "=r"(r));
  return r;
}

// Address of the same shared-memory offset in CTA `rank` of the cluster.
HBSG_DEV uint32_t map_to_rank(uint32_t saddr, uint32_t rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(saddr), "r"(rank));
  return out;
}

HBSG_DEV void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n"
               "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

HBSG_DEV void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr)
               : "memory");
}

// TMA load into this CTA's shared memory whose completion is counted on the
// leader CTA's barrier at the same offset (`leader_bar`: a cluster address).
HBSG_DEV void tma_load_3d_pair(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                               uint32_t leader_bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(leader_bar)
      : "memory");
}

// The pair MMA, and the commit that arrives (once) on the barrier at this
// offset in both CTAs of the pair when all prior tensor-core work of the
// issuing thread completes; from one elected lane of a converged warp (see
// tc_mma_elect).
HBSG_DEV void tc_mma_pair_elect(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p, e;\n\t.reg .b32 l;\n\t"
      "elect.sync l|e, 0xffffffff;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "@e tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

HBSG_DEV void tc_commit_pair_elect(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b16 m;\n\t.reg .pred e;\n\t.reg .b32 l;\n\t"
      "elect.sync l|e, 0xffffffff;\n\t"
      "mov.b16 m, 3;\n\t"
      "@e tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], m;\n\t}\n" ::"r"(smem_u32(bar))
      : "memory");
}

template <int P, int BN, int STAGES>
struct TcPairShape {
  static constexpr int kABytes = kBM * kBK * 2;         // 128 rows of one part
  static constexpr int kBBytes = (BN / 2) * kBK * 2;    // this CTA's half of B, one part
  static constexpr int kStageBytes = P * (kABytes + kBBytes);
  static constexpr int kAllocCols = 2 * BN <= 256 ? 256 : 512;
  static constexpr int kBarBytes = 8 * (2 * STAGES + 4) + 16;
  static constexpr int kColExpBytes = 8 * 4 * (BN / 2);
  static constexpr int kSmemBytes = 1024 + STAGES * kStageBytes + kBarBytes + kColExpBytes;
  static_assert(kSmemBytes <= 232448, "shared memory");
  static_assert(BN % 32 == 0 && BN >= 64 && BN <= 256, "pair UMMA N");
};

// Tiles for the pair body: TileWork with m0 = first row of the 256-row pair
// tile and n0 = first column of its BN columns.
template <int P, int BN, int STAGES, bool SCALED, class Tiles>
__device__ __forceinline__ void tc_pair_body(const Tiles& tiles, const TcRun& run) {
  using S = TcPairShape<P, BN, STAGES>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* smem = smem_raw + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * S::kStageBytes);
  uint64_t* full = bars;             // leader: both CTAs' loads of a stage
  uint64_t* empty = bars + STAGES;   // each CTA: its stage is free again
  uint64_t* tfull = bars + 2 * STAGES;       // each CTA: accumulator buffer ready
  uint64_t* tempty = bars + 2 * STAGES + 2;  // leader: both CTAs drained the buffer
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* col_exp = reinterpret_cast<int*>(smem + STAGES * S::kStageBytes + S::kBarBytes);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1;
  const int pairs = gridDim.x >> 1;
  const int num_tiles = tiles.count();

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 16);
    }
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
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

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      const uint32_t full0_leader = map_to_rank(smem_u32(&full[0]), 0);
      uint32_t it = 0;
      bool ok = true;
      for (int t = pair; t < num_tiles && ok; t += pairs) {
        const TileWork w = tiles.get(t);
        const int arow = w.m0 + kBM * (int)rank;
        const int brow = w.n0 + (BN / 2) * (int)rank;
        for (int kt = 0; kt < w.KT; ++kt, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!wait_bounded(&empty[s], ph ^ 1, abort_flag, lim)) {
            ok = false;
            break;
          }
          const uint32_t sa = base + s * S::kStageBytes;
          const uint32_t sb = sa + P * S::kABytes;
          if (leader) mbar_arrive_expect_tx(&full[s], 2 * S::kStageBytes);
          const uint32_t lbar = full0_leader + 8u * s;
          tma_load_3d_pair(sa, w.ma, (w.kt0 + kt) * kBK, arow, 0, lbar);
          tma_load_3d_pair(sb, w.mb, (w.kt0 + kt) * kBK, brow, 0, lbar);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (leader CTA only) ----------------
    // The whole warp runs the loop converged and one elected lane issues
    // (tc_mma_elect); a wait passes only when it passed on every lane.
    if (leader) {
      constexpr uint32_t idesc = f16_idesc(2 * kBM, BN);
      uint32_t it = 0, ch = 0;
      bool ok = true;
      for (int t = pair; t < num_tiles && ok; t += pairs) {
        const int KT = tiles.get(t).KT;
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
  } else {
    // ---------------- epilogue (warps 2..9, both CTAs) ----------------
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
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
        if (lane == 0) mbar_arrive_remote(tempty_leader0 + 8u * buf);
      }
      if (!ok) break;
      const int col0 = w.n0 + h * COLS;
      int* wexp = col_exp + (warp - 2) * COLS;
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

  // Both CTAs leave their loops (normally or through bounded aborts). After
  // an abort, give in-flight copies and tensor-core work a bounded moment;
  // then the pair synchronises and releases its tensor memory together.
  __syncthreads();
  if (*abort_flag) {
    const unsigned long long t0 = globaltimer();
    while (globaltimer() - t0 < 2000000ull) {
    }
  }
  tc_fence_before();
  cluster_sync();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base),
                 "r"(S::kAllocCols));
  }
}

}  // namespace hbsg
