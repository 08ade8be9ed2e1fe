// FP32 SIMT (FFMA) SGEMM for sm_100a.
//
// Replaces the HammerBench device kernel (apps/sgemm/kernel.cpp:279-333).
// The reference gives each tile of a 16x8 tile group 16x16 output blocks
// round-robin (kernel.cpp:300-302), streams 16x16 blocks of A and B from DRAM
// into scratchpad (load_block, kernel.cpp:36-109) and runs a 4x4
// register-blocked fmaf chain over k (compute_block, kernel.cpp:186-275).
// Here one CTA owns a BM x BN output tile; A and B tiles stream from HBM into
// a STAGES-deep shared-memory ring with 16-byte cp.async (zero-filled at the
// matrix edges), and each thread owns a TM x TN register block that it
// updates with one fused multiply-add per k in ascending k. The arithmetic
// per output element is therefore exactly the reference device kernel's:
// acc = 0.0f; for k = 0..K-1: acc = fmaf(a[m][k], b[k][n], acc).
//
// Layout in shared memory (per stage):
//   A: BM rows x (BK + 4) floats, k contiguous. The +4 pad makes 8
//      consecutive rows fall in 8 distinct 16-byte bank groups, so the
//      8 distinct rows read by a quarter-warp with LDS.128 are conflict-free.
//   B: BK rows x BN floats, n contiguous.
// Thread layout inside a warp: lane = tn*8 + tm (tm < 8, tn < 4). Thread
// (tm, tn) owns rows {tm + 8i} and columns {16j + 4tn + c} of its warp tile:
// a quarter-warp reads 8 distinct A rows (no conflict) and one B float4
// (broadcast); the whole warp reads 64 contiguous bytes of B.
#include "ffma_kernel.cuh"

namespace hbsg {

template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool VEC, bool PAIR,
          bool TA = false, bool TB = false>
__global__ void __launch_bounds__(FfmaShape<BM, BN, BK, WM, WN, STAGES>::kThreads,
                                  FfmaShape<BM, BN, BK, WM, WN, STAGES>::kMinBlocks)
    ffma_sgemm_kernel(FfmaParams p) {
  extern __shared__ __align__(16) float smem[];
  // Rasterised tile order: groups of `raster` tile rows, column-major inside
  // a group, so CTAs resident at the same time share A and B strips in L2.
  const int t = blockIdx.x;
  const int group_span = p.raster * p.tiles_n;
  const int group = t / group_span;
  const int first_m = group * p.raster;
  const int gm = min(p.raster, p.tiles_m - first_m);
  const int in_group = t - group * group_span;
  const int m0 = (first_m + in_group % gm) * BM;
  const int n0 = (in_group / gm) * BN;
  const int batch = blockIdx.z;
  const int split = blockIdx.y;
  const int k_begin = split * p.k_per_split;
  const int k_end = min(p.K, k_begin + p.k_per_split);
  float* C;
  long ldc;
  bool vec_store;
  if (p.splits > 1) {  // split-K slices go to the partial buffer
    C = p.partial + ((long)batch * p.splits + split) * (long)p.M * p.N;
    ldc = p.N;
    vec_store = (p.N & 3) == 0;
  } else {
    C = p.C + batch * p.strideC;
    ldc = p.ldc;
    vec_store = p.vec_store;
  }
  ffma_tile<BM, BN, BK, WM, WN, STAGES, VEC, PAIR, TA, TB>(p.A + batch * p.strideA, p.lda,
                                                   p.B + batch * p.strideB, p.ldb, p.M, p.N,
                                                   k_begin, k_end, m0, n0, C, ldc, vec_store, smem);
}

// Fixed-order reduction of split-K partial slices: C = ((p0 + p1) + p2) + ...
__global__ void splitk_reduce_kernel(const float* __restrict__ partial, float* __restrict__ C,
                                     int M, int N, long ldc, long strideC, int splits, int batches) {
  const long MN = (long)M * N;
  const long total = MN * batches;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const long b = idx / MN;
    const long e = idx - b * MN;
    const float* src = partial + b * splits * MN + e;
    float s = src[0];
    for (int k = 1; k < splits; ++k) s += src[k * MN];
    const long r = e / N;
    const long c = e - r * N;
    C[b * strideC + r * ldc + c] = s;
  }
}

// ---------------------------------------------------------------------------
// Tile table and launcher.

struct FfmaEntry {
  int bm, bn, bk, wm, wn, stages;
  int threads, smem, per_sm;
  cudaError_t (*launch)(const FfmaParams&, dim3, cudaStream_t, bool vec);
};

template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool PAIR>
static cudaError_t launch_ffma(const FfmaParams& p, dim3 grid, cudaStream_t st, bool vec) {
  using S = FfmaShape<BM, BN, BK, WM, WN, STAGES>;
  auto kv = ffma_sgemm_kernel<BM, BN, BK, WM, WN, STAGES, true, PAIR>;
  auto ks = ffma_sgemm_kernel<BM, BN, BK, WM, WN, STAGES, false, PAIR>;
  auto k = vec ? kv : ks;
  static uint64_t mask_v = 0, mask_s = 0;
  if (!set_smem_once(reinterpret_cast<const void*>(k), S::kSmemBytes, vec ? &mask_v : &mask_s))
    return cudaErrorInvalidValue;
  k<<<grid, S::kThreads, S::kSmemBytes, st>>>(p);
  return cudaGetLastError();
}

// Transposed-operand kernels (4-byte copy path) for a tile shape.
template <int BM, int BN, int BK, int WM, int WN, int STAGES>
static cudaError_t launch_ffma_trans(const FfmaParams& p, dim3 grid, cudaStream_t st, int ta,
                                     int tb) {
  using S = FfmaShape<BM, BN, BK, WM, WN, STAGES>;
  auto k10 = ffma_sgemm_kernel<BM, BN, BK, WM, WN, STAGES, false, true, true, false>;
  auto k01 = ffma_sgemm_kernel<BM, BN, BK, WM, WN, STAGES, false, true, false, true>;
  auto k11 = ffma_sgemm_kernel<BM, BN, BK, WM, WN, STAGES, false, true, true, true>;
  auto k = ta && tb ? k11 : ta ? k10 : k01;
  static uint64_t masks[3] = {0, 0, 0};
  const int slot = ta && tb ? 2 : ta ? 0 : 1;
  if (!set_smem_once(reinterpret_cast<const void*>(k), S::kSmemBytes, &masks[slot]))
    return cudaErrorInvalidValue;
  k<<<grid, S::kThreads, S::kSmemBytes, st>>>(p);
  return cudaGetLastError();
}

#define HBSG_FFMA_ENTRY(BM, BN, BK, WM, WN, ST, PAIR)                                   \
  FfmaEntry {                                                                           \
    BM, BN, BK, WM, WN, ST, FfmaShape<BM, BN, BK, WM, WN, ST>::kThreads,                \
        FfmaShape<BM, BN, BK, WM, WN, ST>::kSmemBytes,                                  \
        FfmaShape<BM, BN, BK, WM, WN, ST>::kMinBlocks,                                  \
        &launch_ffma<BM, BN, BK, WM, WN, ST, PAIR>                                      \
  }

static const FfmaEntry kFfmaTiles[] = {
    HBSG_FFMA_ENTRY(128, 128, 16, 64, 64, 4, true),   // 1: 4 warps, 2 CTAs/SM, packed FMA
    HBSG_FFMA_ENTRY(128, 256, 16, 64, 64, 4, true),   // 2: 8 warps, packed FMA
    HBSG_FFMA_ENTRY(64, 64, 16, 32, 32, 4, true),     // 3: 4 warps, small problems
    HBSG_FFMA_ENTRY(128, 64, 16, 64, 32, 4, true),    // 4: 4 warps, narrow N
    HBSG_FFMA_ENTRY(128, 256, 32, 64, 64, 3, true),   // 5: 8 warps, deeper K tile
    HBSG_FFMA_ENTRY(256, 128, 16, 64, 64, 4, true),   // 6: 8 warps, tall
    HBSG_FFMA_ENTRY(128, 128, 32, 64, 64, 3, true),   // 7: 4 warps, deeper K tile
    HBSG_FFMA_ENTRY(128, 128, 16, 64, 64, 4, false),  // 8: as 1 with scalar FMA
    HBSG_FFMA_ENTRY(128, 128, 16, 64, 32, 4, true),   // 9: 8 warps, 8x8 per thread
};
static constexpr int kNumFfmaTiles = sizeof(kFfmaTiles) / sizeof(kFfmaTiles[0]);

int ffma_num_tiles() { return kNumFfmaTiles; }

bool ffma_tile_info(int idx, hbsg_tile_info* out) {
  if (idx < 0 || idx >= kNumFfmaTiles) return false;
  const FfmaEntry& e = kFfmaTiles[idx];
  out->variant_class = 0;
  out->bm = e.bm;
  out->bn = e.bn;
  out->bk = e.bk;
  out->threads = e.threads;
  out->smem_bytes = e.smem;
  out->parts = 0;
  return true;
}

// Pick the tile with the best estimated SM utilisation, preferring the large
// tile when the wave count is high (fewer bytes per flop).
int ffma_pick_tile(int M, int N, int K, int batch, int num_sms) {
  (void)K;
  double best = -1.0;
  int best_idx = 0;
  const int cand[] = {0, 1, 3, 2};  // 128x128, 128x256, 128x64, 64x64
  for (int idx : cand) {
    const FfmaEntry& e = kFfmaTiles[idx];
    const long tiles = (long)((M + e.bm - 1) / e.bm) * ((N + e.bn - 1) / e.bn) * batch;
    const int per_sm = e.per_sm;
    const double slots = (double)num_sms * per_sm;
    const double waves = tiles / slots;
    const double eff = waves / ceil(waves);  // tail efficiency
    // work per tile relative to the biggest tile: bigger tiles amortise loads
    // measured at 8192^3: 128x128 (2 CTAs/SM) is the fastest shape
    const double tile_eff = (e.bm * e.bn == 128 * 128) ? 1.0 : (e.bm * e.bn >= 128 * 256 ? 0.96 : 0.85);
    const double fill = fmin(1.0, tiles / slots);
    // share of the tile's rows and columns inside the matrix (a 128-wide tile
    // on N = 64 computes twice the columns it stores)
    const double inside = (double)M / (((M + e.bm - 1) / e.bm) * e.bm) *
                          ((double)N / (((N + e.bn - 1) / e.bn) * e.bn));
    const double score = eff * tile_eff * (fill < 1.0 ? fill : 1.0) * inside;
    if (score > best + 1e-9) {
      best = score;
      best_idx = idx;
    }
  }
  return best_idx;
}

size_t ffma_workspace_bytes(int M, int N, int batch, int splits) {
  return splits > 1 ? (size_t)M * N * batch * splits * sizeof(float) : 0;
}

cudaError_t ffma_launch(int tile_idx, FfmaParams p, int batch, int sms, cudaStream_t st, int ta,
                        int tb) {
  // transposed operands: 128 x 128 or 64 x 64 tiles (the closest of the two)
  if (ta || tb) {
    const FfmaEntry& big = kFfmaTiles[0];
    const FfmaEntry& e0 = kFfmaTiles[tile_idx];
    tile_idx = (e0.bm * e0.bn >= big.bm * big.bn) ? 0 : 2;
  }
  const FfmaEntry& e = kFfmaTiles[tile_idx];
  p.tiles_m = (p.M + e.bm - 1) / e.bm;
  p.tiles_n = (p.N + e.bn - 1) / e.bn;
  if (p.raster <= 0) p.raster = 8;
  if (p.splits < 1) p.splits = 1;
  if (p.splits > 1) {
    // K slices are whole BK tiles.
    int per = (p.K + p.splits - 1) / p.splits;
    per = (per + e.bk - 1) / e.bk * e.bk;
    p.k_per_split = per;
    p.splits = (p.K + per - 1) / per;
  } else {
    p.k_per_split = p.K;
  }
  const bool vec = !ta && !tb && ((p.lda & 3) == 0) && ((p.ldb & 3) == 0) &&
                   ((reinterpret_cast<uintptr_t>(p.A) & 15) == 0) &&
                   ((reinterpret_cast<uintptr_t>(p.B) & 15) == 0) && ((p.strideA & 3) == 0) &&
                   ((p.strideB & 3) == 0);
  p.vec_store = ((p.ldc & 3) == 0) && ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0) &&
                ((p.strideC & 3) == 0);
  dim3 grid((unsigned)(p.tiles_m * p.tiles_n), (unsigned)p.splits, (unsigned)batch);
  cudaError_t err;
  if (ta || tb) {
    err = tile_idx == 0 ? launch_ffma_trans<128, 128, 16, 64, 64, 4>(p, grid, st, ta, tb)
                        : launch_ffma_trans<64, 64, 16, 32, 32, 4>(p, grid, st, ta, tb);
  } else {
    err = e.launch(p, grid, st, vec);
  }
  if (err != cudaSuccess || p.splits == 1) return err;
  return splitk_reduce(p.partial, p.C, p.M, p.N, p.ldc, p.strideC, p.splits, batch, sms, st);
}

cudaError_t splitk_reduce(const float* partial, float* C, int M, int N, long ldc, long strideC,
                          int splits, int batches, int sms, cudaStream_t st) {
  const long total = (long)M * N * batches;
  const long nb = (total + 255) / 256;
  const long cap = (long)sms * 16;
  const int blocks = (int)(nb < cap ? nb : cap);
  splitk_reduce_kernel<<<blocks, 256, 0, st>>>(partial, C, M, N, ldc, strideC, splits, batches);
  return cudaGetLastError();
}

// Split count for the FFMA kernel: the requested count, or (0) enough K
// slices to fill every SM when the output has too few tiles, keeping at least
// 16 k-tiles (256 of K) per slice.
int ffma_pick_splits(int tile_idx, int M, int N, int K, int batch, int requested, int sms) {
  if (requested > 0) return requested;
  const FfmaEntry& e = kFfmaTiles[tile_idx];
  const long tiles = (long)((M + e.bm - 1) / e.bm) * ((N + e.bn - 1) / e.bn) * batch;
  const long slots = (long)sms * e.per_sm;
  if (tiles * 2 > slots) return 1;
  const long by_k = K / (16 * e.bk) > 1 ? K / (16 * e.bk) : 1;
  const long s = (slots + tiles - 1) / tiles;
  return (int)(s < by_k ? s : by_k);
}

}  // namespace hbsg
