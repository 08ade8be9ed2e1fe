// Launches of the fused-split tensor-core GEMM: C = A*B for FP32 A (M x K)
// and B (K x N), row-major, with the BF16 split done inside the product
// kernel, on CTA pairs (256 x BN output tiles, tc_fused.cuh) or, for narrow
// outputs, on single CTAs that keep A's parts in tensor memory (128 x BN
// tiles, tc_fused_ts.cuh). Each header describes its design.
//
// Work items are (output tile, K slice) pairs in rasterised tile order, as for
// the unfused kernel (tc_gemm.cu): with K slices each slice writes an FP32
// partial to the workspace, reduced in fixed order afterwards. The scaled
// forms read per-row / per-column maxima that a max pass computes first
// (split_bf16.cu); nothing else is staged in HBM. The kernel reads A and B
// through two FP32 TMA tensor maps, so both need 16-byte aligned bases and
// row strides (lda, ldb multiples of 4 floats).
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "tc_fused_ts.cuh"

namespace hbsg {

struct FusedTiles {
  static constexpr bool kInlineSplit = false;
  const FusedParams* p;
  const CUtensorMap* ma;  // FP32 A, box {32, 128}
  const CUtensorMap* mb;  // FP32 B, box {BN/2, 32} (A-in-TMEM tiles: B's parts, box {32, BN, P})
  __device__ __forceinline__ int count() const { return p->num_tiles * p->splits; }
  template <int BN, int TBM>
  __device__ __forceinline__ TileWork get_bn(int item) const {
    const int slice = item / p->num_tiles;
    const int t = item - slice * p->num_tiles;
    const int span = p->raster * p->tiles_n;
    const int g = t / span;
    const int first = g * p->raster;
    const int gm = min(p->raster, p->tiles_m - first);
    const int in = t - g * span;
    TileWork w;
    w.prob = 0;
    w.ready_target = 0;
    w.ma = ma;
    w.mb = mb;
    w.M = p->M;
    w.N = p->N;
    w.m0 = (first + in % gm) * TBM;
    w.n0 = (in / gm) * BN;
    const int KT = (p->K + kBK - 1) / kBK;
    w.kt0 = slice * p->kt_per_split;
    w.KT = max(0, min(p->kt_per_split, KT - w.kt0));
    if (p->splits > 1) {
      w.C = p->C + (long)slice * p->M * p->N;
      w.ldc = p->N;
    } else {
      w.C = p->C;
      w.ldc = p->ldc;
    }
    w.rowmax = p->rowmax;
    w.colmax = p->colmax;
    w.A = p->A;
    w.B = p->B;
    w.lda = p->lda;
    w.ldb = p->ldb;
    w.K = p->K;
    return w;
  }
};

template <int BN, int TBM = 2 * kBM>
struct FusedTilesBN : FusedTiles {
  __device__ __forceinline__ TileWork get(int t) const { return get_bn<BN, TBM>(t); }
};

template <int P, int BN, int STAGES, int SSTAGES, bool SCALED>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kFusedThreads, 1)
    tc_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ FusedParams p, const TcRun run) {
  FusedTilesBN<BN> tiles;
  tiles.p = &p;
  tiles.ma = &tmA;
  tiles.mb = &tmB;
  tc_fused_body<P, BN, STAGES, SSTAGES, SCALED>(tiles, run);
}

// A-in-TMEM form: 128 x BN tiles on single CTAs (tc_fused_ts.cuh).
template <int P, int BN, int SA, int SB, int TSTAGES, bool SCALED>
__global__ void __launch_bounds__(kTsThreads, 1)
    tc_fused_ts_kernel(const __grid_constant__ CUtensorMap tmA,
                       const __grid_constant__ CUtensorMap tmB,
                       const __grid_constant__ FusedParams p, const TcRun run) {
  FusedTilesBN<BN, kBM> tiles;
  tiles.p = &p;
  tiles.ma = &tmA;
  tiles.mb = &tmB;
  tc_fused_ts_body<P, BN, SA, SB, TSTAGES, SCALED>(tiles, run);
}

template <int P, int BN, int STAGES, int SSTAGES>
static const void* fused_kernel_ptr(bool scaled) {
  return scaled ? reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, STAGES, SSTAGES, true>)
                : reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, STAGES, SSTAGES, false>);
}

template <int P, int BN, int STAGES, int SSTAGES>
static cudaError_t launch_fused(const CUtensorMap& a, const CUtensorMap& b, const FusedParams& p,
                                const TcRun& run, int grid, cudaStream_t st, bool scaled) {
  using S = TcFusedShape<P, BN, STAGES, SSTAGES>;
  const void* k = fused_kernel_ptr<P, BN, STAGES, SSTAGES>(scaled);
  static uint64_t masks[2] = {0, 0};
  if (!set_smem_once(k, S::kSmemBytes, &masks[scaled ? 1 : 0])) return cudaErrorInvalidValue;
  static int regs_ok[2] = {0, 0};
  if (!fused_regs_ok(k, &regs_ok[scaled ? 1 : 0])) return cudaErrorInvalidConfiguration;
  if (scaled)
    tc_fused_kernel<P, BN, STAGES, SSTAGES, true><<<grid, kFusedThreads, S::kSmemBytes, st>>>(a, b, p, run);
  else
    tc_fused_kernel<P, BN, STAGES, SSTAGES, false><<<grid, kFusedThreads, S::kSmemBytes, st>>>(a, b, p, run);
  return cudaGetLastError();
}

template <int P, int BN, int STAGES, int SSTAGES>
static int fused_clusters_of(bool scaled) {
  using S = TcFusedShape<P, BN, STAGES, SSTAGES>;
  const void* k = fused_kernel_ptr<P, BN, STAGES, SSTAGES>(scaled);
  static uint64_t masks[2] = {0, 0};
  if (!set_smem_once(k, S::kSmemBytes, &masks[scaled ? 1 : 0])) return 0;
  return fused_resident_clusters(k, S::kSmemBytes);
}

template <int P, int BN, int SA, int SB, int TSTAGES>
static const void* fused_ts_kernel_ptr(bool scaled) {
  return scaled ? reinterpret_cast<const void*>(&tc_fused_ts_kernel<P, BN, SA, SB, TSTAGES, true>)
                : reinterpret_cast<const void*>(&tc_fused_ts_kernel<P, BN, SA, SB, TSTAGES, false>);
}

template <int P, int BN, int SA, int SB, int TSTAGES>
static cudaError_t launch_fused_ts(const CUtensorMap& a, const CUtensorMap& b,
                                   const FusedParams& p, const TcRun& run, int grid,
                                   cudaStream_t st, bool scaled) {
  using S = TcTsShape<P, BN, SA, SB, TSTAGES>;
  const void* k = fused_ts_kernel_ptr<P, BN, SA, SB, TSTAGES>(scaled);
  static uint64_t masks[2] = {0, 0};
  if (!set_smem_once(k, S::kSmemBytes, &masks[scaled ? 1 : 0])) return cudaErrorInvalidValue;
  if (BN > 64) {  // the body's setmaxnreg split needs exactly 128 registers at launch
    static int regs_ok[2] = {0, 0};
    if (!fused_regs_ok(k, &regs_ok[scaled ? 1 : 0])) return cudaErrorInvalidConfiguration;
  }
  if (scaled)
    tc_fused_ts_kernel<P, BN, SA, SB, TSTAGES, true><<<grid, kTsThreads, S::kSmemBytes, st>>>(a, b, p, run);
  else
    tc_fused_ts_kernel<P, BN, SA, SB, TSTAGES, false><<<grid, kTsThreads, S::kSmemBytes, st>>>(a, b, p, run);
  return cudaGetLastError();
}

// Resident CTAs of an A-in-TMEM kernel (0 if unknown).
template <int P, int BN, int SA, int SB, int TSTAGES>
static int fused_ts_ctas_of(bool scaled) {
  using S = TcTsShape<P, BN, SA, SB, TSTAGES>;
  const void* k = fused_ts_kernel_ptr<P, BN, SA, SB, TSTAGES>(scaled);
  static uint64_t masks[2] = {0, 0};
  if (!set_smem_once(k, S::kSmemBytes, &masks[scaled ? 1 : 0])) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTsThreads, S::kSmemBytes) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int sms = current_device_sms(nullptr);
  return sms > 0 ? per_sm * sms : 0;
}

struct FusedEntry {
  int parts, bn, stages, sstages, smem;
  int ts;       // 1: A parts in tensor memory, single-CTA 128-row tiles; 0: CTA pairs, 256 rows
  int bm;       // output rows per tile
  int threads;  // per CTA
  cudaError_t (*launch)(const CUtensorMap&, const CUtensorMap&, const FusedParams&, const TcRun&,
                        int, cudaStream_t, bool);
  int (*slots)(bool);  // concurrently resident work units: clusters of two, or CTAs (ts)
};

#define HBSG_FUSED_ENTRY(P, BN, ST, SST)                                                   \
  FusedEntry{P, BN, ST, SST, TcFusedShape<P, BN, ST, SST>::kSmemBytes, 0, 2 * kBM,        \
             kFusedThreads, &launch_fused<P, BN, ST, SST>, &fused_clusters_of<P, BN, ST, SST>},
#define HBSG_FUSED_TS_ENTRY(P, BN, SA, SB, TST)                                               \
  FusedEntry{P, BN, SA, SB, TcTsShape<P, BN, SA, SB, TST>::kSmemBytes, 1, kBM, kTsThreads,     \
             &launch_fused_ts<P, BN, SA, SB, TST>, &fused_ts_ctas_of<P, BN, SA, SB, TST>},
// CTA-pair tiles first (the grouped plans' fused table, grouped.cu, holds
// these only), then the A-in-TMEM tiles
static const FusedEntry kFused[] = {HBSG_FUSED_TILE_LIST(HBSG_FUSED_ENTRY)
                                    HBSG_FUSED_TS_TILE_LIST(HBSG_FUSED_TS_ENTRY)};
static constexpr int kNumFused = sizeof(kFused) / sizeof(kFused[0]);

int fused_num_tiles() { return kNumFused; }
int fused_tile_parts(int idx) { return kFused[idx].parts; }
int fused_tile_bn(int idx) { return kFused[idx].bn; }
int fused_tile_bm(int idx) { return kFused[idx].bm; }
int fused_tile_ts(int idx) { return kFused[idx].ts; }

bool fused_tile_info(int idx, hbsg_tile_info* out) {
  if (idx < 0 || idx >= kNumFused) return false;
  out->variant_class = 1;
  out->bm = kFused[idx].bm;
  out->bn = kFused[idx].bn;
  out->bk = kBK;
  out->threads = kFused[idx].threads;
  out->smem_bytes = kFused[idx].smem;
  out->parts = kFused[idx].parts;
  return true;
}

// k-tiles the loader prefetches into L2 ahead of its staging loads
// (HBSG_FUSED_L2_AHEAD overrides the default, for tuning; 0 = off).
int fused_l2_ahead() {
  static const int v = [] {
    const char* e = getenv("HBSG_FUSED_L2_AHEAD");
    const int x = e ? atoi(e) : 0;
    return x < 0 ? 0 : x;
  }();
  return v;
}

// Per-CTA k-tile time of each entry in SM cycles at 1.5 GHz, from measured
// kernel times on B200 (4096^3 for the 256-wide pair tiles, 65536x64x4096 for
// the 64-wide ones). Pair tiles: per-role clock64 counters put most of it in
// the converters (the staging, split and part writes share the SM's shared
// memory with the tensor core's operand reads). A-in-TMEM tiles: the MMA issue
// of N = 64 MMAs and the A split.
double fused_ktile_cycles(int idx) {
  const FusedEntry& e = kFused[idx];
  if (e.ts) return e.parts == 3 ? 830.0 : 610.0;
  if (e.bn >= 256) return e.parts == 3 ? 2450.0 : 1950.0;
  return e.parts == 3 ? 1900.0 : 1700.0;
}

// Concurrent work units of an entry on `sms` SMs: clusters of two, or CTAs.
int fused_tile_slots(int idx, int sms) { return kFused[idx].ts ? sms : sms / 2; }

int fused_pick_splits(int idx, int M, int N, int K, int requested, int sms, int* kt_per_split) {
  const FusedEntry& e = kFused[idx];
  const long tiles = (long)((M + e.bm - 1) / e.bm) * ((N + e.bn - 1) / e.bn);
  return tc_slices(tiles, K, fused_tile_slots(idx, sms), requested, kt_per_split);
}

bool fused_operands_ok(const float* A, long lda, const float* B, long ldb) {
  return ((lda & 3) == 0) && ((ldb & 3) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0) &&
         ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
}

bool fused_make_maps(int idx, const float* A, long lda, const float* B, long ldb, int M, int N,
                     int K, void* map_a, void* map_b) {
  if (!fused_operands_ok(A, lda, B, ldb)) return false;
  // B box: this CTA's columns (half the tile on a CTA pair, all of it with ts)
  const int bbox = kFused[idx].ts ? kFused[idx].bn : kFused[idx].bn / 2;
  return tc_make_f32_map(map_a, A, K, M, lda, kBK, kBM, true) &&
         tc_make_f32_map(map_b, B, N, K, ldb, bbox, kBK, false);
}

cudaError_t fused_launch(int idx, FusedParams p, int raster, int chunk_k, int sms,
                         unsigned long long wait_limit_ns, cudaStream_t st, float* partial) {
  const FusedEntry& e = kFused[idx];
  CUtensorMap ma, mb;
  if (p.K > 0) {
    if (e.ts) {  // FP32 A; B's parts from the split pass (box {32, BN, P})
      if (!p.Bparts || (reinterpret_cast<uintptr_t>(p.A) & 15) || (p.lda & 3) ||
          !tc_make_f32_map(&ma, p.A, p.K, p.M, p.lda, kBK, kBM, true) ||
          !tc_make_parts_map(&mb, p.Bparts, e.parts, p.N, p.Kp, e.bn))
        return cudaErrorInvalidValue;
    } else if (!fused_make_maps(idx, p.A, p.lda, p.B, p.ldb, p.M, p.N, p.K, &ma, &mb)) {
      return cudaErrorInvalidValue;
    }
  } else {  // no k-tiles: nothing is loaded, the epilogue stores zeros
    memset(&ma, 0, sizeof(ma));
    memset(&mb, 0, sizeof(mb));
  }
  p.tiles_m = (p.M + e.bm - 1) / e.bm;
  p.tiles_n = (p.N + e.bn - 1) / e.bn;
  p.num_tiles = p.tiles_m * p.tiles_n;
  p.raster = raster > 0 ? raster : 8;
  float* C = p.C;
  const long ldc = p.ldc;
  if (p.splits > 1) {
    p.C = partial;
    p.ldc = p.N;
  }
  TcRun run;
  run.chunk_ktiles = tc_chunk_ktiles(e.parts, chunk_k);
  // (the A-in-TMEM tiles take no L2 prefetch: measured 0-15 % slower with
  // 8-64 k-tiles of A ahead, single boxes or 1 KB-per-row chunks)
  run.l2_ahead = e.ts ? 0 : fused_l2_ahead();
  run.l2_keep = 0;
  run.debug_skip_loads = 0;
  run.wait_limit_ns = wait_limit_ns ? wait_limit_ns : kWaitLimitNs;
  const bool scaled = p.rowmax != nullptr;
  const long items = (long)p.num_tiles * p.splits;
  // work units (clusters, or CTAs) never wait on each other, so a grid larger
  // than what is resident would only run late; it is capped at the resident
  // units
  const int cap = fused_tile_slots(idx, sms);
  int resident = e.slots(scaled);
  if (resident <= 0 || resident > cap) resident = cap;
  const long units = std::max<long>(1, std::min<long>(items, resident));
  cudaError_t err = e.launch(ma, mb, p, run, (int)(e.ts ? units : 2 * units), st, scaled);
  if (err != cudaSuccess || p.splits == 1) return err;
  return splitk_reduce(partial, C, p.M, p.N, ldc, 0, p.splits, 1, sms, st);
}

int fused_read_and_clear_device_error() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)) != cudaSuccess) return HBSG_ERR_CUDA;
  if (v != 0) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int));
  }
  return v;
}

}  // namespace hbsg
