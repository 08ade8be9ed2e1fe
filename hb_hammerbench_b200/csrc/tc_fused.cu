// Launches of the fused-split tensor-core GEMM (tc_fused.cuh): C = A*B for
// FP32 A (M x K) and B (K x N), row-major, with the BF16 split done inside the
// product kernel on CTA pairs (256 x BN output tiles). The design and why it
// uses CTA pairs is described in tc_fused.cuh.
//
// Work items are (output tile, K slice) pairs in rasterised tile order, as for
// the unfused kernel (tc_gemm.cu): with K slices each slice writes an FP32
// partial to the workspace, reduced in fixed order afterwards. The scaled
// forms read per-row / per-column maxima that a max pass computes first
// (split_bf16.cu); nothing else is staged in HBM.
#include <algorithm>

#include "tc_fused.cuh"

namespace hbsg {

struct FusedTiles {
  static constexpr bool kInlineSplit = false;
  const FusedParams* p;
  __device__ __forceinline__ int count() const { return p->num_tiles * p->splits; }
  template <int BN>
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
    w.ma = nullptr;
    w.mb = nullptr;
    w.M = p->M;
    w.N = p->N;
    w.m0 = (first + in % gm) * (2 * kBM);
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

template <int BN>
struct FusedTilesBN : FusedTiles {
  __device__ __forceinline__ TileWork get(int t) const { return get_bn<BN>(t); }
};

template <int P, int BN, int STAGES, bool SCALED, bool VEC>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kFusedThreads, 1)
    tc_fused_kernel(const __grid_constant__ FusedParams p, const TcRun run) {
  FusedTilesBN<BN> tiles;
  tiles.p = &p;
  tc_fused_body<P, BN, STAGES, SCALED, VEC>(tiles, run);
}

template <int P, int BN, int STAGES>
static cudaError_t launch_fused(const FusedParams& p, const TcRun& run, int grid, cudaStream_t st,
                                bool scaled, bool vec) {
  using S = TcFusedShape<P, BN, STAGES>;
  const void* k;
  static uint64_t masks[4] = {0, 0, 0, 0};
  const int slot = (scaled ? 2 : 0) + (vec ? 1 : 0);
  if (scaled) {
    k = vec ? reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, STAGES, true, true>)
            : reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, STAGES, true, false>);
  } else {
    k = vec ? reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, STAGES, false, true>)
            : reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, STAGES, false, false>);
  }
  if (!set_smem_once(k, S::kSmemBytes, &masks[slot])) return cudaErrorInvalidValue;
  static int regs_ok[4] = {0, 0, 0, 0};
  if (!fused_regs_ok(k, &regs_ok[slot])) return cudaErrorInvalidConfiguration;
  if (scaled) {
    if (vec) tc_fused_kernel<P, BN, STAGES, true, true><<<grid, kFusedThreads, S::kSmemBytes, st>>>(p, run);
    else tc_fused_kernel<P, BN, STAGES, true, false><<<grid, kFusedThreads, S::kSmemBytes, st>>>(p, run);
  } else {
    if (vec) tc_fused_kernel<P, BN, STAGES, false, true><<<grid, kFusedThreads, S::kSmemBytes, st>>>(p, run);
    else tc_fused_kernel<P, BN, STAGES, false, false><<<grid, kFusedThreads, S::kSmemBytes, st>>>(p, run);
  }
  return cudaGetLastError();
}

struct FusedEntry {
  int parts, bn, stages, smem;
  cudaError_t (*launch)(const FusedParams&, const TcRun&, int, cudaStream_t, bool, bool);
};

#define HBSG_FUSED_ENTRY(P, BN, ST) \
  FusedEntry { P, BN, ST, TcFusedShape<P, BN, ST>::kSmemBytes, &launch_fused<P, BN, ST> }

#define HBSG_FUSED_ENTRY_COMMA(P, BN, ST) HBSG_FUSED_ENTRY(P, BN, ST),
static const FusedEntry kFused[] = {HBSG_FUSED_TILE_LIST(HBSG_FUSED_ENTRY_COMMA)};
static constexpr int kNumFused = sizeof(kFused) / sizeof(kFused[0]);

int fused_num_tiles() { return kNumFused; }
int fused_tile_parts(int idx) { return kFused[idx].parts; }
int fused_tile_bn(int idx) { return kFused[idx].bn; }

bool fused_tile_info(int idx, hbsg_tile_info* out) {
  if (idx < 0 || idx >= kNumFused) return false;
  out->variant_class = 1;
  out->bm = 2 * kBM;
  out->bn = kFused[idx].bn;
  out->bk = kBK;
  out->threads = kFusedThreads;
  out->smem_bytes = kFused[idx].smem;
  out->parts = kFused[idx].parts;
  return true;
}

// Co-resident clusters of two CTAs of fused entry `idx` (0 if unknown).
static int fused_clusters(int idx, bool scaled) {
  const FusedEntry& e = kFused[idx];
  const void* k = nullptr;
#define HBSG_FUSED_PICK(P, BN, ST)                                                             \
  if (e.parts == P && e.bn == BN)                                                              \
    k = scaled ? reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, ST, true, true>)        \
               : reinterpret_cast<const void*>(&tc_fused_kernel<P, BN, ST, false, true>);
  HBSG_FUSED_TILE_LIST(HBSG_FUSED_PICK)
#undef HBSG_FUSED_PICK
  if (!k) return 0;
  static uint64_t masks[kNumFused][2];
  if (!set_smem_once(k, e.smem, &masks[idx][scaled ? 1 : 0])) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(kFusedThreads, 1, 1);
  cfg.dynamicSmemBytes = e.smem;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = 2;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int fused_pick_splits(int idx, int M, int N, int K, int requested, int sms, int* kt_per_split) {
  const long tiles = (long)((M + 2 * kBM - 1) / (2 * kBM)) * ((N + kFused[idx].bn - 1) / kFused[idx].bn);
  return tc_slices(tiles, K, sms / 2, requested, kt_per_split);
}

cudaError_t fused_launch(int idx, FusedParams p, int raster, int chunk_k, int sms,
                         unsigned long long wait_limit_ns, cudaStream_t st, float* partial) {
  const FusedEntry& e = kFused[idx];
  p.tiles_m = (p.M + 2 * kBM - 1) / (2 * kBM);
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
  run.l2_ahead = 0;
  run.l2_keep = 0;
  run.debug_skip_loads = 0;
  run.wait_limit_ns = wait_limit_ns ? wait_limit_ns : kWaitLimitNs;
  const bool scaled = p.rowmax != nullptr;
  const bool vec = ((p.lda & 3) == 0) && ((reinterpret_cast<uintptr_t>(p.A) & 15) == 0);
  const long items = (long)p.num_tiles * p.splits;
  // pairs never wait on each other, so a grid larger than what is resident
  // would only run late; it is capped at the co-resident clusters
  int resident = fused_clusters(idx, scaled);
  if (resident <= 0) resident = sms / 2;
  const long pairs = std::max<long>(1, std::min<long>(items, std::min(resident, sms / 2)));
  cudaError_t err = e.launch(p, run, (int)(2 * pairs), st, scaled, vec);
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
