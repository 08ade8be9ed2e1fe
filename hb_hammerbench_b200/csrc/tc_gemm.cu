// Split-BF16 tensor-core SGEMM for sm_100a (tcgen05 + TMEM + TMA).
//
// C = A*B for FP32 A (M x K) and B (K x N) from their BF16 parts (split
// pre-pass, split_bf16.cu): with parts hi, mid[, lo] of each operand,
//   3-product form: hi*mid + mid*hi + hi*hi            (2 parts)
//   6-product form: mid*mid + hi*lo + lo*hi + hi*mid + mid*hi + hi*hi
// (terms issued smallest first). All products of one k-step go to the same
// FP32 TMEM accumulator. Every `chunk` of K the accumulator is drained into
// FP32 registers (rounded add), and the next chunk starts from zero, so the
// tensor core only ever accumulates a short run of K.
//
// CTA (persistent, one per SM, 10 warps):
//   warp 0      TMA producer: per k-tile one 3-D box of all A parts and one
//               of all B parts into a STAGES-deep shared-memory ring
//               (64-byte swizzle, K-major), completion on an mbarrier.
//   warp 1      TMEM allocator and MMA issuer: the warp runs the issue loop
//               converged and one elected lane issues
//               tcgen05.mma kind::f16 (M=128, N=BN, K=16) per product and
//               k-step into TMEM buffer (chunk % 2); tcgen05.commit frees the
//               smem stage and, at the end of a chunk, hands the buffer to
//               the epilogue.
//   warps 2-9   epilogue: thread (quadrant q, half h) owns TMEM lane 32q+lane
//               (= output row) and BN/2 columns; it adds each drained chunk
//               to its register sums, releases the buffer, and at the end of
//               the tile scales by 2^(row exp + col exp) and stores C through
//               an 8-lane float4 transpose (128-byte row segments per store).
// No TMA multicast is used; every CTA fetches its own tiles.
// Every wait is bounded: after kWaitLimitNs the kernel records
// HBSG_ERR_DEVICE_TIMEOUT in the device error flag and unwinds.
#include <algorithm>
#include <cstdlib>

#include "tc_kernel2.cuh"

namespace hbsg {

struct TcParams {
  int M, N, K, Kp;
  int tiles_m, tiles_n, num_tiles;
  int raster;
  int splits;        // K slices (1 = none)
  int kt_per_split;  // k-tiles per slice
  float* C;          // output, or the slice partials [splits][M][N] when splits > 1
  long ldc;
  const uint32_t* rowmax;  // null unless scaled
  const uint32_t* colmax;
};

// Tiles of one GEMM in rasterised order: groups of `raster` tile rows,
// column-major inside a group, so CTAs resident together share operand
// strips in L2.
struct SingleTiles {
  static constexpr bool kInlineSplit = false;
  static constexpr bool kQueue = false;  // tiles dealt statically (all the same size)
  __device__ bool wait_ready(int, int, volatile int*, unsigned long long) const { return true; }
  template <int P, bool SCALED>
  __device__ void split_worker(int, volatile int*) const {}
  const CUtensorMap* ma;
  const CUtensorMap* mb;
  const TcParams* p;
  // Work item t = slice * num_tiles + tile: with split-K the slices of all
  // tiles are independent items; slice s covers k-tiles [s*kts, (s+1)*kts)
  // and writes its partial to C + s*M*N (row stride N).
  template <int TBM, int BN>
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
    const int KT = p->Kp / kBK;
    w.kt0 = slice * p->kt_per_split;
    w.KT = min(p->kt_per_split, KT - w.kt0);
    if (p->splits > 1) {
      w.C = p->C + (long)slice * p->M * p->N;
      w.ldc = p->N;
    } else {
      w.C = p->C;
      w.ldc = p->ldc;
    }
    w.rowmax = p->rowmax;
    w.colmax = p->colmax;
    return w;
  }
};

template <int BN, int TBM = kBM>
struct SingleTilesBN : SingleTiles {
  __device__ __forceinline__ int count() const { return p->num_tiles * p->splits; }
  __device__ __forceinline__ TileWork get(int t) const { return get_bn<TBM, BN>(t); }
};

template <int P, int BN, int STAGES, bool SCALED>
__global__ void __launch_bounds__(320, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const __grid_constant__ TcParams p, const TcRun run) {
  SingleTilesBN<BN> tiles;
  tiles.ma = &tmA;
  tiles.mb = &tmB;
  tiles.p = &p;
  tc_body<P, BN, STAGES, SCALED>(tiles, run);
}

// CTA-pair form: 256 x BN tiles on a cluster of two CTAs (tc_kernel2.cuh).
template <int P, int BN, int STAGES, bool SCALED>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(320, 1)
    tc_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const __grid_constant__ TcParams p, const TcRun run) {
  SingleTilesBN<BN, 2 * kBM> tiles;
  tiles.ma = &tmA;
  tiles.mb = &tmB;
  tiles.p = &p;
  tc_pair_body<P, BN, STAGES, SCALED>(tiles, run);
}

// ---------------------------------------------------------------------------
// Host side: tensor maps, tile table, launch.

// Resolved once; function-local static initialisation is thread-safe, so
// concurrent first calls from several host threads all see the pointer.
static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
  }();
  return fn;
}

// 3-D map over parts[P][rows][Kp] bf16 with a box of {32, box_rows, P}.
bool tc_make_parts_map_impl(CUtensorMap* map, const void* parts, int P, int rows, int Kp,
                           int box_rows) {
  auto enc = get_encode();
  if (!enc) return false;
  cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, (cuuint64_t)P};
  cuuint64_t strides[2] = {(cuuint64_t)Kp * 2, (cuuint64_t)rows * Kp * 2};
  cuuint32_t box[3] = {(cuuint32_t)kBK, (cuuint32_t)box_rows, (cuuint32_t)P};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(parts), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool tc_make_f32_map(void* map, const void* base, int inner, int outer, long ld, int box_inner,
                     int box_outer, bool swizzle128) {
  auto enc = get_encode();
  if (!enc || inner <= 0 || outer <= 0) return false;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(static_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                   const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

struct TcEntry {
  int parts, bn, stages;
  int pair;  // 1: CTA-pair kernel, 256-row tiles
  int smem;
  cudaError_t (*launch)(const CUtensorMap&, const CUtensorMap&, const TcParams&, const TcRun&,
                        int grid, cudaStream_t, bool scaled);
};

template <int P, int BN, int STAGES>
static cudaError_t launch_tc(const CUtensorMap& a, const CUtensorMap& b, const TcParams& p,
                             const TcRun& run, int grid, cudaStream_t st, bool scaled) {
  using S = TcShape<P, BN, STAGES>;
  auto k0 = tc_gemm_kernel<P, BN, STAGES, false>;
  auto k1 = tc_gemm_kernel<P, BN, STAGES, true>;
  auto k = scaled ? k1 : k0;
  static uint64_t m0 = 0, m1 = 0;
  if (!set_smem_once(reinterpret_cast<const void*>(k), S::kSmemBytes, scaled ? &m1 : &m0))
    return cudaErrorInvalidValue;
  k<<<grid, S::kThreads, S::kSmemBytes, st>>>(a, b, p, run);
  return cudaGetLastError();
}

#define HBSG_TC_ENTRY(P, BN, ST) \
  TcEntry { P, BN, ST, 0, TcShape<P, BN, ST>::kSmemBytes, &launch_tc<P, BN, ST> }

// Ordered by parts: entries with parts == 3 serve BF16X6, parts == 2 BF16X3.
template <int P, int BN, int STAGES>
static cudaError_t launch_tc_pair(const CUtensorMap& a, const CUtensorMap& b, const TcParams& p,
                                  const TcRun& run, int grid, cudaStream_t st, bool scaled) {
  using S = TcPairShape<P, BN, STAGES>;
  auto k0 = tc_pair_kernel<P, BN, STAGES, false>;
  auto k1 = tc_pair_kernel<P, BN, STAGES, true>;
  auto k = scaled ? k1 : k0;
  static uint64_t m0 = 0, m1 = 0;
  if (!set_smem_once(reinterpret_cast<const void*>(k), S::kSmemBytes, scaled ? &m1 : &m0))
    return cudaErrorInvalidValue;
  k<<<grid, 320, S::kSmemBytes, st>>>(a, b, p, run);
  return cudaGetLastError();
}
#define HBSG_TC_PAIR_ENTRY(P, BN, ST) \
  TcEntry { P, BN, ST, 1, TcPairShape<P, BN, ST>::kSmemBytes, &launch_tc_pair<P, BN, ST> }

#define HBSG_TC_ENTRY_COMMA(P, BN, ST) HBSG_TC_ENTRY(P, BN, ST),
static const TcEntry kTcTiles[] = {HBSG_TC_TILE_LIST(HBSG_TC_ENTRY_COMMA)
                                   HBSG_TC_PAIR_ENTRY(3, 256, 4),   // 256 x 256 pair, 6 products
                                   HBSG_TC_PAIR_ENTRY(2, 256, 6)};  // 256 x 256 pair, 3 products
static constexpr int kNumTcTiles = sizeof(kTcTiles) / sizeof(kTcTiles[0]);

int tc_num_tiles() { return kNumTcTiles; }

bool tc_tile_info(int idx, hbsg_tile_info* out) {
  if (idx < 0 || idx >= kNumTcTiles) return false;
  const TcEntry& e = kTcTiles[idx];
  out->variant_class = 1;
  out->bm = e.pair ? 2 * kBM : kBM;
  out->bn = e.bn;
  out->bk = kBK;
  out->threads = 320;
  out->smem_bytes = e.smem;
  out->parts = e.parts;
  return true;
}

int tc_tile_parts(int idx) { return kTcTiles[idx].parts; }
int tc_tile_bn(int idx) { return kTcTiles[idx].bn; }
int tc_tile_pair(int idx) { return kTcTiles[idx].pair; }

// Co-resident clusters of two CTAs for a pair kernel (0 if unknown).
template <int P, int BN, int STAGES>
static int pair_clusters(bool scaled) {
  using S = TcPairShape<P, BN, STAGES>;
  const void* k = scaled ? reinterpret_cast<const void*>(&tc_pair_kernel<P, BN, STAGES, true>)
                         : reinterpret_cast<const void*>(&tc_pair_kernel<P, BN, STAGES, false>);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(320, 1, 1);
  cfg.dynamicSmemBytes = S::kSmemBytes;
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

bool tc_make_parts_map(void* map, const void* parts, int P, int rows, int Kp, int box_rows) {
  return tc_make_parts_map_impl(static_cast<CUtensorMap*>(map), parts, P, rows, Kp, box_rows);
}

// K slices of the automatic schedule for `tiles` output tiles: enough
// (tile, slice) work items to fill the concurrent slots when the output alone
// has fewer than half as many tiles as slots, each slice keeping >= 8
// k-tiles; `requested` > 0 overrides. Normalised so that no slice is empty.
// Automatic slices shorter than this many k-tiles are not used (see tc_pick_tile).
static constexpr int kMinSliceKtiles = 16;

static int slices_for(long tiles, int KT, int slots, int requested, int* kt_per_split) {
  int s = requested;
  if (s <= 0) {
    s = 1;
    if (tiles * 2 <= slots) s = (int)std::min<long>((slots + tiles - 1) / tiles, std::max(1, KT / 8));
  }
  s = std::max(1, std::min(s, KT));
  const int per = (KT + s - 1) / s;
  if (kt_per_split) *kt_per_split = per;
  return (KT + per - 1) / per;
}

static int ktiles_of(int K) {
  const int KT = ((K + 31) / 32 * 32) / kBK;
  return KT > 0 ? KT : 1;
}

int tc_slices(long tiles, int K, int slots, int requested, int* kt_per_split) {
  const int KT = ktiles_of(K);
  int per = KT;
  int s = slices_for(tiles, KT, slots, requested, &per);
  if (requested <= 0 && s > 1 && per < kMinSliceKtiles) {
    s = 1;
    per = KT;
  }
  if (kt_per_split) *kt_per_split = per;
  return s;
}

// Tile shape for an M x N x K product: scored on the work items it yields
// after K slicing (so a tall-K problem with a small output takes the wide,
// efficient tile and fills the GPU with slices rather than narrow tiles),
// the fraction of the last wave in use, the tile's operand bytes per MMA
// flop, and the rows and columns wasted at the edges. Slices shorter than
// kMinSliceKtiles are not counted: their FP32 partials, the reduction and
// the pipeline refill outweigh the wider tile (measured at 1024^3, 1000^3
// and 128x128x65536: 15-30 % slower than unsliced narrow tiles).
int tc_pick_tile(int M, int N, int K, int parts, int sms, int requested_splits, double* score_out) {
  const int KT = ktiles_of(K);
  int best = -1;
  double best_score = -1.0;
  for (int i = 0; i < kNumTcTiles; ++i) {
    const TcEntry& e = kTcTiles[i];
    if (e.parts != parts) continue;
    const int tbm = e.pair ? 2 * kBM : kBM;
    const int slots = e.pair ? sms / 2 : sms;
    const long tiles = (long)((M + tbm - 1) / tbm) * ((N + e.bn - 1) / e.bn);
    int per = KT;
    int s = slices_for(tiles, KT, slots, requested_splits, &per);
    if (requested_splits <= 0 && s > 1 && per < kMinSliceKtiles) s = 1;
    const long items = tiles * s;
    const double waves = (double)items / slots;
    const double eff = waves / ceil(waves);
    // shared-memory operand bytes per MMA flop (the single-CTA bound)
    const double width = e.pair ? 0.9 : e.bn == 256 ? 0.95 : e.bn == 192 ? 0.9 : e.bn == 128 ? 0.8 : 0.55;
    const double waste = (double)N / (((N + e.bn - 1) / e.bn) * e.bn) *
                         ((double)M / (((M + tbm - 1) / tbm) * tbm));
    const double score = eff * width * waste * fmin(1.0, waves);
    if (score > best_score + 1e-9) {
      best_score = score;
      best = i;
    }
  }
  if (score_out) *score_out = best_score;
  return best;
}

// K slices the launch uses: the same rule the tile choice scored (automatic
// slices shorter than kMinSliceKtiles are dropped for one unsliced pass), so
// the schedule that runs is the one that was chosen, and the workspace holds
// no partial buffer for slices that never run.
int tc_pick_splits(int idx, int M, int N, int K, int requested, int sms, int* kt_per_split) {
  const TcEntry& e = kTcTiles[idx];
  const int tbm = e.pair ? 2 * kBM : kBM;
  const long tiles = (long)((M + tbm - 1) / tbm) * ((N + e.bn - 1) / e.bn);
  return tc_slices(tiles, K, e.pair ? sms / 2 : sms, requested, kt_per_split);
}

cudaError_t tc_launch(int idx, const void* Ap, const void* Bp, int M, int N, int K, int Kp,
                      float* C, long ldc, const uint32_t* rowmax, const uint32_t* colmax,
                      int raster, int chunk_k, int sms, int debug_skip_loads,
                      unsigned long long wait_limit_ns, cudaStream_t st, int splits,
                      float* partial) {
  const TcEntry& e = kTcTiles[idx];
  CUtensorMap ma, mb;
  if (!tc_make_parts_map_impl(&ma, Ap, e.parts, M, Kp, kBM)) return cudaErrorInvalidValue;
  if (!tc_make_parts_map_impl(&mb, Bp, e.parts, N, Kp, e.pair ? e.bn / 2 : e.bn))
    return cudaErrorInvalidValue;
  TcParams p{};
  p.M = M;
  p.N = N;
  p.K = K;
  p.Kp = Kp;
  const int tbm = e.pair ? 2 * kBM : kBM;
  p.tiles_m = (M + tbm - 1) / tbm;
  p.tiles_n = (N + e.bn - 1) / e.bn;
  p.num_tiles = p.tiles_m * p.tiles_n;
  p.raster = raster > 0 ? raster : 16;
  int kts = Kp / kBK;
  p.splits = splits > 1 ? tc_pick_splits(idx, M, N, K, splits, sms, &kts) : 1;
  p.kt_per_split = kts;
  p.C = p.splits > 1 ? partial : C;
  p.ldc = p.splits > 1 ? N : ldc;
  p.rowmax = rowmax;
  p.colmax = colmax;
  TcRun run;
  run.chunk_ktiles = tc_chunk_ktiles(e.parts, chunk_k);
  run.l2_ahead = tc_l2_ahead();
  run.l2_keep = tc_l2_keep();
  run.debug_skip_loads = debug_skip_loads;
  run.wait_limit_ns = wait_limit_ns ? wait_limit_ns : kWaitLimitNs;
  const long items = (long)p.num_tiles * p.splits;
  int grid;
  if (e.pair) {
    // every pair must be resident at once (tiles are dealt statically)
    int resident = e.parts == 3 ? pair_clusters<3, 256, 4>(rowmax != nullptr)
                                : pair_clusters<2, 256, 6>(rowmax != nullptr);
    if (resident <= 0) resident = sms / 2;
    const long cap = std::min<long>(resident, sms / 2);
    const long pairs = items < cap ? items : cap;
    grid = (int)(2 * pairs);
  } else {
    grid = (int)(items < sms ? items : sms);
  }
  cudaError_t err = e.launch(ma, mb, p, run, grid, st, rowmax != nullptr);
  if (err != cudaSuccess || p.splits == 1) return err;
  return splitk_reduce(partial, C, M, N, ldc, 0, p.splits, 1, sms, st);
}

// Default drain interval: every 2 k-tiles (64 of K) for the 6-product form,
// every 4 k-tiles for the 3-product form. Measured at 8192^3 (6-product):
// interval 32 / 64 / 128 / 256 of K gave 4.63 / 4.38 / 4.11 / 4.03 ms and
// relative error 3.4e-7 / 4.4e-7 / 8.2e-7 / 1.6e-6 against FP64 (FFMA:
// 1.6e-6); 64 keeps the error 3.7x below FFMA's. The 3-product form's error
// is set by its 2-part split, not by the interval.
int tc_chunk_ktiles(int parts, int chunk_k) {
  const int ck = chunk_k > 0 ? chunk_k : (parts == 3 ? 64 : 128);
  return ck / kBK > 0 ? ck / kBK : 1;
}

// k-tiles the producer prefetches into L2 ahead of its loads
// (HBSG_TC_L2_AHEAD overrides the default, for tuning).
int tc_l2_ahead() {
  static const int v = [] {
    const char* e = getenv("HBSG_TC_L2_AHEAD");
    const int x = e ? atoi(e) : 0;  // off: measured slower at 2, 4 and 8 (extra TMA operations)
    return x < 0 ? 0 : x;
  }();
  return v;
}

// Operand loads with an L2 evict-last policy (HBSG_TC_L2_KEEP=0/1, for tuning).
int tc_l2_keep() {
  static const int v = [] {
    const char* e = getenv("HBSG_TC_L2_KEEP");
    return e ? (atoi(e) != 0 ? 1 : 0) : 0;
  }();
  return v;
}

int tc_read_and_clear_device_error() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)) != cudaSuccess) return HBSG_ERR_CUDA;
  if (v != 0) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int));
  }
  return v;
}

}  // namespace hbsg
