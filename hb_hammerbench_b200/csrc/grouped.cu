// Grouped SGEMM: many independent FP32 GEMMs of uneven M, N, K in one
// persistent launch, captured with its split passes in one CUDA graph.
//
// The reference's only multi-GEMM form is the NITER loop of independent
// products (apps/sgemm/kernel.cpp:293-297) over equal sizes, and its legacy
// cooperative kernel strides tile groups over the output grid
// (apps/legacy/gemm/sgemm_group_cooperative/kernel.cpp:285-286). Here the
// output tiles of all problems form one list:
//   - problems are ordered by K (the cost of a tile) descending, and each
//     problem's tiles are listed in rasterised order;
//   - the CTAs of the persistent grid claim tiles in that order from a
//     counter in the workspace (zeroed by the launch sequence before the
//     kernel; the single-CTA tensor-core kernels hand the claimed tile to
//     their MMA and epilogue warps through a ring in shared memory with
//     bounded waits, tc_kernel.cuh), so a CTA that drew long tiles takes
//     fewer and the grid ends together;
// so the ~G tiles in flight at any moment have similar cost (balanced waves)
// and mostly belong to one or two problems (their operand strips are shared
// in L2). The CTA-pair and fused-split kernels deal the same list statically
// (pair p takes tiles p, p + G/2, ...).
//
// Split-BF16 forms: one grouped split pass over all problems writes every
// problem's BF16 parts into the workspace; the tensor-core kernel body
// (tc_kernel.cuh) then runs over the tile list with two TMA tensor maps per
// problem kept in global memory. FFMA: the FFMA tile body (ffma_kernel.cuh)
// runs over the tile list.
//
// A plan (hbsg_grouped_plan_create) lays the tables out in the caller's
// workspace, uploads them once, and captures the launches into a CUDA graph;
// hbsg_grouped_run replays that graph on a stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

#include "ffma_kernel.cuh"
#include "split_kernel.cuh"
#include "tc_fused.cuh"

namespace hbsg {

// ---------------------------------------------------------------------------
// Device tables

struct GProblem {  // one problem, as the kernels see it
  const float* A;
  const float* B;
  float* C;
  long lda, ldb, ldc;
  int M, N, K, Kp;
  void* Ap;  // split parts [P][M][Kp]
  void* Bp;  // split parts [P][N][Kp]
  uint32_t* rowmax;
  uint32_t* colmax;
};

struct GTiles {  // tile source for the tensor-core body (split pass run beforehand)
  static constexpr bool kInlineSplit = false;
  // tc_body claims tiles from `queue` (zeroed before each launch); the pair
  // and fused-split bodies deal them statically
  static constexpr bool kQueue = true;
  int* queue;
  __device__ bool wait_ready(int, int, volatile int*, unsigned long long) const { return true; }
  template <int P, bool SCALED>
  __device__ void split_worker(int, volatile int*) const {}
  const GProblem* probs;
  const int4* tiles;  // {problem, m0, n0, inline-split jobs of the problem (0 = split before)}
  const CUtensorMap* maps;  // 2 per problem: A parts, B parts
  int n;
  __device__ __forceinline__ int count() const { return n; }
  __device__ __forceinline__ TileWork get(int t) const {
    const int4 e = tiles[t];
    const GProblem& p = probs[e.x];
    TileWork w;
    w.prob = e.x;
    w.ready_target = e.w;
    w.ma = maps + 2 * e.x;
    w.mb = maps + 2 * e.x + 1;
    w.C = p.C;
    w.ldc = p.ldc;
    w.M = p.M;
    w.N = p.N;
    w.m0 = e.y;
    w.n0 = e.z;
    w.kt0 = 0;
    w.KT = p.K > 0 ? p.Kp / kBK : 0;  // K = 0: no k-tiles, the epilogue stores zeros
    w.rowmax = p.rowmax;
    w.colmax = p.colmax;
    w.A = p.A;
    w.B = p.B;
    w.lda = p.lda;
    w.ldb = p.ldb;
    w.K = p.K;
    return w;
  }
};

template <int P, int BN, int STAGES, bool SCALED>
__global__ void __launch_bounds__(320, 1) tc_grouped_kernel(const GTiles tiles, const TcRun run) {
  tc_body<P, BN, STAGES, SCALED>(tiles, run);
}

// CTA-pair form over 256-row tiles (tc_kernel2.cuh): the tile list holds
// 256 x BN tiles, the A maps have 128-row boxes (each CTA loads its half of
// the tile's rows) and the B maps BN/2-row boxes.
template <int P, int BN, int STAGES, bool SCALED>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(320, 1)
    tc_grouped_pair_kernel(const GTiles tiles, const TcRun run) {
  tc_pair_body<P, BN, STAGES, SCALED>(tiles, run);
}

// Fused-split form: CTA pairs over 256-row tiles, the split done by the
// product kernel's converter warps (tc_fused.cuh); no split pass and no parts
// in the workspace.
template <int P, int BN, int STAGES, int SSTAGES, bool SCALED>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kFusedThreads, 1)
    tc_grouped_fused_kernel(const GTiles tiles, const TcRun run) {
  tc_fused_body<P, BN, STAGES, SSTAGES, SCALED>(tiles, run);
}

// ---- inline split --------------------------------------------------------------
// The split of the operands into BF16 parts runs inside the tensor-core
// kernel, on two extra warps per CTA, while the tensor cores work on earlier
// problems. Work is cut into jobs of 32 x 32 operand elements, numbered in
// the problems' tile order (A jobs then B jobs per problem); splitter warps
// claim jobs from a global counter (so progress never depends on which CTAs
// are resident) and count finished jobs per problem. A CTA's TMA producer
// loads a problem's first tile only after that count is complete. Splitters
// wait on nothing, so the dependency chain always ends.
struct SplitJob {
  int valid, isA, r0, k0;
};

// The problem a splitter warp is working on, cached in registers: claims are
// mostly consecutive within one problem, so the job-to-problem search (a
// chain of dependent global loads) is only repeated when a claim leaves it.
struct SplitCursor {
  int first = 0, last = -1;  // job range [first, last) of the cached problem
  int prob = -1;
  const float* A;
  const float* B;
  long lda, ldb;
  int M, N, K, Kp, kb, na, nb;
  __nv_bfloat16* Ap;
  __nv_bfloat16* Bp;
  const uint32_t* rowmax;
  const uint32_t* colmax;
};

struct GTilesInline : GTiles {
  static constexpr bool kInlineSplit = true;
  int* ready;            // finished jobs per problem (zeroed before the launch)
  int* job_counter;      // next unclaimed job (zeroed before the launch)
  const int* order;      // problem index of the i-th problem in tile order
  const int* job_start;  // first job of the i-th problem in tile order; [count] = total
  const int* jobs_of;    // jobs per problem
  int num_problems;
  int num_jobs;

  __device__ __forceinline__ bool wait_ready(int prob, int target, volatile int* abort_flag,
                                             unsigned long long limit_ns) const {
    const int* addr = ready + prob;
    const unsigned long long t0 = globaltimer();
    for (uint32_t i = 0;; ++i) {
      int v;
      asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(addr) : "memory");
      if (v >= target) break;
      if (*abort_flag) return false;
      if ((i & 15) == 15 && globaltimer() - t0 > limit_ns) {
        *abort_flag = 1;
        atomicExch(&g_device_error, (int)HBSG_ERR_DEVICE_TIMEOUT);
        return false;
      }
      __nanosleep(64);
    }
    // the parts were written through the generic proxy; the TMA reads them
    // through the async proxy
    asm volatile("fence.proxy.async.global;" ::: "memory");
    return true;
  }

  __device__ __forceinline__ void seek(SplitCursor& c, int j) const {
    int lo = 0, hi = num_problems;  // largest i with job_start[i] <= j
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(job_start + mid) <= j) lo = mid;
      else hi = mid;
    }
    const int p = __ldg(order + lo);
    const GProblem& g = probs[p];
    c.first = __ldg(job_start + lo);
    c.last = __ldg(job_start + lo + 1);
    c.prob = p;
    c.A = g.A;
    c.B = g.B;
    c.lda = g.lda;
    c.ldb = g.ldb;
    c.M = g.M;
    c.N = g.N;
    c.K = g.K;
    c.Kp = g.Kp;
    c.kb = g.Kp / 32;
    c.na = ((g.M + 31) / 32) * c.kb;
    c.nb = (g.N + 31) / 32;
    c.Ap = static_cast<__nv_bfloat16*>(g.Ap);
    c.Bp = static_cast<__nv_bfloat16*>(g.Bp);
    c.rowmax = g.rowmax;
    c.colmax = g.colmax;
  }

  __device__ __forceinline__ SplitJob decode(const SplitCursor& c, int j) const {
    SplitJob d{};
    d.valid = 1;
    int local = j - c.first;
    if (local < c.na) {
      d.isA = 1;
      d.r0 = (local / c.kb) * 32;
      d.k0 = (local % c.kb) * 32;
    } else {
      local -= c.na;
      d.isA = 0;
      d.r0 = (local % c.nb) * 32;
      d.k0 = (local / c.nb) * 32;
    }
    return d;
  }

  // Lane l loads row r0 + l of A (32 consecutive k), or column r0 + l of B
  // (32 consecutive k, each load instruction coalesced across the warp).
  __device__ __forceinline__ void load(const SplitCursor& c, const SplitJob& d, int lane,
                                       float* v) const {
    const int r = d.r0 + lane;
    if (d.isA) {
      if (r >= c.M) return;
      const float* src = c.A + (long)r * c.lda + d.k0;
      if (d.k0 + 32 <= c.K && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float4 x = __ldg(reinterpret_cast<const float4*>(src + 4 * i));
          v[4 * i] = x.x;
          v[4 * i + 1] = x.y;
          v[4 * i + 2] = x.z;
          v[4 * i + 3] = x.w;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = (d.k0 + i < c.K) ? __ldg(src + i) : 0.0f;
      }
    } else {
      const bool in = r < c.N;
      const float* src = c.B + (long)d.k0 * c.ldb + r;
#pragma unroll
      for (int i = 0; i < 32; ++i)
        v[i] = (in && d.k0 + i < c.K) ? __ldg(src + (long)i * c.ldb) : 0.0f;
    }
  }

  template <int P, bool SCALED>
  __device__ __forceinline__ void store(const SplitCursor& c, const SplitJob& d, int lane,
                                        const float* v) const {
    const int r = d.r0 + lane;
    const int rows = d.isA ? c.M : c.N;
    if (r >= rows) return;
    int e = 0;
    if constexpr (SCALED) e = exp_from_maxbits(d.isA ? c.rowmax[r] : c.colmax[r]);
    const long plane = (long)rows * c.Kp;
    __nv_bfloat16* dst = (d.isA ? c.Ap : c.Bp) + (long)r * c.Kp + d.k0;
#pragma unroll
    for (int gi = 0; gi < 4; ++gi) {
      __align__(16) __nv_bfloat16 parts[P][8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        __nv_bfloat16 o[3];
        split_value<P>(v[8 * gi + i], e, o);
#pragma unroll
        for (int q = 0; q < P; ++q) parts[q][i] = o[q];
      }
#pragma unroll
      for (int q = 0; q < P; ++q)
        *reinterpret_cast<uint4*>(dst + q * plane + 8 * gi) = *reinterpret_cast<const uint4*>(parts[q]);
    }
  }

  // L2 prefetch of the source lines of job j (lane l: A row r0 + l, or B row
  // k0 + l of the job's 32 columns): 128 bytes per lane.
  __device__ __forceinline__ void prefetch(SplitCursor& c, int j, int lane) const {
    if (j >= num_jobs) return;
    if (j < c.first || j >= c.last) seek(c, j);
    const SplitJob d = decode(c, j);
    const float* src = nullptr;
    if (d.isA) {
      const int r = d.r0 + lane;
      if (r < c.M && d.k0 < c.K) src = c.A + (long)r * c.lda + d.k0;
    } else {
      const int k = d.k0 + lane;
      if (k < c.K && d.r0 < c.N) src = c.B + (long)k * c.ldb + d.r0;
    }
    if (src) asm volatile("prefetch.global.L2 [%0];" ::"l"(src));
  }

  template <int P, bool SCALED>
  __device__ __forceinline__ void split_worker(int lane, volatile int* abort_flag) const {
    constexpr int BATCH = 2;  // jobs loaded together (64 loads in flight per lane)
    SplitCursor cur, pcur;
    int next = 0;
    if (lane == 0) next = atomicAdd(job_counter, BATCH);
    next = __shfl_sync(0xffffffffu, next, 0);
#pragma unroll
    for (int b = 0; b < BATCH; ++b) prefetch(pcur, next + b, lane);
    for (;;) {
      if (*abort_flag) return;
      const int j0 = next;
      if (j0 >= num_jobs) return;
      // claim the following batch now; the atomic's latency overlaps this batch
      if (lane == 0) next = atomicAdd(job_counter, BATCH);
      SplitJob d[BATCH];
      int prob[BATCH];
      float v[BATCH][32];
#pragma unroll
      for (int b = 0; b < BATCH; ++b) {
        const int j = j0 + b;
        d[b].valid = 0;
        prob[b] = -1;
        if (j >= num_jobs) continue;
        if (j < cur.first || j >= cur.last) seek(cur, j);
        d[b] = decode(cur, j);
        prob[b] = cur.prob;
        load(cur, d[b], lane, v[b]);
      }
      // pull the following batch's source lines into L2 while this one is
      // in flight, so its loads hit L2
      next = __shfl_sync(0xffffffffu, next, 0);
#pragma unroll
      for (int b = 0; b < BATCH; ++b) prefetch(pcur, next + b, lane);
#pragma unroll
      for (int b = 0; b < BATCH; ++b) {
        if (!d[b].valid) continue;
        const int j = j0 + b;
        if (j < cur.first || j >= cur.last) seek(cur, j);
        store<P, SCALED>(cur, d[b], lane, v[b]);
      }
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      asm volatile("fence.proxy.async.global;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
#pragma unroll
        for (int b = 0; b < BATCH; ++b)
          if (prob[b] >= 0)
            asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(ready + prob[b]) : "memory");
      }
    }
  }
};

template <int P, int BN, int STAGES, bool SCALED>
__global__ void __launch_bounds__(384, 1)
    tc_grouped_inline_kernel(const GTilesInline tiles, const TcRun run) {
  tc_body<P, BN, STAGES, SCALED>(tiles, run);
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool VEC, bool PAIR>
__global__ void __launch_bounds__(FfmaShape<BM, BN, BK, WM, WN, STAGES>::kThreads,
                                  FfmaShape<BM, BN, BK, WM, WN, STAGES>::kMinBlocks)
    ffma_grouped_kernel(const GProblem* __restrict__ probs, const int4* __restrict__ tiles, int n,
                        int* __restrict__ queue) {
  // Tiles are claimed from `queue` (zeroed before the launch): thread 0 claims
  // the next tile when a tile starts, so the atomic's latency overlaps it.
  extern __shared__ __align__(16) float smem[];
  __shared__ int s_next;
  if (threadIdx.x == 0) s_next = atomicAdd(queue, 1);
  __syncthreads();
  int t = s_next;
  while (t < n) {
    int nxt = 0;
    if (threadIdx.x == 0) nxt = atomicAdd(queue, 1);
    const int4 e = tiles[t];
    const GProblem& p = probs[e.x];
    const bool vec_store = ((p.ldc & 3) == 0) && ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0);
    ffma_tile<BM, BN, BK, WM, WN, STAGES, VEC, PAIR>(p.A, p.lda, p.B, p.ldb, p.M, p.N, 0, p.K,
                                                     e.y, e.z, p.C, p.ldc, vec_store, smem);
    __syncthreads();  // the tile's last reads of the ring and of s_next are done
    if (threadIdx.x == 0) s_next = nxt;
    __syncthreads();
    t = s_next;
  }
}

// ---- grouped split passes ----------------------------------------------------
// Jobs are int4 {problem, a, b, c}; one CTA per job.

// A rows: job {problem, first 8-element unit, unit count, 0}; units are
// row-major over [M][Kp/8].
template <int P, bool SCALED>
__global__ void __launch_bounds__(256) gsplit_a_kernel(const GProblem* __restrict__ probs,
                                                       const int4* __restrict__ jobs) {
  const int4 j = jobs[blockIdx.x];
  const GProblem& p = probs[j.x];
  const int upr = p.Kp / 8;
  const long plane = (long)p.M * p.Kp;
  auto* Ap = static_cast<__nv_bfloat16*>(p.Ap);
  for (int u = threadIdx.x; u < j.z; u += blockDim.x) {
    const long unit = (long)j.y + u;
    const int m = (int)(unit / upr);
    const int k0 = (int)(unit - (long)m * upr) * 8;
    const int e = SCALED ? exp_from_maxbits(p.rowmax[m]) : 0;
    const float* src = p.A + (long)m * p.lda + k0;
    float v[8];
    if (k0 + 8 <= p.K && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
      const float4 x0 = *reinterpret_cast<const float4*>(src);
      const float4 x1 = *reinterpret_cast<const float4*>(src + 4);
      v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w;
      v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = (k0 + i < p.K) ? src[i] : 0.0f;
    }
    __align__(16) __nv_bfloat16 parts[P][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      __nv_bfloat16 o[3];
      split_value<P>(v[i], e, o);
#pragma unroll
      for (int q = 0; q < P; ++q) parts[q][i] = o[q];
    }
    __nv_bfloat16* dst = Ap + (long)m * p.Kp + k0;
#pragma unroll
    for (int q = 0; q < P; ++q)
      *reinterpret_cast<uint4*>(dst + q * plane) = *reinterpret_cast<const uint4*>(parts[q]);
  }
}

// B: job {problem, k0, n0, 0}: one 64 x 64 block transposed through shared
// memory into [N][Kp] (8 threads write each 128-byte output row segment).
// CTAs are persistent and walk the job list with the grid's stride; each
// thread issues its 16 loads of the next block before the current block is
// split and stored, so the job-table lookups and DRAM latency of one block
// overlap the work on the previous one. (One block per CTA left both exposed:
// 3.8 TB/s against 6.4 TB/s for the A pass.)
template <int P, bool SCALED>
__global__ void __launch_bounds__(256, 4) gsplit_b_kernel(const GProblem* __restrict__ probs,
                                                       const int4* __restrict__ jobs, int njobs) {
  __shared__ float tile[64][65];
  int job = blockIdx.x;
  if (job >= njobs) return;
  int4 j = jobs[job];
  const GProblem* p = probs + j.x;
  float v[16];
  split_b_load(p->B, p->ldb, p->K, p->N, j.y, j.z, v);
  for (;;) {
    __syncthreads();  // every thread is done reading the previous block
    split_b_to_tile(v, tile);
    __syncthreads();
    const int next = job + (int)gridDim.x;
    int4 jn = j;
    const GProblem* pn = p;
    if (next < njobs) {
      jn = jobs[next];
      pn = probs + jn.x;
      split_b_load(pn->B, pn->ldb, pn->K, pn->N, jn.y, jn.z, v);
    }
    split_b_from_tile<P, SCALED>(p->N, p->Kp, static_cast<__nv_bfloat16*>(p->Bp), p->colmax,
                                 j.y, j.z, tile);
    if (next >= njobs) break;
    job = next;
    j = jn;
    p = pn;
  }
}

// Row maxima: job {problem, first row, rows (<= 8), 0}, one warp per row.
__global__ void __launch_bounds__(256) growmax_kernel(const GProblem* __restrict__ probs,
                                                      const int4* __restrict__ jobs) {
  const int4 j = jobs[blockIdx.x];
  const GProblem& p = probs[j.x];
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= j.z) return;
  const int m = j.y + w;
  const float* row = p.A + (long)m * p.lda;
  float mx = 0.0f;
  for (int k = lane; k < p.K; k += 32) {
    const float a = fabsf(row[k]);
    if (isfinite(a)) mx = fmaxf(mx, a);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) p.rowmax[m] = __float_as_uint(mx);
}

// Column maxima: job {problem, n0, k0, 0}: 256 columns x 256 rows of B.
__global__ void __launch_bounds__(256) gcolmax_kernel(const GProblem* __restrict__ probs,
                                                      const int4* __restrict__ jobs) {
  const int4 j = jobs[blockIdx.x];
  const GProblem& p = probs[j.x];
  const int n = j.y + threadIdx.x;
  if (n >= p.N) return;
  const int k1 = min(p.K, j.z + 256);
  float mx = 0.0f;
  for (int k = j.z; k < k1; ++k) {
    const float b = fabsf(p.B[(long)k * p.ldb + n]);
    if (isfinite(b)) mx = fmaxf(mx, b);
  }
  if (mx > 0.0f) atomicMax(p.colmax + n, __float_as_uint(mx));
}

// ---------------------------------------------------------------------------
// Host side

static size_t al(size_t x, size_t a) { return (x + a - 1) / a * a; }

static int parts_of_v(int v) { return (v == HBSG_BF16X6 || v == HBSG_BF16X6_SCALED) ? 3 : 2; }
static bool scaled_of_v(int v) { return v == HBSG_BF16X3_SCALED || v == HBSG_BF16X6_SCALED; }

struct GLayout {
  size_t probs_off, tiles_off, maps_off, jobs_off, queue_off, sync_off, parts_off, max_off, total;
  long num_tiles, num_jobs_a, num_jobs_b, num_jobs_rmax, num_jobs_cmax;
  long inline_jobs;  // 32 x 32 split jobs of the inline split (0 when split separately)
  size_t colmax_bytes;
  size_t sync_bytes;  // ready[count] + job counter (zeroed per run), then order, job_start, jobs_of
};

struct GroupedPlan {
  int variant;
  int count;
  bool inline_split;
  int ffma_tile;   // index into the FFMA table, or -1
  int tc_tile;     // index into the tensor-core table, or -1
  int fused_tile;  // index into the fused table, or -1
  GLayout L;
  uint8_t* ws;
  int grid;
  int sms;  // SMs of the plan's device (sizes the persistent split grid)
  TcRun run;
  bool vec;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

// Default share of the split work (in jobs) done inside the product kernel:
// none. Measured on B200 with the 512-problem batch (M, N, K in 64..2048),
// moving 20-60 % of the split onto two extra warps per CTA made the product
// slower than splitting everything beforehand (the tensor-core pipeline loses
// more than the overlap gains), so the inline split is opt-in.
static constexpr int kDefaultInlinePct = -1;

static int kp_of(int k) { return std::max(32, (k + 31) / 32 * 32); }

// 32 x 32 split jobs of one problem (A then B).
static long inline_jobs_of(const hbsg_problem& q) {
  if (q.m <= 0 || q.n <= 0) return 0;
  const int Kp = kp_of(q.k);
  return (long)((q.m + 31) / 32) * (Kp / 32) + (long)(Kp / 32) * ((q.n + 31) / 32);
}

// Problems in tile order (K descending, stable) and which of them the
// product kernel splits itself: the problems processed last, holding about
// `pct` percent of the split jobs. The others are split by separate kernels
// before the product starts.
struct GSets {
  std::vector<int> order;
  std::vector<char> inl;
  bool any_inline = false;
};

static GSets grouped_sets(int count, const hbsg_problem* pr, int variant, const hbsg_config* cfg) {
  GSets S;
  S.order.resize(count);
  std::iota(S.order.begin(), S.order.end(), 0);
  std::stable_sort(S.order.begin(), S.order.end(),
                   [&](int x, int y) { return pr[x].k > pr[y].k; });
  S.inl.assign(count, 0);
  int pct = cfg && cfg->inline_split_pct != 0 ? cfg->inline_split_pct : kDefaultInlinePct;
  if (variant == HBSG_FFMA || pct < 0) pct = 0;
  pct = std::min(pct, 100);
  long total = 0;
  for (int i = 0; i < count; ++i) total += inline_jobs_of(pr[i]);
  const long target = total * pct / 100;
  long acc = 0;
  for (int i = count - 1; i >= 0 && acc < target; --i) {
    const int p = S.order[i];
    acc += inline_jobs_of(pr[p]);
    S.inl[p] = 1;
    S.any_inline = true;
  }
  return S;
}

// Tile counts and job counts for a problem set (host arrays).
static GLayout grouped_layout(int count, const hbsg_problem* pr, int variant, int bm, int bn,
                              const GSets& sets, bool fused = false) {
  const bool inline_split = sets.any_inline;
  GLayout L{};
  const bool split = variant != HBSG_FFMA;
  const bool parts_in_hbm = split && !fused;
  const int P = split ? parts_of_v(variant) : 0;
  const bool scaled = split && scaled_of_v(variant);
  size_t parts = 0, maxes = 0, cmax = 0;
  for (int i = 0; i < count; ++i) {
    const hbsg_problem& q = pr[i];
    if (q.m <= 0 || q.n <= 0) continue;
    L.num_tiles += (long)((q.m + bm - 1) / bm) * ((q.n + bn - 1) / bn);
    if (parts_in_hbm) {
      const int Kp = kp_of(q.k);
      parts += al((size_t)P * q.m * Kp * 2, 256) + al((size_t)P * q.n * Kp * 2, 256);
      if (sets.inl[i]) {
        L.inline_jobs += inline_jobs_of(q);
      } else {
        const long units = (long)q.m * (Kp / 8);
        L.num_jobs_a += (units + 2047) / 2048;
        L.num_jobs_b += (long)((Kp + 63) / 64) * ((q.n + 63) / 64);
      }
    }
    if (split) {
      if (scaled) {
        maxes += al((size_t)q.m * 4, 256);
        cmax += al((size_t)q.n * 4, 256);
        L.num_jobs_rmax += (q.m + 7) / 8;
        L.num_jobs_cmax += (long)((q.n + 255) / 256) * ((q.k + 255) / 256);
      }
    }
  }
  L.probs_off = 0;
  L.tiles_off = al(sizeof(GProblem) * (size_t)count, 256);
  L.maps_off = al(L.tiles_off + sizeof(int4) * (size_t)L.num_tiles, 256);
  // two tensor maps per problem: its BF16 parts (split pass) or, fused, its
  // FP32 operands
  L.jobs_off = al(L.maps_off + (split ? sizeof(CUtensorMap) * 2 * (size_t)count : 0), 256);
  const long jobs = L.num_jobs_a + L.num_jobs_b + L.num_jobs_rmax + L.num_jobs_cmax;
  L.queue_off = al(L.jobs_off + sizeof(int4) * (size_t)jobs, 256);  // tile queue counter
  L.sync_off = L.queue_off + 256;
  L.sync_bytes = inline_split ? al(sizeof(int) * ((size_t)count + 1), 256) : 0;
  const size_t sync_tables = inline_split ? al(sizeof(int) * (3 * (size_t)count + 1), 256) : 0;
  L.parts_off = al(L.sync_off + L.sync_bytes + sync_tables, 256);
  L.max_off = L.parts_off + parts;
  L.colmax_bytes = cmax;
  L.total = L.max_off + cmax + maxes;  // colmax block first (one memset), then rowmax
  return L;
}

static bool tile_shape(int variant, const hbsg_config* cfg, int* ffma_idx, int* tc_idx,
                       int* fused_idx, int* bm, int* bn) {
  const int nf = ffma_num_tiles();
  const int tile = cfg && cfg->tile > 0 ? cfg->tile - 1 : -1;
  hbsg_tile_info info;
  *fused_idx = -1;
  if (variant == HBSG_FFMA) {
    int idx = tile >= 0 ? tile : 0;  // default: 128 x 128, packed FMA
    if (idx >= nf) return false;
    ffma_tile_info(idx, &info);
    *ffma_idx = idx;
    *tc_idx = -1;
    *bm = info.bm;
    *bn = info.bn;
    return true;
  }
  const int P = parts_of_v(variant);
  int idx = -1;
  if (tile >= nf + tc_num_tiles()) {  // a fused-split tile
    const int f = tile - nf - tc_num_tiles();
    // grouped plans run the CTA-pair fused tiles only (the first entries of
    // the fused table)
    if (f >= fused_num_tiles() || fused_tile_ts(f) || fused_tile_parts(f) != P) return false;
    fused_tile_info(f, &info);
    *ffma_idx = -1;
    *tc_idx = -1;
    *fused_idx = f;
    *bm = info.bm;
    *bn = info.bn;
    return true;
  }
  if (tile >= 0) {
    idx = tile - nf;
    if (idx < 0 || idx >= tc_num_tiles() || tc_tile_parts(idx) != P) return false;
  } else {
    for (int i = 0; i < tc_num_tiles(); ++i)  // default: the single-CTA BN = 256 tile
      if (tc_tile_parts(i) == P && tc_tile_bn(i) == 256 && !tc_tile_pair(i)) idx = i;
  }
  if (idx < 0) return false;
  tc_tile_info(idx, &info);
  *ffma_idx = -1;
  *tc_idx = idx;
  *bm = info.bm;
  *bn = info.bn;
  return true;
}

// FFMA grouped instantiations mirror the FFMA tile table (ffma_sgemm.cu).
struct GFfmaEntry {
  int smem, threads, per_sm;
  const void* kv;
  const void* ks;
};
template <int BM, int BN, int BK, int WM, int WN, int ST, bool PAIR>
static GFfmaEntry gffma_entry() {
  using S = FfmaShape<BM, BN, BK, WM, WN, ST>;
  return {S::kSmemBytes, S::kThreads, S::kMinBlocks,
          reinterpret_cast<const void*>(&ffma_grouped_kernel<BM, BN, BK, WM, WN, ST, true, PAIR>),
          reinterpret_cast<const void*>(&ffma_grouped_kernel<BM, BN, BK, WM, WN, ST, false, PAIR>)};
}
static GFfmaEntry gffma_table(int idx) {
  switch (idx) {
    case 0: return gffma_entry<128, 128, 16, 64, 64, 4, true>();
    case 1: return gffma_entry<128, 256, 16, 64, 64, 4, true>();
    case 2: return gffma_entry<64, 64, 16, 32, 32, 4, true>();
    case 3: return gffma_entry<128, 64, 16, 64, 32, 4, true>();
    case 4: return gffma_entry<128, 256, 32, 64, 64, 3, true>();
    case 5: return gffma_entry<256, 128, 16, 64, 64, 4, true>();
    case 6: return gffma_entry<128, 128, 32, 64, 64, 3, true>();
    case 7: return gffma_entry<128, 128, 16, 64, 64, 4, false>();
    default: return gffma_entry<128, 128, 16, 64, 32, 4, true>();
  }
}

struct GTcEntry {
  int smem;
  const void* k0;
  const void* k1;
};
#define HBSG_GTC_ENTRY(P, BN, ST)                                                        \
  GTcEntry{TcShape<P, BN, ST>::kSmemBytes,                                               \
           reinterpret_cast<const void*>(&tc_grouped_kernel<P, BN, ST, false>),          \
           reinterpret_cast<const void*>(&tc_grouped_kernel<P, BN, ST, true>)},
static const GTcEntry kGTc[] = {HBSG_TC_TILE_LIST(HBSG_GTC_ENTRY)};
static constexpr int kNumGTc = sizeof(kGTc) / sizeof(kGTc[0]);
// The tensor-core table's CTA-pair entries (tc_gemm.cu), in its order after
// the single-CTA tiles: 256 x 256 with 3 parts (4 stages), with 2 parts (6).
#define HBSG_GTCP_ENTRY(P, BN, ST)                                                       \
  GTcEntry{TcPairShape<P, BN, ST>::kSmemBytes,                                           \
           reinterpret_cast<const void*>(&tc_grouped_pair_kernel<P, BN, ST, false>),     \
           reinterpret_cast<const void*>(&tc_grouped_pair_kernel<P, BN, ST, true>)},
static const GTcEntry kGTcPair[] = {HBSG_GTCP_ENTRY(3, 256, 4) HBSG_GTCP_ENTRY(2, 256, 6)};
static uint64_t g_tcp_masks[2][2];
#define HBSG_GTCI_ENTRY(P, BN, ST)                                                          \
  GTcEntry{TcShape<P, BN, ST>::kSmemBytes,                                                  \
           reinterpret_cast<const void*>(&tc_grouped_inline_kernel<P, BN, ST, false>),      \
           reinterpret_cast<const void*>(&tc_grouped_inline_kernel<P, BN, ST, true>)},
static const GTcEntry kGTcInline[] = {HBSG_TC_TILE_LIST(HBSG_GTCI_ENTRY)};
static uint64_t g_tci_masks[sizeof(kGTcInline) / sizeof(kGTcInline[0])][2];

static uint64_t g_ffma_masks[9][2];
static uint64_t g_tc_masks[sizeof(kGTc) / sizeof(kGTc[0])][2];

struct GFusedEntry {
  int smem;
  const void* k[2];  // [scaled]
};
#define HBSG_GFUSED_ENTRY(P, BN, ST, SST)                                                     \
  GFusedEntry{TcFusedShape<P, BN, ST, SST>::kSmemBytes,                                       \
              {reinterpret_cast<const void*>(&tc_grouped_fused_kernel<P, BN, ST, SST, false>), \
               reinterpret_cast<const void*>(&tc_grouped_fused_kernel<P, BN, ST, SST, true>)}},
static const GFusedEntry kGFused[] = {HBSG_FUSED_TILE_LIST(HBSG_GFUSED_ENTRY)};
static constexpr int kNumGFused = sizeof(kGFused) / sizeof(kGFused[0]);
static uint64_t g_fused_masks[kNumGFused][2];
static int g_fused_regs[kNumGFused][2];

// Co-resident clusters of two 320-thread CTAs of a pair kernel (0 if unknown).
static int pair_resident_clusters(const void* kernel, int smem) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(320, 1, 1);
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

// Launches of one grouped product on `st` (no host synchronisation, no
// allocation: capturable).
static cudaError_t grouped_launch(const GroupedPlan& pl, cudaStream_t st) {
  const GLayout& L = pl.L;
  const GProblem* probs = reinterpret_cast<const GProblem*>(pl.ws + L.probs_off);
  const int4* tiles = reinterpret_cast<const int4*>(pl.ws + L.tiles_off);
  if (L.num_tiles == 0) return cudaSuccess;
  if (pl.variant == HBSG_FFMA) {
    const GFfmaEntry e = gffma_table(pl.ffma_tile);
    const void* k = pl.vec ? e.kv : e.ks;
    if (!set_smem_once(k, e.smem, &g_ffma_masks[pl.ffma_tile][pl.vec ? 0 : 1]))
      return cudaErrorInvalidValue;
    int n = (int)L.num_tiles;
    int* queue = reinterpret_cast<int*>(pl.ws + L.queue_off);
    cudaError_t qe = cudaMemsetAsync(queue, 0, sizeof(int), st);
    if (qe != cudaSuccess) return qe;
    void* args[] = {&probs, &tiles, &n, &queue};
    return cudaLaunchKernel(k, dim3(pl.grid), dim3(e.threads), args, e.smem, st);
  }
  const int P = parts_of_v(pl.variant);
  const bool scaled = scaled_of_v(pl.variant);
  const int4* jobs = reinterpret_cast<const int4*>(pl.ws + L.jobs_off);
  const int4* ja = jobs;
  const int4* jb = ja + L.num_jobs_a;
  const int4* jr = jb + L.num_jobs_b;
  const int4* jc = jr + L.num_jobs_rmax;
  if (scaled) {
    cudaError_t e = cudaMemsetAsync(pl.ws + L.max_off, 0, L.colmax_bytes, st);
    if (e != cudaSuccess) return e;
    if (L.num_jobs_rmax) growmax_kernel<<<(unsigned)L.num_jobs_rmax, 256, 0, st>>>(probs, jr);
    if (L.num_jobs_cmax) gcolmax_kernel<<<(unsigned)L.num_jobs_cmax, 256, 0, st>>>(probs, jc);
  }
  if (L.num_jobs_a) {
    if (P == 3) {
      if (scaled) gsplit_a_kernel<3, true><<<(unsigned)L.num_jobs_a, 256, 0, st>>>(probs, ja);
      else gsplit_a_kernel<3, false><<<(unsigned)L.num_jobs_a, 256, 0, st>>>(probs, ja);
    } else {
      if (scaled) gsplit_a_kernel<2, true><<<(unsigned)L.num_jobs_a, 256, 0, st>>>(probs, ja);
      else gsplit_a_kernel<2, false><<<(unsigned)L.num_jobs_a, 256, 0, st>>>(probs, ja);
    }
  }
  if (L.num_jobs_b) {
    const int njb = (int)L.num_jobs_b;
    const unsigned nb = (unsigned)std::min<long>(L.num_jobs_b, 4L * pl.sms);
    if (P == 3) {
      if (scaled) gsplit_b_kernel<3, true><<<nb, 256, 0, st>>>(probs, jb, njb);
      else gsplit_b_kernel<3, false><<<nb, 256, 0, st>>>(probs, jb, njb);
    } else {
      if (scaled) gsplit_b_kernel<2, true><<<nb, 256, 0, st>>>(probs, jb, njb);
      else gsplit_b_kernel<2, false><<<nb, 256, 0, st>>>(probs, jb, njb);
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  GTiles gt;
  gt.queue = reinterpret_cast<int*>(pl.ws + L.queue_off);
  e = cudaMemsetAsync(gt.queue, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  gt.probs = probs;
  gt.tiles = tiles;
  gt.maps = reinterpret_cast<const CUtensorMap*>(pl.ws + L.maps_off);
  gt.n = (int)L.num_tiles;
  TcRun run = pl.run;
  if (pl.fused_tile >= 0) {
    run.l2_ahead = fused_l2_ahead();
    const int slot = scaled ? 1 : 0;
    const GFusedEntry& fe = kGFused[pl.fused_tile];
    const void* k = fe.k[slot];
    if (!set_smem_once(k, fe.smem, &g_fused_masks[pl.fused_tile][slot]))
      return cudaErrorInvalidValue;
    if (!fused_regs_ok(k, &g_fused_regs[pl.fused_tile][slot])) return cudaErrorInvalidConfiguration;
    void* args[] = {&gt, &run};
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(pl.grid);
    lc.blockDim = dim3(kFusedThreads);
    lc.dynamicSmemBytes = fe.smem;
    lc.stream = st;
    return cudaLaunchKernelExC(&lc, k, args);
  }
  if (pl.inline_split) {
    e = cudaMemsetAsync(pl.ws + L.sync_off, 0, L.sync_bytes, st);
    if (e != cudaSuccess) return e;
    const GTcEntry& te = kGTcInline[pl.tc_tile];
    const void* k = scaled ? te.k1 : te.k0;
    if (!set_smem_once(k, te.smem, &g_tci_masks[pl.tc_tile][scaled ? 1 : 0]))
      return cudaErrorInvalidValue;
    GTilesInline gi;
    static_cast<GTiles&>(gi) = gt;
    gi.ready = reinterpret_cast<int*>(pl.ws + L.sync_off);
    gi.job_counter = gi.ready + pl.count;
    gi.order = reinterpret_cast<const int*>(pl.ws + L.sync_off + L.sync_bytes);
    gi.job_start = gi.order + pl.count;
    gi.jobs_of = gi.job_start + pl.count + 1;
    gi.num_problems = pl.count;
    gi.num_jobs = (int)L.inline_jobs;
    void* args[] = {&gi, &run};
    return cudaLaunchKernel(k, dim3(pl.grid), dim3(384), args, te.smem, st);
  }
  if (pl.tc_tile >= kNumGTc) {  // CTA pairs (cluster dimensions compiled in)
    const int pi = pl.tc_tile - kNumGTc;
    const GTcEntry& te = kGTcPair[pi];
    const void* k = scaled ? te.k1 : te.k0;
    if (!set_smem_once(k, te.smem, &g_tcp_masks[pi][scaled ? 1 : 0])) return cudaErrorInvalidValue;
    void* args[] = {&gt, &run};
    return cudaLaunchKernel(k, dim3(pl.grid), dim3(320), args, te.smem, st);
  }
  const GTcEntry& te = kGTc[pl.tc_tile];
  const void* k = scaled ? te.k1 : te.k0;
  if (!set_smem_once(k, te.smem, &g_tc_masks[pl.tc_tile][scaled ? 1 : 0]))
    return cudaErrorInvalidValue;
  void* args[] = {&gt, &run};
  return cudaLaunchKernel(k, dim3(pl.grid), dim3(320), args, te.smem, st);
}

static int status_of(cudaError_t e) {
  if (e == cudaSuccess) return HBSG_OK;
  cudaGetLastError();
  return (e == cudaErrorInvalidValue || e == cudaErrorLaunchOutOfResources) ? HBSG_ERR_LAUNCH
                                                                            : HBSG_ERR_CUDA;
}

static int validate(int count, const hbsg_problem* pr, int variant) {
  if (count < 0 || (count > 0 && !pr)) return HBSG_ERR_INVALID_ARG;
  if (variant < HBSG_FFMA || variant > HBSG_BF16X6_SCALED) return HBSG_ERR_UNSUPPORTED;
  for (int i = 0; i < count; ++i) {
    const hbsg_problem& q = pr[i];
    if (q.m < 0 || q.n < 0 || q.k < 0) return HBSG_ERR_INVALID_ARG;
    if (q.m == 0 || q.n == 0) continue;
    if (!q.c || q.ldc < q.n) return HBSG_ERR_INVALID_ARG;
    if (q.k > 0 && (!q.a || !q.b || q.lda < q.k || q.ldb < q.n)) return HBSG_ERR_INVALID_ARG;
    if ((long)q.m * ((q.k + 31) / 32 * 4) > 0x7fffffffL) return HBSG_ERR_UNSUPPORTED;
  }
  return HBSG_OK;
}

// Builds the host copies of the tables and uploads them into the workspace.
static int plan_build(GroupedPlan* pl, int count, const hbsg_problem* pr, const hbsg_config* cfg,
                      void* ws, size_t ws_bytes) {
  int bm = 0, bn = 0;
  if (!tile_shape(pl->variant, cfg, &pl->ffma_tile, &pl->tc_tile, &pl->fused_tile, &bm, &bn))
    return HBSG_ERR_UNSUPPORTED;
  const bool fused = pl->fused_tile >= 0;
  const bool pair = pl->tc_tile >= 0 && tc_tile_pair(pl->tc_tile);
  pl->count = count;
  hbsg_config no_inline{};
  if (cfg) no_inline = *cfg;
  // fused plans split inside the product kernel already; the CTA-pair kernel
  // has no splitter warps
  no_inline.inline_split_pct = -1;
  const GSets sets = grouped_sets(count, pr, pl->variant, (fused || pair) ? &no_inline : cfg);
  pl->inline_split = sets.any_inline;
  pl->L = grouped_layout(count, pr, pl->variant, bm, bn, sets, fused);
  const GLayout& L = pl->L;
  if (!ws || ws_bytes < L.total || (reinterpret_cast<uintptr_t>(ws) & 255)) return HBSG_ERR_WORKSPACE;
  pl->ws = static_cast<uint8_t*>(ws);
  const int sms = current_device_sms(nullptr);
  if (sms < 0) return HBSG_ERR_NO_DEVICE;
  pl->sms = sms;
  const bool split = pl->variant != HBSG_FFMA;
  const int P = split ? parts_of_v(pl->variant) : 0;
  const bool scaled = split && scaled_of_v(pl->variant);

  std::vector<GProblem> probs(count);
  size_t parts_cur = L.parts_off, cmax_cur = L.max_off, rmax_cur = L.max_off + L.colmax_bytes;
  pl->vec = true;
  for (int i = 0; i < count; ++i) {
    const hbsg_problem& q = pr[i];
    GProblem g{};
    g.A = q.a;
    g.B = q.b;
    g.C = q.c;
    g.lda = q.lda;
    g.ldb = q.ldb;
    g.ldc = q.ldc;
    g.M = q.m;
    g.N = q.n;
    g.K = q.k;
    g.Kp = std::max(32, (q.k + 31) / 32 * 32);
    if (q.m > 0 && q.n > 0) {
      if ((q.lda & 3) || (q.ldb & 3) || (reinterpret_cast<uintptr_t>(q.a) & 15) ||
          (reinterpret_cast<uintptr_t>(q.b) & 15))
        pl->vec = false;
      if (split) {
        if (!fused) {
          g.Ap = pl->ws + parts_cur;
          parts_cur += al((size_t)P * q.m * g.Kp * 2, 256);
          g.Bp = pl->ws + parts_cur;
          parts_cur += al((size_t)P * q.n * g.Kp * 2, 256);
        }
        if (scaled) {
          g.colmax = reinterpret_cast<uint32_t*>(pl->ws + cmax_cur);
          cmax_cur += al((size_t)q.n * 4, 256);
          g.rowmax = reinterpret_cast<uint32_t*>(pl->ws + rmax_cur);
          rmax_cur += al((size_t)q.m * 4, 256);
        }
      }
    }
    probs[i] = g;
  }

  // tile list: problems by K descending (stable), rasterised tiles inside
  const std::vector<int>& order = sets.order;
  const int raster = cfg && cfg->raster_group > 0 ? cfg->raster_group : 8;
  std::vector<int4> tiles;
  tiles.reserve(L.num_tiles);
  for (int i : order) {
    const hbsg_problem& q = pr[i];
    if (q.m <= 0 || q.n <= 0) continue;
    const int tm = (q.m + bm - 1) / bm, tn = (q.n + bn - 1) / bn;
    for (int g0 = 0; g0 < tm; g0 += raster) {
      const int gm = std::min(raster, tm - g0);
      const int target = sets.inl[i] ? (int)inline_jobs_of(q) : 0;
      for (int c = 0; c < tn; ++c)
        for (int r = 0; r < gm; ++r) tiles.push_back(make_int4(i, (g0 + r) * bm, c * bn, target));
    }
  }

  std::vector<int4> jobs;
  std::vector<CUtensorMap> maps;
  if (split) {
    if (!fused) {
      for (int i = 0; i < count; ++i) {  // A split jobs (problems split before the product)
        const GProblem& g = probs[i];
        if (g.M <= 0 || g.N <= 0 || sets.inl[i]) continue;
        const long units = (long)g.M * (g.Kp / 8);
        for (long u = 0; u < units; u += 2048)
          jobs.push_back(make_int4(i, (int)u, (int)std::min<long>(2048, units - u), 0));
      }
      for (int i = 0; i < count; ++i) {  // B split jobs: 64 x 64 blocks
        const GProblem& g = probs[i];
        if (g.M <= 0 || g.N <= 0 || sets.inl[i]) continue;
        for (int n0 = 0; n0 < g.N; n0 += 64)  // n-major: neighbouring CTAs write one row run
          for (int k0 = 0; k0 < g.Kp; k0 += 64) jobs.push_back(make_int4(i, k0, n0, 0));
      }
    }
    if (scaled) {
      for (int i = 0; i < count; ++i) {
        const GProblem& g = probs[i];
        if (g.M <= 0 || g.N <= 0) continue;
        for (int m0 = 0; m0 < g.M; m0 += 8) jobs.push_back(make_int4(i, m0, std::min(8, g.M - m0), 0));
      }
      for (int i = 0; i < count; ++i) {
        const GProblem& g = probs[i];
        if (g.M <= 0 || g.N <= 0) continue;
        for (int n0 = 0; n0 < g.N; n0 += 256)
          for (int k0 = 0; k0 < g.K; k0 += 256) jobs.push_back(make_int4(i, n0, k0, 0));
      }
    }
    maps.resize(2 * (size_t)count);
    for (int i = 0; i < count; ++i) {
      const GProblem& g = probs[i];
      if (g.M <= 0 || g.N <= 0 || (fused && g.K <= 0)) {  // nothing is loaded for these
        memset(&maps[2 * i], 0, 2 * sizeof(CUtensorMap));
        continue;
      }
      const bool ok = fused ? fused_make_maps(pl->fused_tile, g.A, g.lda, g.B, g.ldb, g.M, g.N,
                                              g.K, &maps[2 * i], &maps[2 * i + 1])
                            : tc_make_parts_map(&maps[2 * i], g.Ap, P, g.M, g.Kp, kBM) &&
                                  tc_make_parts_map(&maps[2 * i + 1], g.Bp, P, g.N, g.Kp,
                                                    pair ? bn / 2 : bn);
      if (!ok) return HBSG_ERR_UNSUPPORTED;
    }
    pl->run.chunk_ktiles = tc_chunk_ktiles(P, cfg ? cfg->chunk_k : 0);
    pl->run.l2_ahead = tc_l2_ahead();
    pl->run.l2_keep = tc_l2_keep();
    pl->run.wait_limit_ns = kWaitLimitNs;
    pl->run.debug_skip_loads = 0;
  }

  // one synchronous upload per table
  cudaError_t e = cudaMemcpy(pl->ws + L.probs_off, probs.data(), sizeof(GProblem) * count,
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMemcpy(pl->ws + L.tiles_off, tiles.data(), sizeof(int4) * tiles.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !maps.empty())
    e = cudaMemcpy(pl->ws + L.maps_off, maps.data(), sizeof(CUtensorMap) * maps.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !jobs.empty())
    e = cudaMemcpy(pl->ws + L.jobs_off, jobs.data(), sizeof(int4) * jobs.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && pl->inline_split) {
    // order (tile order of the problems), job_start (prefix in that order), jobs_of
    std::vector<int> tabs(3 * (size_t)count + 1, 0);
    int* ord = tabs.data();
    int* jstart = ord + count;
    int* jof = jstart + count + 1;
    long acc = 0;
    for (int i = 0; i < count; ++i) {
      const int p = order[i];
      const GProblem& g = probs[p];
      const long nj = sets.inl[p] ? inline_jobs_of(pr[p]) : 0;
      (void)g;
      ord[i] = p;
      jstart[i] = (int)acc;
      jof[p] = (int)nj;
      acc += nj;
    }
    jstart[count] = (int)acc;
    if (acc > 0x7fffffffL) return HBSG_ERR_UNSUPPORTED;
    e = cudaMemcpy(pl->ws + L.sync_off + L.sync_bytes, tabs.data(), sizeof(int) * tabs.size(),
                   cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) return status_of(e);

  if (fused) {
    // CTA pairs: grid = 2 x min(tiles, co-resident clusters)
    const int slot = scaled ? 1 : 0;
    const GFusedEntry& fe = kGFused[pl->fused_tile];
    if (!set_smem_once(fe.k[slot], fe.smem, &g_fused_masks[pl->fused_tile][slot]))
      return HBSG_ERR_LAUNCH;
    int resident = fused_resident_clusters(fe.k[slot], fe.smem);
    if (resident <= 0 || resident > sms / 2) resident = sms / 2;
    pl->grid = (int)(2 * std::max<long>(1, std::min<long>(resident, L.num_tiles)));
    return HBSG_OK;
  }
  if (pair) {
    // pairs are dealt tiles statically: every cluster must be resident at once
    const int pi = pl->tc_tile - kNumGTc;
    const int slot = scaled ? 1 : 0;
    const GTcEntry& te = kGTcPair[pi];
    const void* k = slot ? te.k1 : te.k0;
    if (!set_smem_once(k, te.smem, &g_tcp_masks[pi][slot])) return HBSG_ERR_LAUNCH;
    int resident = pair_resident_clusters(k, te.smem);
    if (resident <= 0 || resident > sms / 2) resident = sms / 2;
    pl->grid = (int)(2 * std::max<long>(1, std::min<long>(resident, L.num_tiles)));
    return HBSG_OK;
  }
  const long slots = split ? sms : (long)sms * gffma_table(pl->ffma_tile).per_sm;
  pl->grid = (int)std::max<long>(1, std::min<long>(slots, L.num_tiles));
  return HBSG_OK;
}

int grouped_read_and_clear_device_error() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)) != cudaSuccess) return HBSG_ERR_CUDA;
  if (v != 0) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int));
  }
  return v;
}

}  // namespace hbsg

using namespace hbsg;

struct hbsg_grouped_plan_s {
  GroupedPlan p;
};

extern "C" {

size_t hbsg_grouped_workspace_size(int count, const hbsg_problem* problems, int variant,
                                   const hbsg_config* cfg) {
  if (validate(count, problems, variant) != HBSG_OK) return 0;
  int fi, ti, ui, bm, bn;
  if (!tile_shape(variant, cfg, &fi, &ti, &ui, &bm, &bn)) return 0;
  const bool fused = ui >= 0;
  const bool pair = ti >= 0 && tc_tile_pair(ti);
  hbsg_config no_inline{};
  if (cfg) no_inline = *cfg;
  no_inline.inline_split_pct = -1;
  return grouped_layout(count, problems, variant, bm, bn,
                        grouped_sets(count, problems, variant,
                                     (fused || pair) ? &no_inline : cfg),
                        fused).total;
}

int hbsg_grouped_plan_create(hbsg_grouped_plan* out, int count, const hbsg_problem* problems,
                             int variant, const hbsg_config* cfg, void* workspace,
                             size_t workspace_bytes) {
  if (!out) return HBSG_ERR_INVALID_ARG;
  *out = nullptr;
  int st = validate(count, problems, variant);
  if (st != HBSG_OK) return st;
  auto* h = new (std::nothrow) hbsg_grouped_plan_s();
  if (!h) return HBSG_ERR_INVALID_ARG;
  h->p.variant = variant;
  st = plan_build(&h->p, count, problems, cfg, workspace, workspace_bytes);
  if (st != HBSG_OK) {
    delete h;
    return st;
  }
  // Capture the launches once on a private stream; runs replay the graph.
  cudaStream_t cs = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const cudaError_t le = grouped_launch(h->p, cs);
    e = cudaStreamEndCapture(cs, &h->p.graph);
    if (le != cudaSuccess) e = le;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->p.exec, h->p.graph, 0);
  if (cs) cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    if (h->p.exec) cudaGraphExecDestroy(h->p.exec);
    if (h->p.graph) cudaGraphDestroy(h->p.graph);
    delete h;
    return status_of(e);
  }
  *out = h;
  return HBSG_OK;
}

int hbsg_grouped_run(hbsg_grouped_plan plan, hbsg_stream_t stream) {
  if (!plan || !plan->p.exec) return HBSG_ERR_INVALID_ARG;
  return status_of(cudaGraphLaunch(plan->p.exec, reinterpret_cast<cudaStream_t>(stream)));
}

int hbsg_grouped_plan_destroy(hbsg_grouped_plan plan) {
  if (!plan) return HBSG_ERR_INVALID_ARG;
  if (plan->p.exec) cudaGraphExecDestroy(plan->p.exec);
  if (plan->p.graph) cudaGraphDestroy(plan->p.graph);
  delete plan;
  return HBSG_OK;
}

int hbsg_gemm_grouped(int count, const hbsg_problem* problems, int variant, const hbsg_config* cfg,
                      void* workspace, size_t workspace_bytes, hbsg_stream_t stream) {
  int st = validate(count, problems, variant);
  if (st != HBSG_OK) return st;
  GroupedPlan p{};
  p.variant = variant;
  // The tables are uploaded with blocking copies; order them after prior
  // work on `stream` that may still read the workspace.
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
    return status_of(cudaGetLastError());
  st = plan_build(&p, count, problems, cfg, workspace, workspace_bytes);
  if (st != HBSG_OK) return st;
  return status_of(grouped_launch(p, reinterpret_cast<cudaStream_t>(stream)));
}

}  // extern "C"
