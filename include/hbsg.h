/*
 * hbsg.h -- C ABI of the B200 (sm_100a) SGEMM hot path that stands in for the
 * HammerBench `apps/sgemm` benchmark kernel.
 *
 * Conventions
 *   - All matrices are FP32, row-major unless a trans flag says otherwise,
 *     in caller-owned device memory. The library allocates nothing: every
 *     scratch buffer is caller-provided (`workspace`, sized by the matching
 *     *_workspace_size query).
 *   - Every entry point is asynchronous on `stream` (a cudaStream_t; NULL is
 *     the legacy default stream) and returns an hbsg_status (0 = success,
 *     negative = error). Argument errors are detected before anything is
 *     launched and never abort the process.
 *   - Thread-safe for calls on distinct streams with distinct workspaces.
 */
#ifndef HBSG_H
#define HBSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same object as cudaStream_t; declared here so callers need no CUDA header. */
typedef struct CUstream_st* hbsg_stream_t;

typedef enum hbsg_status {
    HBSG_OK = 0,
    HBSG_ERR_INVALID_ARG = -1,    /* null pointer, bad size, bad leading dim */
    HBSG_ERR_UNSUPPORTED = -2,    /* variant/config/alignment not supported */
    HBSG_ERR_WORKSPACE = -3,      /* workspace missing, misaligned or too small */
    HBSG_ERR_LAUNCH = -4,         /* kernel launch failed */
    HBSG_ERR_DEVICE_TIMEOUT = -5, /* a bounded device-side wait expired */
    HBSG_ERR_NO_DEVICE = -6,      /* no sm_100 device current */
    HBSG_ERR_CUDA = -7            /* other CUDA runtime error */
} hbsg_status;

/* Arithmetic forms of C = A*B. */
typedef enum hbsg_variant {
    HBSG_FFMA = 0,          /* FP32 SIMT: one fused multiply-add per k, k ascending */
    HBSG_BF16X3 = 1,        /* split-BF16 (hi, mid), 3 tensor-core products */
    HBSG_BF16X6 = 2,        /* split-BF16 (hi, mid, lo), 6 tensor-core products */
    HBSG_BF16X3_SCALED = 3, /* as BF16X3 after exact per-row (A) / per-column (B) 2^e scaling */
    HBSG_BF16X6_SCALED = 4  /* as BF16X6 after exact per-row (A) / per-column (B) 2^e scaling */
} hbsg_variant;

/* Explicit schedule (used by the autotuner). Fields left at 0 mean "library
 * heuristic". */
typedef struct hbsg_config {
    int tile;          /* tile-shape id, 1-based index into hbsg_tile_info (0 = heuristic) */
    int split_k;       /* K slices, reduced in fixed order. FFMA: 0/1 = none (keeps the one
                          sequential FMA chain per output), n > 1 = n slices. Split-BF16:
                          0 = library heuristic (slices only when the output has too few
                          tiles to fill the GPU), 1 = none, n > 1 = n slices. */
    int raster_group;  /* tile rows per rasterisation group (0 = heuristic) */
    int chunk_k;       /* split-BF16: K elements accumulated on the tensor core before the
                          partial is added in FP32 registers (0 = heuristic) */
    int flags;         /* HBSG_FLAG_* */
    int inline_split_pct; /* grouped split-BF16 plans: percent of the split work (problems
                             processed last) done by extra warps inside the product kernel
                             while the tensor cores run; 0 = library default (none),
                             < 0 = none */
} hbsg_config;

/* hbsg_config.flags. PRESPLIT_A / PRESPLIT_B: the workspace already holds the
 * BF16 split of A / B made by an earlier call with the same operand values,
 * shape, transpose flag, variant and workspace (e.g. a constant operand), so
 * the split pass for it is skipped. */
#define HBSG_FLAG_PRESPLIT_A 1
#define HBSG_FLAG_PRESPLIT_B 2
/* SPLIT_ONLY: run only the split passes (fill the workspace), no product;
 * a later call with PRESPLIT_A | PRESPLIT_B computes C from them. */
#define HBSG_FLAG_SPLIT_ONLY 4


typedef struct hbsg_tile_info {
    int variant_class; /* 0 = FFMA kernel family, 1 = split-BF16 tensor-core family */
    int bm, bn, bk;    /* CTA tile */
    int threads;       /* threads per CTA */
    int smem_bytes;    /* dynamic shared memory per CTA */
    int parts;         /* split-BF16 family: BF16 parts per operand (3 -> BF16X6 forms,
                          2 -> BF16X3 forms); 0 for the FFMA family */
    int fused;         /* 1: the FP32 -> BF16 split runs inside the product kernel
                          (row-major operands with 16-byte aligned rows only): for both
                          operands on the 256-row CTA-pair tiles (no parts in the
                          workspace); for A on the 128-row tiles, which keep A's parts in
                          tensor memory and split B in a pass into the workspace */
} hbsg_tile_info;

/* ---------------------------------------------------------------------------
 * Benchmark entry point.
 *
 * Replaces the device kernel `int kernel(float* mat1, float* mat2,
 * float* result, int pod_id)` (apps/sgemm/kernel.cpp:279-333) together with
 * its launch `hb_mc_kernel_enqueue(..., "kernel", 4, {mat1, mat2, result,
 * pod})` + `hb_mc_device_pods_kernels_execute` (apps/sgemm/main.cpp:86-98).
 * N and NITER were compile-time macros there (apps/sgemm/template.mk:30-31);
 * here they are arguments. result[i] = mat1[i] * mat2[i] for i < niter, each
 * an n x n row-major matrix at element offset n*n*i (kernel.cpp:293-297).
 * Arithmetic is that of the reference device kernel: every output starts at
 * 0.0f and receives one fused multiply-add per k in ascending k
 * (kernel.cpp:24-32,208-263), so results are bit-identical to it.
 */
int hbsg_sgemm(const float* mat1, const float* mat2, float* result,
               int n, int niter, hbsg_stream_t stream);

/* Same batch layout with a chosen variant (split-BF16 needs a workspace). */
int hbsg_sgemm_variant(const float* mat1, const float* mat2, float* result,
                       int n, int niter, int variant,
                       void* workspace, size_t workspace_bytes,
                       hbsg_stream_t stream);
size_t hbsg_sgemm_workspace_size(int n, int niter, int variant);

/* ---------------------------------------------------------------------------
 * General strided GEMM C[m x n] = op(A)[m x k] * op(B)[k x n].
 *
 * Follows the rectangular interface of the legacy data-parallel kernel
 * `kernel_mm_opt(hb_tensor_t* result, hb_tensor_t* mat1, hb_tensor_t* mat2)`
 * (apps/legacy/gemm/sgemm_data_parallel/kernel.cpp:323-344, sizes and
 * strides from hb_tensor.hpp:26-54), with optional transposed operands
 * (its transposed-A load, kernel.cpp:21-48). trans_a != 0 means A is stored
 * k x m (element (i,p) at a[p*lda + i]); likewise trans_b (B stored n x k).
 */
int hbsg_gemm(int trans_a, int trans_b, int m, int n, int k,
              const float* a, int64_t lda, const float* b, int64_t ldb,
              float* c, int64_t ldc, int variant,
              void* workspace, size_t workspace_bytes, hbsg_stream_t stream);

/* As hbsg_gemm with an explicit schedule (cfg may be NULL). */
int hbsg_gemm_ex(int trans_a, int trans_b, int m, int n, int k,
                 const float* a, int64_t lda, const float* b, int64_t ldb,
                 float* c, int64_t ldc, int variant, const hbsg_config* cfg,
                 void* workspace, size_t workspace_bytes, hbsg_stream_t stream);

/* Workspace bytes for hbsg_gemm / hbsg_gemm_ex on the current device. The
 * split-BF16 schedule, and so its K-slice partial buffer, depends on the
 * device's SM count: with no sm_100 device current the split-BF16 forms
 * report 0 (and the product call itself returns HBSG_ERR_NO_DEVICE). */
size_t hbsg_gemm_workspace_size(int m, int n, int k, int variant,
                                const hbsg_config* cfg);
/* The same for a call with transposed operands (the automatic schedule of a
 * transposed call never uses a fused-split tile, so its size can differ).
 * Both sizes cover either schedule the call may take: a fused-split tile needs
 * 16-byte aligned operand rows, which these queries cannot see. */
size_t hbsg_gemm_workspace_size_ex(int trans_a, int trans_b, int m, int n, int k, int variant,
                                   const hbsg_config* cfg);
/* The exact workspace of a call on these operands (no reference counterpart):
 * with aligned rows a fused-split schedule may need far less (no BF16 parts). */
size_t hbsg_gemm_workspace_size_for(int trans_a, int trans_b, int m, int n, int k,
                                    const float* a, int64_t lda, const float* b, int64_t ldb,
                                    int variant, const hbsg_config* cfg);

/* Where the split-BF16 path keeps the operand parts inside its workspace
 * (byte offsets from the workspace start). Parts are BF16, K-major:
 *   A parts: [parts][m][kp] at a_offset   (op(A) rows, K padded to kp with zeros)
 *   B parts: [parts][n][kp] at b_offset   (op(B) columns, transposed)
 *   rowmax / colmax: m / n uint32 FP32 bit patterns of max|row| / max|column|
 *   (scaled variants only; offsets equal total_bytes otherwise).
 * Part 0 = hi, 1 = mid, 2 = lo. */
typedef struct hbsg_split_layout {
    int parts;
    int kp;
    size_t a_offset, b_offset, rowmax_offset, colmax_offset, total_bytes;
} hbsg_split_layout;
int hbsg_get_split_layout(int m, int n, int k, int variant, hbsg_split_layout* out);

/* ---------------------------------------------------------------------------
 * Grouped GEMM: many independent row-major products C_i = A_i * B_i of uneven
 * sizes in one persistent launch.
 *
 * Generalises the reference's NITER loop of independent products
 * (apps/sgemm/kernel.cpp:293-297, all N x N) to per-problem M, N, K and
 * strides, with the output tiles of all problems scheduled on one grid
 * (cf. the grid-strided tile groups of
 * apps/legacy/gemm/sgemm_group_cooperative/kernel.cpp:285-286).
 *
 * A plan lays its tables out in the caller's workspace, uploads them once
 * (blocking copies) and captures the product's launches into a CUDA graph;
 * hbsg_grouped_run replays the graph on a stream. The plan keeps the
 * problems' pointers: rerun it whenever the operand contents change, and
 * keep the workspace alive and untouched while the plan exists.
 * hbsg_gemm_grouped builds the tables and launches directly (no graph).
 *
 * Both hbsg_grouped_plan_create and hbsg_gemm_grouped write their tables into
 * the workspace with blocking host-to-device copies that are not ordered
 * after work on other streams: the workspace must be idle (every earlier
 * launch that reads it, such as a previous hbsg_grouped_run on another
 * stream, complete) when either is called.
 */
typedef struct hbsg_problem {
    int m, n, k;
    const float* a; int64_t lda;   /* m x k, row stride lda >= k */
    const float* b; int64_t ldb;   /* k x n, row stride ldb >= n */
    float* c; int64_t ldc;         /* m x n, row stride ldc >= n */
} hbsg_problem;

typedef struct hbsg_grouped_plan_s* hbsg_grouped_plan;

size_t hbsg_grouped_workspace_size(int count, const hbsg_problem* problems, int variant,
                                   const hbsg_config* cfg);
int hbsg_grouped_plan_create(hbsg_grouped_plan* plan, int count, const hbsg_problem* problems,
                             int variant, const hbsg_config* cfg,
                             void* workspace, size_t workspace_bytes);
int hbsg_grouped_run(hbsg_grouped_plan plan, hbsg_stream_t stream);
int hbsg_grouped_plan_destroy(hbsg_grouped_plan plan);
int hbsg_gemm_grouped(int count, const hbsg_problem* problems, int variant,
                      const hbsg_config* cfg, void* workspace, size_t workspace_bytes,
                      hbsg_stream_t stream);

/* ---------------------------------------------------------------------------
 * Allocation-free split-BF16 GEMM. No counterpart in the reference.
 *
 * For callers that cannot allocate device memory at the moment they need a
 * product: applications whose memory pool has already reserved (nearly) all
 * of the GPU, so a workspace allocation would fail or force the pool to
 * release memory; and latency-critical loops, where cudaMalloc/cudaFree may
 * synchronise the device and stall every stream. Same arguments and result
 * as hbsg_gemm with a split-BF16 variant (BF16X3, BF16X6 and their _SCALED
 * forms), but the split parts live in a fixed scratch array compiled into
 * the library: HBSG_NOALLOC_SCRATCH_BYTES (16 MiB) of device memory that
 * every GPU which loads the library holds until the process exits.
 *
 *   - Problems whose workspace (hbsg_gemm_workspace_size_for on the same
 *     operands, no config) exceeds HBSG_NOALLOC_SCRATCH_BYTES are
 *     rejected with HBSG_ERR_WORKSPACE before anything is launched. With a
 *     split pass, M = N = K = 1024 BF16X6 needs 12.6 MB and fits; shapes the
 *     library serves with a fused-split tile need only the K-slice partials
 *     and, for the scaled forms, the row and column maxima.
 *   - FFMA is rejected with HBSG_ERR_UNSUPPORTED (it needs no scratch: call
 *     hbsg_gemm).
 *   - The first call on each device looks up the array's device address
 *     (set-up, no allocation); make that first call before any stream
 *     capture begins. The address is kept for the process's life and does
 *     not survive cudaDeviceReset: do not call this entry point on a device
 *     after resetting it.
 *   - All calls on a device share the one array: calls that may overlap on
 *     the GPU (different streams without ordering between them) race on it
 *     and must be serialised by the caller. Nothing needs clearing between
 *     calls: each call rewrites every scratch byte it later reads.
 */
#define HBSG_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int hbsg_gemm_noalloc(int trans_a, int trans_b, int m, int n, int k,
                      const float* a, int64_t lda, const float* b, int64_t ldb,
                      float* c, int64_t ldc, int variant, hbsg_stream_t stream);

/* ---------------------------------------------------------------------------
 * 7-point Jacobi step, the suite's dense stencil benchmark on the same host
 * interface.
 *
 * Replaces the device kernel `int kernel(int c0, int c1, float* A0,
 * float* Anext, const int nx, const int ny, const int nz, int pod_id)`
 * (apps/jacobi/kernel.cpp:47-143) with its enqueue (apps/jacobi/main.cpp:
 * 95-102). A0 and Anext are caller-owned device grids of nx*ny*nz floats,
 * element (x, y, z) at ((y*nx)+x)*nz + z, and must not overlap. Anext =
 * c1 * (sum of the six neighbours, 0 outside the grid) - c0 * A0, with the
 * host reference's operation order (apps/jacobi/main.cpp:19-48), so results
 * are bit-identical to it. Asynchronous on `stream`.
 */
int hbsg_jacobi(int c0, int c1, const float* A0, float* Anext, int nx, int ny, int nz,
                hbsg_stream_t stream);

/* ---------------------------------------------------------------------------
 * Black-Scholes European option pricing, the suite's apps/blackscholes
 * benchmark on the same host interface.
 *
 * hbsg_option has the layout of the reference's OptionData
 * (apps/blackscholes/option_data.hpp:2-13), so an array of those records
 * binds directly. Prices are the device kernel's arithmetic
 * (BlkSchlsEqEuroNoDiv_kernel, apps/blackscholes/bs_kernel.hpp:163-198):
 * Taylor-series ln and exp and Hull's cumulative normal, every step the same
 * IEEE operation, so results are bit-identical to that kernel; against the
 * host reference (bs.hpp:60-125, libm exp/log) they stay inside the
 * testbench's bound (sum of squared call and put differences <= 0.01 over
 * its 32768 options, main.cpp:119-141). Inputs are meant for the range that
 * kernel was written for (s / strike near 1, as in the benchmark's input).
 */
typedef struct hbsg_option {
    float s;      /* spot price */
    float strike; /* strike price */
    float r;      /* risk-free interest rate */
    float v;      /* volatility */
    float t;      /* time to maturity in years */
    float call;   /* output: call price */
    float put;    /* output: put price */
    float unused;
} hbsg_option;

/* Replaces the device kernel `int kernel(OptionData* data, int num_option,
 * int pod_id)` (apps/blackscholes/kernel.cpp:27-113) with its enqueue
 * (apps/blackscholes/main.cpp:79-90): prices num_option records of the
 * caller-owned device array `options` in place, writing call and put only.
 * Any num_option >= 0 (the reference kernel needs a multiple of its chunk of
 * 4). Asynchronous on `stream`. */
int hbsg_blackscholes(hbsg_option* options, int64_t num_option, hbsg_stream_t stream);

/* The same pricing on separate device arrays of n floats (28 bytes per
 * option instead of the record's 32 read and 32 written): call[i], put[i]
 * from s[i], strike[i], r[i], v[i], t[i]. call and put must not overlap each
 * other or any input. No counterpart in the reference (its records are the
 * only layout); bit-identical to hbsg_blackscholes on the same values. */
int hbsg_blackscholes_arrays(const float* s, const float* strike, const float* r,
                             const float* v, const float* t, float* call, float* put,
                             int64_t n, hbsg_stream_t stream);

/* Tile-shape table for the autotuner: number of ids and their description. */
int hbsg_num_tiles(void);
int hbsg_tile_describe(int tile, hbsg_tile_info* out);

/* ---------------------------------------------------------------------------
 * Error reporting.
 */
const char* hbsg_strerror(int status);

/* Synchronises `stream`, then reports and clears the device-side error flag
 * raised by bounded waits inside the kernels (HBSG_OK if none). */
int hbsg_check_device(hbsg_stream_t stream);

/* Test hook for the failure path of the tensor-core kernel: launches it on a
 * tiny problem with its tile loads suppressed and a 0.2 s bound on every
 * wait, so the waits expire, the kernel records HBSG_ERR_DEVICE_TIMEOUT,
 * releases its tensor memory and returns. `workspace` (>= 64 KiB, 256-byte
 * aligned) only backs the tensor maps; nothing is read or written. The next
 * hbsg_check_device reports the timeout. No reference counterpart. */
int hbsg_debug_timeout_probe(void* workspace, size_t workspace_bytes, hbsg_stream_t stream);

/* FP32 SIMT throughput probe (no reference counterpart): launches a kernel
 * of independent fused multiply-add chains on every SM of the current device
 * (packed != 0: the packed two-lane __ffma2_rn the FFMA kernel issues;
 * 0: scalar FMA) for `iters` steps and stores in *flops_out the FP32 flops it
 * performs. Time the launch on `stream` (CUDA events) to get the device's
 * FP32 roof: the denominator of the FFMA kernel's roofline fraction. `sink`
 * is one device float the kernel writes only on an impossible result. */
int hbsg_fp32_peak_probe(int packed, int iters, float* sink, double* flops_out,
                         hbsg_stream_t stream);

/* ABI version (major * 100 + minor). */
int hbsg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* HBSG_H */
