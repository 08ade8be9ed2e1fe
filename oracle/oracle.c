/*
 * CPU oracle for the SGEMM hot path. TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the arithmetic of the HammerBench SGEMM
 * benchmark (apps/sgemm) so that the GPU kernels of hb_hammerbench_b200 can be
 * checked against it. Only the test-suite, the smoke check and the CPU
 * baseline leg of bench.py load it; the product library never does.
 *
 * Functions and the reference lines they restate:
 *   oracle_host_mm_rows    apps/sgemm/main.cpp:15-26 (host_mm): for each y, x a
 *                          float sum starting at 0.0f, z ascending,
 *                          `sum += a*b` with the product and the add rounded
 *                          separately (this file is built with
 *                          -ffp-contract=off so the compiler cannot fuse them).
 *                          Generalised from the compile-time square N to
 *                          M x N x K with leading dimensions and a row range
 *                          (rows are independent, so a row range is an exact
 *                          sub-computation).
 *   oracle_host_mm_fma     apps/sgemm/kernel.cpp:24-32,186-275,293-322 (device
 *                          kernel): every output starts from 0.0f (reset_out)
 *                          and receives one fmaf per k in ascending k order
 *                          (z blocks ascending, sz, sz+1 inside a block); the
 *                          partial sum round-trips through the scratchpad
 *                          unchanged between blocks.
 *   oracle_gemm_f64        FP64 product used to measure error: every product
 *                          of two floats is exact in double; the sum is taken
 *                          in double, k ascending.
 *   oracle_split_bf16      The split of an FP32 value into round-to-nearest-
 *                          even BF16 parts hi, mid, lo (each part rounds the
 *                          exact remainder of the previous ones), optionally
 *                          after an exact power-of-two scale. Restates the
 *                          published split-precision method; used to check the
 *                          GPU split pass bit for bit.
 *   oracle_fill_*          Input generators of the reference testbench
 *                          (apps/sgemm/main.cpp:49-52; legacy fixtures in
 *                          apps/legacy/gemm/sgemm_512/main.cpp:69-80 and
 *                          apps/legacy/gemm/sgemm_data_parallel/main.cpp:206-223).
 *   oracle_host_jacobi     apps/jacobi/main.cpp:19-48 (host_jacobi): the
 *                          7-point Jacobi step Anext = c1*(sum of the six
 *                          neighbours, zero outside the grid, summed x-1, x+1,
 *                          y-1, y+1, z-1, z+1 left to right) - c0*self, each
 *                          product and the difference rounded separately;
 *                          element (x, y, z) at ((y*nx)+x)*nz + z.
 *   oracle_fill_jacobi     apps/jacobi/main.cpp:70-73: A0[i] = i % 13.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* host_mm restated (apps/sgemm/main.cpp:15-26), general sizes, rows [row0,row1). */
void oracle_host_mm_rows(int M, int N, int K,
                         const float* A, long lda,
                         const float* B, long ldb,
                         float* C, long ldc,
                         int row0, int row1)
{
    (void)M;
    for (int y = row0; y < row1; y++) {
        for (int x = 0; x < N; x++) {
            float sum = 0.0f;
            for (int z = 0; z < K; z++) {
                float prod = A[(long)y * lda + z] * B[(long)z * ldb + x];
                sum = sum + prod;
            }
            C[(long)y * ldc + x] = sum;
        }
    }
}

/* Same loop, rows split over OpenMP threads (used for the multi-core CPU
 * baseline; per-element arithmetic is unchanged). Returns threads used. */
int oracle_host_mm_rows_mt(int M, int N, int K,
                           const float* A, long lda,
                           const float* B, long ldb,
                           float* C, long ldc,
                           int row0, int row1, int nthreads)
{
    int used = 1;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
    #pragma omp parallel num_threads(nthreads)
    {
        #pragma omp single
        used = omp_get_num_threads();
        #pragma omp for schedule(dynamic, 1)
        for (int y = row0; y < row1; y++)
            oracle_host_mm_rows(M, N, K, A, lda, B, ldb, C, ldc, y, y + 1);
    }
#else
    (void)nthreads;
    oracle_host_mm_rows(M, N, K, A, lda, B, ldb, C, ldc, row0, row1);
#endif
    return used;
}

/* Square batched form with the reference's argument meaning:
 * NITER independent N x N products, matrix i at offset N*N*i
 * (apps/sgemm/main.cpp:54-56, kernel.cpp:293-297). */
void oracle_host_mm_batched(const float* mat1, const float* mat2, float* result,
                            int n, int niter)
{
    for (int i = 0; i < niter; i++) {
        long off = (long)n * n * i;
        oracle_host_mm_rows(n, n, n, mat1 + off, n, mat2 + off, n,
                            result + off, n, 0, n);
    }
}

/* Device-kernel arithmetic restated: one fmaf per k, ascending, from 0.0f. */
void oracle_host_mm_fma(int M, int N, int K,
                        const float* A, long lda,
                        const float* B, long ldb,
                        float* C, long ldc)
{
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < M; y++) {
        for (int x = 0; x < N; x++) {
            float acc = 0.0f;
            for (int z = 0; z < K; z++)
                acc = fmaf(A[(long)y * lda + z], B[(long)z * ldb + x], acc);
            C[(long)y * ldc + x] = acc;
        }
    }
}

/* FP64 product: exact float products, double sum, k ascending. */
void oracle_gemm_f64(int M, int N, int K,
                     const float* A, long lda,
                     const float* B, long ldb,
                     double* C, long ldc)
{
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < M; y++) {
        for (int x = 0; x < N; x++) {
            double acc = 0.0;
            for (int z = 0; z < K; z++)
                acc += (double)A[(long)y * lda + z] * (double)B[(long)z * ldb + x];
            C[(long)y * ldc + x] = acc;
        }
    }
}

/* ---- BF16 split ---------------------------------------------------------- */

/* float -> bf16 bits, round to nearest, ties to even (NaN kept quiet). */
uint16_t oracle_f32_to_bf16_rne(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu))
        return (uint16_t)((u >> 16) | 0x0040u);
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}

float oracle_bf16_to_f32(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* Exponent e such that 2^e > max|x| >= 2^(e-1) over a vector (0 if all zero
 * or non-finite). Scaling by 2^-e puts the largest magnitude in [0.5, 1). */
int oracle_pow2_exponent(const float* x, long n, long stride)
{
    float mx = 0.0f;
    for (long i = 0; i < n; i++) {
        float a = fabsf(x[i * stride]);
        if (isfinite(a) && a > mx) mx = a;
    }
    if (mx == 0.0f) return 0;
    int e;
    frexpf(mx, &e);
    return e;
}

/* Split n values: v' = v * 2^-exp, hi = bf16(v'), mid = bf16(v' - hi),
 * lo = bf16(v' - hi - mid). Each remainder is exact in FP32. parts = 2 or 3.
 * Output arrays of n bf16 bit patterns each (lo ignored when parts == 2). */
void oracle_split_bf16(const float* v, long n, int exp, int parts,
                       uint16_t* hi, uint16_t* mid, uint16_t* lo)
{
    for (long i = 0; i < n; i++) {
        float x = ldexpf(v[i], -exp);
        uint16_t h = oracle_f32_to_bf16_rne(x);
        float r1 = x - oracle_bf16_to_f32(h);
        uint16_t m = oracle_f32_to_bf16_rne(r1);
        hi[i] = h;
        mid[i] = m;
        if (parts == 3) {
            float r2 = r1 - oracle_bf16_to_f32(m);
            lo[i] = oracle_f32_to_bf16_rne(r2);
        }
    }
}

/* ---- input generators ---------------------------------------------------- */

/* apps/sgemm/main.cpp:49-52: mat1[i] = i % 7, mat2[i] = i % 3 over NITER*N*N. */
void oracle_fill_mod(float* mat1, float* mat2, long count)
{
    for (long i = 0; i < count; i++) {
        mat1[i] = (float)(i % 7);
        mat2[i] = (float)(i % 3);
    }
}

/* apps/legacy/gemm/sgemm_512/main.cpp:69-80: A[i] = i, B = identity. */
void oracle_fill_ramp_identity(float* A, float* B, int n)
{
    for (long i = 0; i < (long)n * n; i++) {
        A[i] = (float)i;
        B[i] = 0.0f;
    }
    for (int i = 0; i < n; i++) B[(long)i * n + i] = 1.0f;
}

/* apps/legacy/gemm/sgemm_data_parallel/main.cpp:206-223: A = I (M x K),
 * B[i] = i (K x N). */
void oracle_fill_identity_ramp(float* A, int M, int K, float* B, int N)
{
    for (long i = 0; i < (long)M * K; i++) A[i] = 0.0f;
    for (int y = 0; y < M && y < K; y++) A[(long)y * K + y] = 1.0f;
    for (long i = 0; i < (long)K * N; i++) B[i] = (float)i;
}

/* host_jacobi restated (apps/jacobi/main.cpp:19-48). */
void oracle_host_jacobi(int c0, int c1, const float* A0, float* Anext, int nx, int ny, int nz)
{
    const float c0f = (float)c0;
    const float c1f = (float)c1;
#define HBSG_IDX(x, y, z) ((((long)(y) * nx) + (x)) * nz + (z))
    for (int x = 0; x < nx; x++) {
        for (int y = 0; y < ny; y++) {
            for (int z = 0; z < nz; z++) {
                const float self = A0[HBSG_IDX(x, y, z)];
                const float xm1 = x > 0 ? A0[HBSG_IDX(x - 1, y, z)] : 0.0f;
                const float xp1 = x < nx - 1 ? A0[HBSG_IDX(x + 1, y, z)] : 0.0f;
                const float ym1 = y > 0 ? A0[HBSG_IDX(x, y - 1, z)] : 0.0f;
                const float yp1 = y < ny - 1 ? A0[HBSG_IDX(x, y + 1, z)] : 0.0f;
                const float zm1 = z > 0 ? A0[HBSG_IDX(x, y, z - 1)] : 0.0f;
                const float zp1 = z < nz - 1 ? A0[HBSG_IDX(x, y, z + 1)] : 0.0f;
                const float neighbor = xm1 + xp1 + ym1 + yp1 + zm1 + zp1;
                const float a = c1f * neighbor;
                const float b = c0f * self;
                Anext[HBSG_IDX(x, y, z)] = a - b;
            }
        }
    }
#undef HBSG_IDX
}

/* apps/jacobi/main.cpp:70-73: A0[i] = i % 13. */
void oracle_fill_jacobi(float* A0, long count)
{
    for (long i = 0; i < count; i++) A0[i] = (float)(i % 13);
}

int oracle_version(void) { return 1; }
