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
 *   oracle_bs_host         apps/blackscholes/bs.hpp:5-125 (CNDF,
 *                          BlkSchlsEqEuroNoDiv): the host reference the
 *                          testbench validates against (main.cpp:109-141),
 *                          with the C library's expf, logf and sqrt.
 *   oracle_bs_device       apps/blackscholes/bs_kernel.hpp:33-198 (my_logf,
 *                          expf_0, fast_expf, dual_CNDF,
 *                          BlkSchlsEqEuroNoDiv_kernel): the device kernel's
 *                          own arithmetic, built only from IEEE operations.
 *                          Each fmadd_asm / fnmsub_asm is one fmaf; every
 *                          other product, sum, quotient and square root is
 *                          rounded on its own (the device build is ISO
 *                          C++14 with no contraction of plain expressions).
 *   Both work in place on option records of 8 floats (option_data.hpp:2-13:
 *   s, strike, r, v, t, call, put, unused), writing call and put only.
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

/* ---- Black-Scholes (apps/blackscholes) ---------------------------------- */

enum { BS_S = 0, BS_STRIKE = 1, BS_R = 2, BS_V = 3, BS_T = 4, BS_CALL = 5, BS_PUT = 6, BS_REC = 8 };

/* CNDF restated (bs.hpp:6-58): Hull's polynomial approximation of the
 * cumulative normal, with expf from the C library. */
static float bs_host_cndf(float InputX)
{
    int sign = 0;
    if (InputX < 0.0f) {
        InputX = -InputX;
        sign = 1;
    }
    const float xInput = InputX;
    const float expValues = expf(-0.5f * InputX * InputX);
    const float xNPrimeofX = expValues * 0.39894228040143270286f;
    float xK2 = 0.2316419f * xInput;
    xK2 = 1.0f + xK2;
    xK2 = 1.0f / xK2;
    const float xK2_2 = xK2 * xK2;
    const float xK2_3 = xK2_2 * xK2;
    const float xK2_4 = xK2_3 * xK2;
    const float xK2_5 = xK2_4 * xK2;
    float xLocal_1 = xK2 * 0.319381530f;
    float xLocal_2 = xK2_2 * (-0.356563782f);
    float xLocal_3 = xK2_3 * 1.781477937f;
    xLocal_2 = xLocal_2 + xLocal_3;
    xLocal_3 = xK2_4 * (-1.821255978f);
    xLocal_2 = xLocal_2 + xLocal_3;
    xLocal_3 = xK2_5 * 1.330274429f;
    xLocal_2 = xLocal_2 + xLocal_3;
    xLocal_1 = xLocal_2 + xLocal_1;
    float xLocal = xLocal_1 * xNPrimeofX;
    xLocal = 1.0f - xLocal;
    return sign ? 1.0f - xLocal : xLocal;
}

/* BlkSchlsEqEuroNoDiv restated (bs.hpp:60-125), n records in place. */
void oracle_bs_host(float* data, long n)
{
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        float* o = data + i * BS_REC;
        const float s = o[BS_S], k = o[BS_STRIKE], r = o[BS_R], v = o[BS_V], t = o[BS_T];
        const float sqrt_t = sqrtf(t);
        const float logValues = logf(s / k);
        float xPowerTerm = v * v;
        xPowerTerm = xPowerTerm * 0.5f;
        float xD1 = r + xPowerTerm;
        xD1 = xD1 * t;
        xD1 = xD1 + logValues;
        const float xDen = v * sqrt_t;
        xD1 = xD1 / xDen;
        const float xD2 = xD1 - xDen;
        const float NofXd1 = bs_host_cndf(xD1);
        const float NofXd2 = bs_host_cndf(xD2);
        const float FutureValueX = k * expf(-r * t);
        o[BS_CALL] = (s * NofXd1) - (FutureValueX * NofXd2);
        const float NegNofXd1 = 1.0f - NofXd1;
        const float NegNofXd2 = 1.0f - NofXd2;
        o[BS_PUT] = (FutureValueX * NegNofXd2) - (s * NegNofXd1);
    }
}

/* my_logf (bs_kernel.hpp:33-49): Taylor series of ln around 1, Horner form. */
static float bs_dev_logf(float x)
{
    const float diff = x - 1.0f;
    float r = fmaf(diff, 0.20000000f, -0.25000000f);
    r = fmaf(r, diff, 0.33333333f);
    r = fmaf(r, diff, -0.50000000f);
    r = fmaf(r, diff, 1.00000000f);
    return r * diff;
}

/* expf_0 (bs_kernel.hpp:52-65): Taylor series of exp around 0. */
static float bs_dev_exp0(float x)
{
    float r = fmaf(x, 0.0083333338f, 0.04166667f);
    r = fmaf(r, x, 0.16666666f);
    r = fmaf(r, x, 0.5f);
    r = fmaf(r, x, 1.0f);
    r = fmaf(r, x, 1.0f);
    return r;
}

/* fast_expf (bs_kernel.hpp:69-91), x < 0: whole steps of e^-1, one optional
 * e^-0.5 step, then expf_0 of the remainder; 0 below -15. */
static float bs_dev_fast_expf(float x)
{
    if (x < -15.0f) return 0.0f;
    float part1 = 1.0f;
    while (x <= -1.0f) {
        part1 *= 0.36787945f;
        x += 1.0f;
    }
    if (x <= -0.5f) {
        part1 *= 0.60653066f;
        x += 0.5f;
    }
    return part1 * bs_dev_exp0(x);
}

/* One CNDF of dual_CNDF (bs_kernel.hpp:95-160); the two lanes there are
 * independent and identical. */
static float bs_dev_cndf(float x)
{
    const int sign = x < 0.0f;
    const float xa = fabsf(x);
    const float e = bs_dev_fast_expf(-0.5f * xa * xa) * 0.39894228040143270286f;
    float k = fmaf(0.2316419f, xa, 1.0f);
    k = 1.0f / k;
    float f = fmaf(k, 1.330274429f, -1.821255978f);
    f = fmaf(f, k, 1.781477937f);
    f = fmaf(f, k, -0.356563782f);
    f = fmaf(f, k, 0.319381530f);
    f = f * k;
    float out = fmaf(-f, e, 1.0f); /* fnmsub: -(f * e) + 1, one rounding */
    if (sign) out = 1.0f - out;
    return out;
}

/* BlkSchlsEqEuroNoDiv_kernel restated (bs_kernel.hpp:163-198), n records in place. */
void oracle_bs_device(float* data, long n)
{
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        float* o = data + i * BS_REC;
        const float s = o[BS_S], k = o[BS_STRIKE], v = o[BS_V], t = o[BS_T], r = o[BS_R];
        const float sqrt_t = sqrtf(t);
        const float logValues = (s == k) ? 0.0f : bs_dev_logf(s / k);
        float xD1 = fmaf(v * v, 0.5f, r);
        xD1 = fmaf(xD1, t, logValues);
        const float xDen = v * sqrt_t;
        xD1 = xD1 / xDen;
        const float xD2 = xD1 - xDen;
        const float c1 = bs_dev_cndf(xD1);
        const float c2 = bs_dev_cndf(xD2);
        const float fv = k * bs_dev_exp0(-r * t);
        o[BS_CALL] = (s * c1) - (fv * c2);
        const float n1 = 1.0f - c1;
        const float n2 = 1.0f - c2;
        o[BS_PUT] = (fv * n2) - (s * n1);
    }
}

int oracle_version(void) { return 1; }
