// C++ testbench for the SGEMM hot path, following the flow of the reference
// testbench apps/sgemm/main.cpp (sgemm_multipod, :30-148):
//   inputs mat1[i] = i % 7, mat2[i] = i % 3 (or seeded U[-1,1)) -> host
//   reference product per matrix (:54-56) -> device alloc (:76-78) -> H2D
//   (:81-85) -> kernel call (:86-98, here hbsg_sgemm) -> D2H (:114-117) ->
//   validation: print each differing element, fail if SSE >= 0.01 (:119-134).
// The host reference is the oracle's restatement of host_mm (oracle/oracle.c);
// this program is test infrastructure and links the oracle for that reason.
//
// usage: sgemm_testbench N NITER [mod|uniform] [variant]
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "hbsg.h"

extern "C" {
void oracle_host_mm_batched(const float* mat1, const float* mat2, float* result, int n, int niter);
void oracle_fill_mod(float* mat1, float* mat2, long count);
}

// Mirrors BSG_CUDA_CALL: stop on the first failing call with its status.
#define CHECK_CUDA(stmt)                                                        \
  do {                                                                          \
    cudaError_t e_ = (stmt);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      fprintf(stderr, "%s failed: %s\n", #stmt, cudaGetErrorString(e_));        \
      return 2;                                                                 \
    }                                                                           \
  } while (0)
#define CHECK_HBSG(stmt)                                                        \
  do {                                                                          \
    int s_ = (stmt);                                                            \
    if (s_ != HBSG_OK) {                                                        \
      fprintf(stderr, "%s failed: %s\n", #stmt, hbsg_strerror(s_));             \
      return 2;                                                                 \
    }                                                                           \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s N NITER [mod|uniform] [variant]\n", argv[0]);
    return 1;
  }
  const int N = atoi(argv[1]);
  const int NITER = atoi(argv[2]);
  const bool uniform = argc > 3 && strcmp(argv[3], "uniform") == 0;
  const int variant = argc > 4 ? atoi(argv[4]) : HBSG_FFMA;
  printf("N=%d\nNITER=%d\n", N, NITER);

  const long count = (long)NITER * N * N;
  std::vector<float> mat1(count), mat2(count), expected(count), actual(count);
  if (uniform) {
    std::mt19937 gen;
    gen.seed(42);
    std::uniform_real_distribution<float> dist(-1, 1);
    for (long i = 0; i < count; i++) mat1[i] = dist(gen);
    for (long i = 0; i < count; i++) mat2[i] = dist(gen);
  } else {
    oracle_fill_mod(mat1.data(), mat2.data(), count);
  }
  oracle_host_mm_batched(mat1.data(), mat2.data(), expected.data(), N, NITER);

  float *d_mat1 = nullptr, *d_mat2 = nullptr, *d_result = nullptr;
  void* d_ws = nullptr;
  CHECK_CUDA(cudaMalloc(&d_mat1, count * sizeof(float)));
  CHECK_CUDA(cudaMalloc(&d_mat2, count * sizeof(float)));
  CHECK_CUDA(cudaMalloc(&d_result, count * sizeof(float)));
  CHECK_CUDA(cudaMemcpy(d_mat1, mat1.data(), count * sizeof(float), cudaMemcpyHostToDevice));
  CHECK_CUDA(cudaMemcpy(d_mat2, mat2.data(), count * sizeof(float), cudaMemcpyHostToDevice));

  if (variant == HBSG_FFMA) {
    CHECK_HBSG(hbsg_sgemm(d_mat1, d_mat2, d_result, N, NITER, nullptr));
  } else {
    size_t ws = hbsg_sgemm_workspace_size(N, NITER, variant);
    if (ws) CHECK_CUDA(cudaMalloc(&d_ws, ws));
    CHECK_HBSG(hbsg_sgemm_variant(d_mat1, d_mat2, d_result, N, NITER, variant, d_ws, ws, nullptr));
  }
  CHECK_HBSG(hbsg_check_device(nullptr));
  CHECK_CUDA(cudaMemcpy(actual.data(), d_result, count * sizeof(float), cudaMemcpyDeviceToHost));

  double sse = 0.0;
  long ndiff = 0;
  for (long i = 0; i < count; i++) {
    const float diff = expected[i] - actual[i];
    sse += (double)diff * diff;
    if (diff != 0.0f) {
      if (ndiff < 16) printf("[%ld] actual=%f, expected=%f\n", i, actual[i], expected[i]);
      ndiff++;
    }
  }
  printf("differing elements: %ld, SSE = %g\n", ndiff, sse);
  cudaFree(d_mat1);
  cudaFree(d_mat2);
  cudaFree(d_result);
  if (d_ws) cudaFree(d_ws);
  if (sse >= 0.01) {
    printf("Matrix Mismatch. SSE= %f\n", sse);
    printf("HBSG REGRESSION TEST FAILED\n");
    return 1;
  }
  printf("HBSG REGRESSION TEST PASSED\n");
  return 0;
}
