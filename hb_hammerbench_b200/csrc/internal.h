// Internal interfaces between the C-ABI layer (api.cu) and the kernel files.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/hbsg.h"

namespace hbsg {

// ---- FFMA family ------------------------------------------------------------
struct FfmaParams {
  const float* A;
  const float* B;
  float* C;
  float* partial;  // split-K slices, [batch][split][M][N]
  long lda, ldb, ldc;
  long strideA, strideB, strideC;  // batch strides in elements
  int M, N, K;
  int k_per_split;
  int splits;
  int tiles_m, tiles_n;
  int raster;
  bool vec_store;
};

int ffma_num_tiles();
bool ffma_tile_info(int idx, hbsg_tile_info* out);
int ffma_pick_tile(int M, int N, int K, int batch, int num_sms);
size_t ffma_workspace_bytes(int M, int N, int batch, int splits);
cudaError_t ffma_launch(int tile_idx, FfmaParams p, int batch, cudaStream_t st, int ta = 0,
                        int tb = 0);

// ---- split-BF16 family ----------------------------------------------------------
cudaError_t split_operand_a(const float* A, long lda, int M, int K, int Kp, int parts, bool scaled,
                            void* Ap, uint32_t* rowmax, int sms, cudaStream_t st);
cudaError_t split_operand_b(const float* B, long ldb, int K, int N, int Kp, int parts, bool scaled,
                            void* Bp, uint32_t* colmax, int sms, cudaStream_t st);
int tc_num_tiles();
bool tc_tile_info(int idx, hbsg_tile_info* out);
int tc_tile_parts(int idx);
int tc_pick_tile(int M, int N, int K, int parts, int sms, int requested_splits);
cudaError_t tc_launch(int idx, const void* Ap, const void* Bp, int M, int N, int K, int Kp,
                      float* C, long ldc, const uint32_t* rowmax, const uint32_t* colmax,
                      int raster, int chunk_k, int sms, int debug_skip_loads,
                      unsigned long long wait_limit_ns, cudaStream_t st, int splits = 1,
                      float* partial = nullptr);
int tc_pick_splits(int idx, int M, int N, int K, int requested, int sms, int* kt_per_split);
int ffma_pick_splits(int tile_idx, int M, int N, int K, int batch, int requested, int sms);
// C[b] = sum over s of partial[b][s] (fixed order), partial rows of N floats.
cudaError_t splitk_reduce(const float* partial, float* C, int M, int N, long ldc, long strideC,
                          int splits, int batches, int sms, cudaStream_t st);
int tc_read_and_clear_device_error();
int grouped_read_and_clear_device_error();
int tc_chunk_ktiles(int parts, int chunk_k);
int tc_l2_ahead();
int tc_l2_keep();
bool tc_make_parts_map(void* map, const void* parts, int P, int rows, int Kp, int box_rows);
int tc_tile_bn(int idx);
int tc_tile_pair(int idx);

// ---- device state -------------------------------------------------------------
// Returns the SM count of the current device (cached per device), or -1 when
// no sm_100 device is current.
int current_device_sms(int* device_out);

// Sets a kernel's dynamic shared memory limit once per device.
bool set_smem_once(const void* func, int bytes, uint32_t* device_mask);

}  // namespace hbsg
