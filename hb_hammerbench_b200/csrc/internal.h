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
cudaError_t ffma_launch(int tile_idx, FfmaParams p, int batch, int sms, cudaStream_t st,
                        int ta = 0, int tb = 0);

// ---- split-BF16 family ----------------------------------------------------------
cudaError_t split_operand_a(const float* A, long lda, int M, int K, int Kp, int parts, bool scaled,
                            void* Ap, uint32_t* rowmax, int sms, cudaStream_t st);
cudaError_t split_operand_b(const float* B, long ldb, int K, int N, int Kp, int parts, bool scaled,
                            void* Bp, uint32_t* colmax, int sms, cudaStream_t st);
int tc_num_tiles();
bool tc_tile_info(int idx, hbsg_tile_info* out);
int tc_tile_parts(int idx);
// Best split-pass tile by score (~ the fraction of the tensor-core rate the
// tile reaches on this shape; returned in *score_out when given).
int tc_pick_tile(int M, int N, int K, int parts, int sms, int requested_splits,
                 double* score_out = nullptr);
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

// ---- fused split-BF16 family (tc_fused.cu) ---------------------------------------
struct FusedParams {
  const float* A;  // M x K, row stride lda
  const float* B;  // K x N, row stride ldb
  float* C;        // M x N, row stride ldc (the launch redirects slices to partials)
  long lda, ldb, ldc;
  int M, N, K;
  int tiles_m, tiles_n, num_tiles;
  int raster;
  int splits;        // K slices (1 = none)
  int kt_per_split;  // k-tiles (of 32) per slice
  const uint32_t* rowmax;  // scaled forms: FP32 bit patterns of max|A row| / max|B column|
  const uint32_t* colmax;
  // A-in-TMEM tiles (fused_tile_ts): B's BF16 parts made by the split pass,
  // parts[P][N][Kp] (the unfused kernels' layout); unused by the pair tiles
  const void* Bparts;
  int Kp;
};
int fused_num_tiles();
bool fused_tile_info(int idx, hbsg_tile_info* out);
int fused_tile_parts(int idx);
int fused_tile_bn(int idx);
int fused_tile_bm(int idx);     // output rows per tile (256: CTA pair, 128: A in TMEM)
int fused_tile_ts(int idx);     // 1: the A-in-TMEM single-CTA form
int fused_tile_slots(int idx, int sms);  // concurrent work units (clusters or CTAs)
int fused_pick_splits(int idx, int M, int N, int K, int requested, int sms, int* kt_per_split);
// C = A*B on fused entry idx; partial: [splits][M][N] FP32 when p.splits > 1.
cudaError_t fused_launch(int idx, FusedParams p, int raster, int chunk_k, int sms,
                         unsigned long long wait_limit_ns, cudaStream_t st, float* partial);
int fused_read_and_clear_device_error();
int fused_l2_ahead();
// Measured SM cycles one CTA of fused entry idx spends per k-tile (the
// converters' shared-memory traffic bounds it), for the schedule's cost model.
double fused_ktile_cycles(int idx);
// Fused kernels read A and B through FP32 TMA maps: 16-byte aligned bases and
// row strides that are multiples of 4 floats.
bool fused_operands_ok(const float* A, long lda, const float* B, long ldb);
// The two FP32 tensor maps (CUtensorMap, 128 bytes each) of fused entry idx.
bool fused_make_maps(int idx, const float* A, long lda, const float* B, long ldb, int M, int N,
                     int K, void* map_a, void* map_b);
// 2-D FP32 map over rows of `inner` elements (row stride ld elements), box
// {box_inner, box_outer}, 128-byte swizzle or none; zeros outside the matrix.
bool tc_make_f32_map(void* map, const void* base, int inner, int outer, long ld, int box_inner,
                     int box_outer, bool swizzle128);
// K slices of the automatic schedule for `tiles` output tiles on `slots`
// concurrent work slots (requested > 0 overrides); shared by both families.
int tc_slices(long tiles, int K, int slots, int requested, int* kt_per_split);
// Row / column maxima of |x| (FP32 bit patterns) for the scaled forms.
cudaError_t maxabs_rows(const float* A, long lda, int M, int K, uint32_t* rowmax, cudaStream_t st);
cudaError_t maxabs_cols(const float* B, long ldb, int K, int N, uint32_t* colmax, cudaStream_t st);

// Workspace of one hbsg_gemm call on these operands (their alignment decides
// whether a fused-split schedule may run).
size_t gemm_workspace_exact(int trans_a, int trans_b, int m, int n, int k, const float* a,
                            long lda, const float* b, long ldb, int variant,
                            const hbsg_config* cfg);

// ---- device state -------------------------------------------------------------
// Device ordinals the per-device tables cover (one bit each in a uint64_t).
static constexpr int kMaxDevices = 64;

// Returns the SM count of the current device (cached per device), or -1 when
// no sm_100 device is current (or its ordinal is >= kMaxDevices).
int current_device_sms(int* device_out);

// Sets a kernel's dynamic shared memory limit once per device (one bit of
// *device_mask per device ordinal).
bool set_smem_once(const void* func, int bytes, uint64_t* device_mask);

}  // namespace hbsg
