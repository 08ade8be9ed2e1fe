// 7-point Jacobi step on a 3-D grid for sm_100a: the suite's dense stencil
// benchmark (apps/jacobi) on the same host interface as the SGEMM path.
//
// Reference: the device kernel `kernel(c0, c1, A0, Anext, nx, ny, nz, pod_id)`
// (apps/jacobi/kernel.cpp:47-143) tiles x and y over the 16 x 8 tile group and
// streams z through scratchpad; its result must equal the host reference
// host_jacobi (apps/jacobi/main.cpp:19-48) exactly (main.cpp:141-150):
//   Anext[x,y,z] = c1 * (A[x-1] + A[x+1] + A[y-1] + A[y+1] + A[z-1] + A[z+1])
//                  - c0 * A[x,y,z]
// with neighbours outside the grid taken as 0.0f, the six-term sum taken left
// to right and the two products and the difference each rounded once (no
// fused multiply-add). Element (x, y, z) lies at ((y * nx) + x) * nz + z.
//
// B200 form: the step reads each element once and writes each once (8 bytes
// per point), so it is HBM-bound. A CTA of 32 (z) x 8 (x) threads marches
// along y over a slab of kYSlab planes: each thread keeps its column's y-1, y
// and y+1 values in registers, so only the new y+1 plane comes from DRAM,
// while the x and z neighbours come from the neighbouring threads' loads of
// the same plane (L1 hits). Loads go through the read-only path.
//
// Vector form (nz a multiple of 4, both grids 16-byte aligned): a thread owns
// 4 consecutive z of its column (one 16-byte load per plane and neighbour
// row, one 16-byte store), the z neighbours of its own 4 values are in its
// registers, those across lanes come by warp shuffle, and only the warp's
// two edge lanes load the z halo. That issues ~1/3 of the scalar form's
// instructions per point (the scalar form measured 66 % issue-active at 0.60
// of the HBM roof on 512^3).
#include <cuda_runtime.h>

#include "internal.h"

namespace hbsg {

static constexpr int kZT = 32;    // threads along z (one warp, coalesced)
static constexpr int kXT = 8;     // threads along x
static constexpr int kYSlab = 16;  // y planes per CTA

__global__ void __launch_bounds__(kZT * kXT) jacobi_kernel(float c0f, float c1f,
                                                           const float* __restrict__ A0,
                                                           float* __restrict__ An, int nx, int ny,
                                                           int nz) {
  const int z = blockIdx.x * kZT + threadIdx.x;
  const int x = blockIdx.y * kXT + threadIdx.y;
  const int y0 = blockIdx.z * kYSlab;
  if (z >= nz || x >= nx) return;
  const long sx = nz;
  const long sy = (long)nx * nz;
  const int y1 = min(ny, y0 + kYSlab);
  const long col = (long)x * sx + z;  // element (x, 0, z)
  float ym = y0 > 0 ? __ldg(A0 + col + (long)(y0 - 1) * sy) : 0.0f;
  float cur = __ldg(A0 + col + (long)y0 * sy);
  for (int y = y0; y < y1; ++y) {
    const long i = col + (long)y * sy;
    const float yp = y + 1 < ny ? __ldg(A0 + i + sy) : 0.0f;
    const float xm = x > 0 ? __ldg(A0 + i - sx) : 0.0f;
    const float xp = x < nx - 1 ? __ldg(A0 + i + sx) : 0.0f;
    const float zm = z > 0 ? __ldg(A0 + i - 1) : 0.0f;
    const float zp = z < nz - 1 ? __ldg(A0 + i + 1) : 0.0f;
    const float nb = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(xm, xp), ym), yp), zm), zp);
    An[i] = __fsub_rn(__fmul_rn(c1f, nb), __fmul_rn(c0f, cur));
    ym = cur;
    cur = yp;
  }
}

static constexpr int kZ4T = 32;  // threads along z in the vector form (128 z per warp)

__global__ void __launch_bounds__(kZ4T * kXT) jacobi_kernel4(float c0f, float c1f,
                                                             const float* __restrict__ A0,
                                                             float* __restrict__ An, int nx, int ny,
                                                             int nz) {
  const int lane = threadIdx.x;  // one warp per x row of the block
  const int zq = blockIdx.x * kZ4T + lane;
  const int x = blockIdx.y * kXT + threadIdx.y;
  const int y0 = blockIdx.z * kYSlab;
  if (x >= nx) return;  // whole warp (the warp shares x)
  const int nq = nz >> 2;
  const bool live = zq < nq;
  const int z0 = 4 * zq;
  const long sx = nz;
  const long sy = (long)nx * nz;
  const int y1 = min(ny, y0 + kYSlab);
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  // element (x, y, z0) of the first plane; lanes past the end point at the
  // row's first quad and never load or store through it
  const long col = (long)x * sx + (live ? z0 : 0);
  const bool has_xm = x > 0, has_xp = x < nx - 1;
  const bool has_zm = live && z0 > 0, has_zp = live && z0 + 4 < nz;
  auto ld4 = [](const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); };
  float4 ym = (live && y0 > 0) ? ld4(A0 + col + (long)(y0 - 1) * sy) : zero4;
  float4 cur = live ? ld4(A0 + col + (long)y0 * sy) : zero4;
  for (int y = y0; y < y1; ++y) {
    const long i = col + (long)y * sy;
    const float4 yp = (live && y + 1 < ny) ? ld4(A0 + i + sy) : zero4;
    const float4 xm = (live && has_xm) ? ld4(A0 + i - sx) : zero4;
    const float4 xp = (live && has_xp) ? ld4(A0 + i + sx) : zero4;
    // z neighbours across the thread's quad: the lanes beside it, or the
    // global halo at the warp's edges; 0 outside the grid
    const float up = __shfl_up_sync(0xffffffffu, cur.w, 1);
    const float dn = __shfl_down_sync(0xffffffffu, cur.x, 1);
    float zm0 = 0.0f, zp3 = 0.0f;
    if (has_zm) zm0 = lane > 0 ? up : __ldg(A0 + i - 1);
    if (has_zp) zp3 = lane < kZ4T - 1 ? dn : __ldg(A0 + i + 4);
    const float xs[4] = {xm.x, xm.y, xm.z, xm.w}, xq[4] = {xp.x, xp.y, xp.z, xp.w};
    const float ys[4] = {ym.x, ym.y, ym.z, ym.w}, yq[4] = {yp.x, yp.y, yp.z, yp.w};
    const float c[4] = {cur.x, cur.y, cur.z, cur.w};
    const float zm[4] = {zm0, cur.x, cur.y, cur.z}, zp[4] = {cur.y, cur.z, cur.w, zp3};
    float o[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float nb =
          __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(xs[e], xq[e]), ys[e]), yq[e]), zm[e]),
                    zp[e]);
      o[e] = __fsub_rn(__fmul_rn(c1f, nb), __fmul_rn(c0f, c[e]));
    }
    if (live) *reinterpret_cast<float4*>(An + i) = make_float4(o[0], o[1], o[2], o[3]);
    ym = cur;
    cur = yp;
  }
}

}  // namespace hbsg

using namespace hbsg;

extern "C" int hbsg_jacobi(int c0, int c1, const float* A0, float* Anext, int nx, int ny, int nz,
                           hbsg_stream_t stream) {
  if (nx < 0 || ny < 0 || nz < 0) return HBSG_ERR_INVALID_ARG;
  const long n = (long)nx * ny * nz;
  if (n == 0) return HBSG_OK;
  if (!A0 || !Anext) return HBSG_ERR_INVALID_ARG;
  // the step reads neighbours of every element: the output may not overlap the input
  const char* a = reinterpret_cast<const char*>(A0);
  const char* b = reinterpret_cast<const char*>(Anext);
  if (a < b + n * 4 && b < a + n * 4) return HBSG_ERR_INVALID_ARG;
  if (current_device_sms(nullptr) < 0) return HBSG_ERR_NO_DEVICE;
  if ((nz + kZT - 1) / kZT > 0x7fffffff || (nx + kXT - 1) / kXT > 65535 ||
      (ny + kYSlab - 1) / kYSlab > 65535)
    return HBSG_ERR_UNSUPPORTED;
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const bool vec = (nz & 3) == 0 && ((reinterpret_cast<uintptr_t>(A0) | reinterpret_cast<uintptr_t>(Anext)) & 15) == 0;
  if (vec) {
    const dim3 grid((nz / 4 + kZ4T - 1) / kZ4T, (nx + kXT - 1) / kXT, (ny + kYSlab - 1) / kYSlab);
    jacobi_kernel4<<<grid, dim3(kZ4T, kXT), 0, st>>>((float)c0, (float)c1, A0, Anext, nx, ny, nz);
  } else {
    const dim3 grid((nz + kZT - 1) / kZT, (nx + kXT - 1) / kXT, (ny + kYSlab - 1) / kYSlab);
    jacobi_kernel<<<grid, dim3(kZT, kXT), 0, st>>>((float)c0, (float)c1, A0, Anext, nx, ny, nz);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HBSG_OK : HBSG_ERR_LAUNCH;
}
