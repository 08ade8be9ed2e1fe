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
  const dim3 grid((nz + kZT - 1) / kZT, (nx + kXT - 1) / kXT, (ny + kYSlab - 1) / kYSlab);
  jacobi_kernel<<<grid, dim3(kZT, kXT), 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      (float)c0, (float)c1, A0, Anext, nx, ny, nz);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HBSG_OK : HBSG_ERR_LAUNCH;
}
