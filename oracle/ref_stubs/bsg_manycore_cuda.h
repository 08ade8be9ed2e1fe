/*
 * Compile-only stand-in for the HammerBlade CUDA-lite runtime header, which
 * is not available outside the HammerBlade toolchain. It exists so that the
 * reference testbench source apps/sgemm/main.cpp compiles on x86 and its
 * host reference product host_mm (main.cpp:15-26) can be called as the
 * CPU reference. Every runtime call below fails with HB_MC_FAIL; the
 * testbench's device path is never executed from this build.
 */
#ifndef HBSG_REF_STUB_BSG_MANYCORE_CUDA_H
#define HBSG_REF_STUB_BSG_MANYCORE_CUDA_H
#include <stdint.h>
#include <stddef.h>
#include <vector>

#define HB_MC_SUCCESS 0
#define HB_MC_FAIL (-1)
#define HB_MC_DEVICE_ID 0

typedef uint32_t eva_t;
typedef int hb_mc_pod_id_t;
typedef struct { int unused; } hb_mc_device_t;
typedef struct { uint32_t x, y; } hb_mc_dimension_t;
typedef struct { eva_t d_addr; void* h_addr; size_t size; } hb_mc_dma_htod_t;
typedef struct { eva_t d_addr; void* h_addr; size_t size; } hb_mc_dma_dtoh_t;

#define BSG_CUDA_CALL(stmt) do { int hbsg_stub_rc = (stmt); if (hbsg_stub_rc != HB_MC_SUCCESS) return hbsg_stub_rc; } while (0)
#define hb_mc_device_foreach_pod_id(dev, pod) for ((pod) = 0; (pod) < 0; (pod)++)

static inline int hb_mc_device_init(hb_mc_device_t*, const char*, int) { return HB_MC_FAIL; }
static inline int hb_mc_device_set_default_pod(hb_mc_device_t*, hb_mc_pod_id_t) { return HB_MC_FAIL; }
static inline int hb_mc_device_program_init(hb_mc_device_t*, const char*, const char*, int) { return HB_MC_FAIL; }
static inline int hb_mc_device_malloc(hb_mc_device_t*, size_t, eva_t*) { return HB_MC_FAIL; }
static inline int hb_mc_device_transfer_data_to_device(hb_mc_device_t*, const hb_mc_dma_htod_t*, size_t) { return HB_MC_FAIL; }
static inline int hb_mc_device_transfer_data_to_host(hb_mc_device_t*, const hb_mc_dma_dtoh_t*, size_t) { return HB_MC_FAIL; }
static inline int hb_mc_kernel_enqueue(hb_mc_device_t*, hb_mc_dimension_t, hb_mc_dimension_t, const char*, int, const uint32_t*) { return HB_MC_FAIL; }
static inline int hb_mc_device_pods_kernels_execute(hb_mc_device_t*) { return HB_MC_FAIL; }
static inline int hb_mc_device_finish(hb_mc_device_t*) { return HB_MC_FAIL; }
#endif
