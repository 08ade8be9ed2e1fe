/* Compile-only stand-in (see bsg_manycore_cuda.h). */
#ifndef HBSG_REF_STUB_BSG_MANYCORE_EVA_H
#define HBSG_REF_STUB_BSG_MANYCORE_EVA_H
#endif
