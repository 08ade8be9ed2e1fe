/* Compile-only stand-in (see bsg_manycore_cuda.h): the regression harness's
 * program-main macro becomes empty, so the reference testbench defines only
 * its functions. */
#ifndef HBSG_REF_STUB_BSG_MANYCORE_REGRESSION_H
#define HBSG_REF_STUB_BSG_MANYCORE_REGRESSION_H
#define declare_program_main(name, fn)
#endif
