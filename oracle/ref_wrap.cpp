/*
 * Builds the reference testbench's own host reference product, host_mm
 * (apps/sgemm/main.cpp:15-26), from the reference source where it lies, and
 * exports it under a C name. TEST INFRASTRUCTURE ONLY (see Makefile: target
 * `ref`). The reference fixes N at compile time (apps/sgemm/template.mk:30-31),
 * so one object is built per N; host_mm and sgemm_multipod are renamed per
 * object on the command line so several N can share one library.
 * REF_MAIN is the quoted path of apps/sgemm/main.cpp.
 */
#define HBREF_CAT2(a, b) a##b
#define HBREF_CAT(a, b) HBREF_CAT2(a, b)
#include REF_MAIN

extern "C" void HBREF_CAT(HBREF_PREFIX, N)(float* result, float* mat1, float* mat2)
{
    host_mm(result, mat1, mat2);
}
