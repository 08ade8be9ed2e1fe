/*
 * Builds the reference Jacobi testbench's own host reference, host_jacobi
 * (apps/jacobi/main.cpp:19-48), from the reference source where it lies, and
 * exports it under a C name. TEST INFRASTRUCTURE ONLY (see Makefile: target
 * `ref`). REF_JACOBI_MAIN is the quoted path of apps/jacobi/main.cpp; its
 * grid size macros (NX, NY, NZ) only size the testbench's own run, which this
 * build never calls, so they are set to 1.
 */
#include REF_JACOBI_MAIN

extern "C" void hbref_host_jacobi(int c0, int c1, float* A0, float* Anext, int nx, int ny, int nz)
{
    host_jacobi(c0, c1, A0, Anext, nx, ny, nz);
}
