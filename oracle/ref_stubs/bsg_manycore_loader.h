/* Compile-only stand-in (see bsg_manycore_cuda.h): the HammerBlade runtime
 * header the reference Jacobi testbench includes; it declares nothing the
 * host reference function host_jacobi uses. */
#pragma once
