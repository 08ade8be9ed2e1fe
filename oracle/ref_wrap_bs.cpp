/*
 * Builds the reference Black-Scholes testbench's own host reference,
 * BlkSchlsEqEuroNoDiv with its CNDF (apps/blackscholes/bs.hpp), from the
 * reference source where it lies, and exports a loop over option records
 * under a C name. TEST INFRASTRUCTURE ONLY (see Makefile: target `ref`).
 * REF_BS_HPP is the quoted path of apps/blackscholes/bs.hpp; the testbench
 * (main.cpp:109-112) calls the function once per option in the same way.
 */
#include REF_BS_HPP

extern "C" void hbref_bs_host(OptionData* options, long n)
{
    for (long i = 0; i < n; i++) BlkSchlsEqEuroNoDiv(&options[i]);
}
