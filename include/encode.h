/*
 * Canonical CKKS encode / decode, the reference's headerless encode.cpp
 * functions (reference src/encode.cpp:13-44; callers re-declare them, e.g.
 * tests/test_alpha10.cpp:14-15). Same names, arguments and results, bit for
 * bit: z holds N/2 slots, m N integer coefficients at scale Delta. Runs on
 * the current CUDA device through a process-wide encoder per (device, N).
 */
#pragma once
#include <complex>
#include <cstdint>
#include <vector>

namespace gpufhe {
void encode_host(std::vector<int64_t>& m, const std::vector<std::complex<double>>& z, uint32_t N, double Delta);
void decode_host(std::vector<std::complex<double>>& z, const std::vector<int64_t>& m, uint32_t N, double Delta);
}  // namespace gpufhe
