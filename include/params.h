/*
 * Native CKKS parameter generation, the reference's headerless params.cpp
 * functions (reference src/params.cpp:29-75; callers re-declare them, e.g.
 * tests/test_native_e2e.cpp:13-20). Same names, arguments and results.
 */
#pragma once
#include <cstdint>
#include <vector>

namespace gpufhe {
/* Appends primes q = 1 mod 2n, descending from 2^bits, skipping `avoid`,
 * until out.size() == count (reference params.cpp:29-39). */
void native_primes(std::vector<uint64_t>& out, uint32_t count, uint32_t bits, uint32_t n,
                   const std::vector<uint64_t>& avoid);
/* Smallest-generator primitive 2n-th root of unity mod q (params.cpp:42-48). */
uint64_t native_root(uint32_t n, uint64_t q);
/* s1[i] = q_last^-1 mod q_i, s2[i] = floor(Ql*(Ql^-1 mod q_last)/q_last) mod q_i
 * for i < last (params.cpp:54-75). */
void native_rescale_consts(std::vector<uint64_t>& s1, std::vector<uint64_t>& s2,
                           const std::vector<uint64_t>& mod, uint32_t last);
}  // namespace gpufhe
