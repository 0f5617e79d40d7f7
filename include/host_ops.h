#pragma once
#include <cstdint>
#include <vector>

/* Host-vector helpers that the reference defines without a header (in
 * src/rotate.cpp and src/ptops.cpp) and that its tests declare where they
 * call them (tests/test_rotate.cpp:15, test_ptops.cpp:17-23,
 * test_c2s_engine.cpp:20-31, test_alpha10.cpp:19-22, test_poly2.cpp:17-23,
 * test_modraise.cpp:20). Vectors are [towers][n] eval form, tower t modulo
 * mod[t]. Each call runs on the current device and returns after its result
 * is back in host memory; errors throw std::invalid_argument (bad sizes, even
 * Galois element) or std::runtime_error (CUDA failures). */
namespace gpufhe {
struct KeySwitchConstants;

/* sigma_k on every tower in place; v is left with towers*n words
 * (reference rotate.cpp:87-101). k odd. */
void automorphism_eval_host(std::vector<uint64_t>& v, uint32_t towers, uint32_t n, uint32_t k,
                            const std::vector<uint64_t>& mod, const std::vector<uint64_t>& root);
/* out = NTT of the integer plaintext m embedded mod each tower
 * (reference rotate.cpp:104-112). */
void pt_to_eval_host(std::vector<uint64_t>& out, const std::vector<int64_t>& m, uint32_t towers, uint32_t n,
                     const std::vector<uint64_t>& mod, const std::vector<uint64_t>& root);
/* Homomorphic rotation (sigma_k(c0) + ba0, ba1) with (ba0, ba1) the
 * keyswitch of sigma_k(c1) under the rotation key in Krot
 * (reference rotate.cpp:176-188). */
void rotate_ct_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, uint32_t k, const KeySwitchConstants& Krot,
                    uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod,
                    const std::vector<uint64_t>& root);
/* c0 += d0, c1 += d1 on the first towers*n words (reference ptops.cpp:13-18). */
void ct_add_ct_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, const std::vector<uint64_t>& d0,
                    const std::vector<uint64_t>& d1, uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod);
/* c0 *= ptEval, c1 *= ptEval on the first towers*n words (reference ptops.cpp:20-26). */
void ct_mul_pt_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, const std::vector<uint64_t>& ptEval,
                    uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod);
}  // namespace gpufhe
