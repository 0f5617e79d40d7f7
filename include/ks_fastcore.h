#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* out0 += digit*b, out1 += digit*a (mod q) for one tower. Replaces reference
 * include/ks_fastcore.h:9-12. */
extern "C" void LaunchKSMultAcc(uint64_t* d_out0, uint64_t* d_out1, const uint64_t* d_digit, const uint64_t* d_b,
                                const uint64_t* d_a, uint64_t q, uint32_t n, cudaStream_t s);
/* Same for `towers` QP towers in one launch: digit tower t at d_digits[t],
 * key row d_keyRow[t] of bv/av, modulus d_mods[t]. Replaces reference
 * include/ks_fastcore.h:13-18. */
extern "C" void LaunchKSMultAccBatched(uint64_t* d_out0, uint64_t* d_out1, const uint64_t* const* d_digits,
                                       const uint64_t* d_bv, const uint64_t* d_av, const uint32_t* d_keyRow,
                                       const uint64_t* d_mods, uint32_t towers, uint32_t n, cudaStream_t s);
