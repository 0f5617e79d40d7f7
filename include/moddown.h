#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* ans = (a - b)*s mod q for one Q tower (ApproxModDown combine). Replaces
 * reference include/moddown.h:7-9. */
extern "C" void LaunchModDownCombine(uint64_t* d_ans, const uint64_t* d_a, const uint64_t* d_b, uint64_t s,
                                     uint64_t q, uint32_t n, cudaStream_t st);
