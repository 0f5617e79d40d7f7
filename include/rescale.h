#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* a[j] = (a[j]*s1 + b[j]*s2) mod q for one tower in place. Replaces
 * reference include/rescale.h:9-11. */
extern "C" void LaunchRescaleFuse(uint64_t* d_a, const uint64_t* d_b, uint64_t s1, uint64_t s2, uint64_t q,
                                  uint32_t n, cudaStream_t s);
