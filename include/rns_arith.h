#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* r = a*b mod q coefficient-wise for one tower (plain residues in and out).
 * Replaces reference include/rns_arith.h:7-9. */
extern "C" void LaunchRNSMultTower(const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_r,
                                   uint64_t q, uint32_t n, cudaStream_t stream);
