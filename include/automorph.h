#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* Coefficient-domain Galois automorphism of one tower:
 * out[(j*k) mod 2n] = +-in[j], negated when the index lands in [n,2n).
 * Replaces reference include/automorph.h:4-6. */
extern "C" void LaunchAutomorphPermute(uint64_t* d_out, const uint64_t* d_in, uint32_t n, uint64_t k, uint64_t q,
                                       cudaStream_t s);
