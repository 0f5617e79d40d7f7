#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* Forward negacyclic NTT of one tower in place: Cooley-Tukey, standard order
 * in, bit-reversed out, result in [0,q); d_roots[i] = psi^bitrev(i) and
 * d_precon[i] = floor(d_roots[i]*2^64/q). Replaces reference include/ntt.h:8-10. */
extern "C" void LaunchNTT_CT(uint64_t* d_x, const uint64_t* d_roots, const uint64_t* d_precon,
                             uint32_t n, uint64_t q, cudaStream_t s);
