#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* Inverse NTT of one tower in place: Gentleman-Sande, bit-reversed in,
 * standard out, times n^-1 (n_inv with its Shoup precon). Replaces reference
 * include/intt.h:7-10. */
extern "C" void LaunchINTT_GS(uint64_t* d_x, const uint64_t* d_invroots, const uint64_t* d_invprecon,
                              uint32_t n, uint64_t q, uint64_t n_inv, uint64_t n_inv_precon, cudaStream_t s);
