#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* ApproxSwitchCRTBasis: sizeQ source towers [sizeQ][n] (coefficient form)
 * -> sizeP target towers [sizeP][n]: x_i = a_i*QHatInvModq_i (Shoup),
 * dst_j = (sum_i x_i * QHatModp[i*sizeP+j]) mod p_j with mu = floor(2^128/p_j)
 * split lo/hi. Replaces reference include/basis_convert.h:9-14. */
extern "C" void LaunchApproxSwitchCRTBasis(const uint64_t* d_src, uint64_t* d_dst,
                                           const uint64_t* d_QHatInvModq, const uint64_t* d_QHatInvModqPrecon,
                                           const uint64_t* d_q, const uint64_t* d_QHatModp, const uint64_t* d_p,
                                           const uint64_t* d_mu_lo, const uint64_t* d_mu_hi, uint32_t sizeQ,
                                           uint32_t sizeP, uint32_t n, cudaStream_t s);
