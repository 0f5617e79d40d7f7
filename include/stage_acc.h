#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* acc0 += b0*d, acc1 += b1*d (mod q), one tower. Replaces reference
 * include/stage_acc.h:4-7. */
extern "C" void LaunchPtMulAcc(uint64_t* d_acc0, uint64_t* d_acc1, const uint64_t* d_b0, const uint64_t* d_b1,
                               const uint64_t* d_d, uint64_t q, uint32_t n, cudaStream_t s);
/* a = a + b mod q, one tower. Replaces reference include/stage_acc.h:8-9. */
extern "C" void LaunchAddInto(uint64_t* d_a, const uint64_t* d_b, uint64_t q, uint32_t n, cudaStream_t s);
