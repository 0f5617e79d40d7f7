#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* t0 = a0*b0, t1 = a0*b1 + a1*b0, t2 = a1*b1 over sizeQ towers in one launch
 * (moduli in device array d_mods). The reference declares these without a
 * header (kernels/tensor.cu:28-36, 53-61; re-declared by callers such as
 * bench/bench_evalmult_resident.cpp:17-20). */
extern "C" void LaunchTensor(const uint64_t* c0a, const uint64_t* c1a, const uint64_t* c0b, const uint64_t* c1b,
                             uint64_t* t0, uint64_t* t1, uint64_t* t2, const uint64_t* d_mods, uint32_t sizeQ,
                             uint32_t n, cudaStream_t s);
/* r0 = t0 + ba0, r1 = t1 + ba1 over sizeQ towers. */
extern "C" void LaunchCombine(uint64_t* r0, uint64_t* r1, const uint64_t* t0, const uint64_t* t1,
                              const uint64_t* ba0, const uint64_t* ba1, const uint64_t* d_mods, uint32_t sizeQ,
                              uint32_t n, cudaStream_t s);
