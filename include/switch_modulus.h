#pragma once
#include <cuda_runtime.h>
#include <cstdint>

/* In-place switch of one tower from q_old to q_new keeping the centered
 * representative (strict v > q_old/2). Replaces reference
 * include/switch_modulus.h:7-8. */
extern "C" void LaunchSwitchModulus(uint64_t* d_v, uint64_t q_old, uint64_t q_new, uint32_t n, cudaStream_t s);
