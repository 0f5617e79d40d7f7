#pragma once
#include <cstdint>
#include <vector>

#include "device_ciphertext.h"

namespace gpufhe {

/* Per-modulus root tables resident on the device (reference
 * include/ckks_ops.h:11-18). The root of each modulus is the
 * smallest-generator primitive 2n-th root (reference ckks_ops.cpp:25-38). */
struct DeviceTables {
    std::vector<uint64_t*> d_froots, d_fprecon, d_iroots, d_iprecon;
    std::vector<uint64_t> q;
    std::vector<uint64_t> ninv, ninv_precon;
    uint32_t n = 0;
    ~DeviceTables();
};

void build_device_tables(DeviceTables& T, uint32_t n, const std::vector<uint64_t>& moduli);

/* a *= b per tower (eval form), in place on the device, one launch
 * (reference ckks_ops.h:27-28). */
void mul_resident(DeviceCiphertext& a, const DeviceCiphertext& b, const DeviceTables& T, cudaStream_t stream);

/* Drops the last tower of both components: INTT(last), per survivor
 * SwitchModulus -> NTT -> a*s1 + b*s2; scratch and dropCoeff are n-word
 * device buffers (reference ckks_ops.h:33-36). */
void rescale_resident(DeviceCiphertext& ct, const DeviceTables& T, const std::vector<uint64_t>& s1,
                      const std::vector<uint64_t>& s2, cudaStream_t stream, uint64_t* scratch, uint64_t* dropCoeff);

}  // namespace gpufhe
