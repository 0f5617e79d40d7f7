#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

namespace gpufhe {
struct DeviceKSContext;
struct DeviceKSWork;
struct KeySwitchConstants;

/* Host key material, eval form [towers][n] (reference include/keygen.h:6-9). */
struct KeyPairHost {
    std::vector<uint64_t> s;
    std::vector<uint64_t> pkA, pkB;
};

/* 0 = uniform ternary secret (default), else exactly h nonzero coefficients. */
void set_secret_hamming_weight(uint32_t h);

/* Rotation on device pointers: c0 <- sigma_k(c0) + ba0, c1 <- ba1 with
 * (ba0, ba1) = keyswitch(sigma_k(c1)) under the rotation key in C
 * (reference rotate.cpp:118-132). d_scratch is n words; d_b0/d_b1 are
 * [towers][n] scratch. */
void rotate_ct_device(uint64_t* d_c0, uint64_t* d_c1, uint32_t k, const DeviceKSContext& C, DeviceKSWork& W,
                      uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod,
                      const std::vector<uint64_t>& root, uint64_t* d_scratch, uint64_t* d_b0, uint64_t* d_b1,
                      cudaStream_t s);
/* sigma_k on every tower of an eval-form poly in place (reference
 * rotate.cpp:70-84); d_scratch is n words. */
void automorphism_eval_device(uint64_t* d_v, uint32_t towers, uint32_t n, uint32_t k,
                              const std::vector<uint64_t>& mod, const std::vector<uint64_t>& root,
                              uint64_t* d_scratch, cudaStream_t s);
/* Host-vector rotation through the resident path (reference rotate.cpp:140-172). */
void rotate_ct_resident(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, uint32_t k,
                        const KeySwitchConstants& Krot, uint32_t towers, uint32_t n,
                        const std::vector<uint64_t>& mod, const std::vector<uint64_t>& root);

/* Seeded keygen over `moduli` (eval form): same mt19937_64 / normal
 * distribution draw order as reference src/keygen.cpp:55-112. */
KeyPairHost keygen_host(uint32_t n, const std::vector<uint64_t>& moduli, const std::vector<uint64_t>& roots,
                        uint64_t ns, double sigma, uint64_t seed);
/* Eval key for switching sOld -> s over full QP into K.av / K.bv
 * (reference src/evalkeygen.cpp:42-96); evalkeygen_host uses sOld = s^2. */
void evalkeygen_host_sold(KeySwitchConstants& K, const std::vector<uint64_t>& sQP,
                          const std::vector<uint64_t>& sOld, const std::vector<uint64_t>& pkA_QP,
                          const std::vector<uint64_t>& pkB_QP, const std::vector<uint64_t>& PModq_QP,
                          const std::vector<uint64_t>& modQP, const std::vector<uint64_t>& rootQP, uint64_t ns,
                          double sigma, uint64_t seed);
void evalkeygen_host(KeySwitchConstants& K, const std::vector<uint64_t>& sQP, const std::vector<uint64_t>& pkA_QP,
                     const std::vector<uint64_t>& pkB_QP, const std::vector<uint64_t>& PModq_QP,
                     const std::vector<uint64_t>& modQP, const std::vector<uint64_t>& rootQP, uint64_t ns,
                     double sigma, uint64_t seed);
/* Integer-coefficient encrypt / tower-0 decrypt (reference src/encdec.cpp:41-81). */
void encrypt_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, const std::vector<int64_t>& m,
                  const std::vector<uint64_t>& pkA, const std::vector<uint64_t>& pkB, uint32_t n,
                  const std::vector<uint64_t>& mod, const std::vector<uint64_t>& root, uint64_t ns, double sigma,
                  uint64_t seed);
void decrypt_host(std::vector<int64_t>& mout, const std::vector<uint64_t>& c0, const std::vector<uint64_t>& c1,
                  const std::vector<uint64_t>& s, uint32_t n, const std::vector<uint64_t>& mod,
                  const std::vector<uint64_t>& root);
}  // namespace gpufhe
