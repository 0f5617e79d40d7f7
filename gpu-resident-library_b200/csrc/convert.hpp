// ApproxSwitchCRTBasis launchers shared by the reference ABI entry
// (LaunchApproxSwitchCRTBasis, ref_abi.cu) and gpufhe_approx_switch
// (convert_mma.cu). Arguments as LaunchApproxSwitchCRTBasis; every form gives
// the same bits.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace cv {

// Integer pipes: 128-bit multiply-adds and Barrett, one thread per coefficient.
cudaError_t approx_switch_integer(const uint64_t* src, uint64_t* dst, const uint64_t* qhi, const uint64_t* qhip,
                                  const uint64_t* q, const uint64_t* qmp, const uint64_t* p, const uint64_t* mulo,
                                  const uint64_t* muhi, uint32_t sizeQ, uint32_t sizeP, uint32_t n, cudaStream_t s);
// Tensor cores (tcgen05.mma kind::i8) by byte limbs.
cudaError_t approx_switch_tcgen05(const uint64_t* src, uint64_t* dst, const uint64_t* qhi, const uint64_t* qhip,
                                  const uint64_t* q, const uint64_t* qmp, const uint64_t* p, const uint64_t* mulo,
                                  const uint64_t* muhi, uint32_t sizeQ, uint32_t sizeP, uint32_t n, cudaStream_t s);
// Shapes the tcgen05 form takes: sizeQ <= 12, sizeP <= 64, n a multiple of 128.
bool tcgen05_shape(uint32_t sizeQ, uint32_t sizeP, uint32_t n);

}  // namespace cv
