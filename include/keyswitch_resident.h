#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "keyswitch.h"

namespace gpufhe {

/* A/B switch the reference defines beside its keyswitch (reference
 * src/keyswitch_resident.cpp:16) and its rotation test writes
 * (tests/test_rot_resident.cpp:17,188-200) to time its batched inner product
 * against one launch per digit. This library runs every keyswitch as one fused
 * plan; the variable exists so such callers link, and its value changes
 * neither the launches nor the result. */
extern bool g_ks_batched;

/* Shared read-only device state for one level: constants, eval key, root
 * tables (reference include/keyswitch_resident.h:11-29). Built once by
 * ks_context_create; any number of streams may use it concurrently, each
 * with its own DeviceKSWork. `impl` owns the fused pipeline's context, which
 * keyswitch_resident runs on. The public fields carry the reference's device
 * tables under its names and layouts, for callers that compose the Launch*
 * entry points themselves:
 *   d_fr, d_fp, d_ir, d_ip  per modulus of modList: psi^bitrev(i) and its
 *                           Shoup precomputation, the same from psi^-1
 *                           (shared by every context, never freed);
 *   ninv, ninv_p            per modulus: n^-1 and its precomputation (host);
 *   d_qhi ... d_mhi, complModHost   per digit: the ApproxSwitchCRTBasis
 *                           constants of KeySwitchConstants (device; host);
 *   d_av, d_bv              per digit: the eval key rows as given (device);
 *   d_pHatInv ... d_mdMuHi  the ModDown constants (device);
 *   d_modsQlP, d_keyRow     per QlP tower: modulus and eval-key row. */
struct DeviceKSContext {
    uint32_t n = 0, sizeQl = 0, sizeP = 0, sizeQlP = 0, numPart = 0, fullQ = 0;
    std::vector<uint64_t> modList;
    std::vector<uint64_t*> d_fr, d_fp, d_ir, d_ip;
    std::vector<uint64_t> ninv, ninv_p;
    std::vector<uint32_t> sizePart, sizeCompl, startIdx;
    std::vector<std::vector<uint64_t>> complModHost;
    std::vector<uint64_t*> d_qhi, d_qhip, d_srcMod, d_qmp, d_complMod, d_mlo, d_mhi;
    std::vector<uint64_t*> d_av, d_bv;
    uint64_t *d_pHatInv = nullptr, *d_pHatInvPrec = nullptr, *d_pMod = nullptr, *d_pHatModq = nullptr,
             *d_qMod = nullptr, *d_mdMuLo = nullptr, *d_mdMuHi = nullptr;
    std::vector<uint64_t> pInvModqHost, qModHost, pModHost;
    uint64_t* d_modsQlP = nullptr;
    uint32_t* d_keyRow = nullptr;
    void* impl = nullptr;
};

/* Per-stream work buffers for one keyswitch in flight (reference
 * keyswitch_resident.h:32-39). keyswitch_resident uses d_ws (the pipeline
 * workspace) and impl (its plan); the reference's scratch buffers are
 * allocated at its sizes for callers that compose their own sequence:
 * d_part (largest digit x n), d_compl, d_res0, d_res1 (sizeQlP x n),
 * d_pwork (sizeP x n), d_qsw (sizeQl x n), d_digPtrs (sizeQlP pointers). */
struct DeviceKSWork {
    uint64_t *d_part = nullptr, *d_compl = nullptr, *d_res0 = nullptr, *d_res1 = nullptr;
    uint64_t *d_pwork = nullptr, *d_qsw = nullptr;
    const uint64_t** d_digPtrs = nullptr;
    uint64_t* d_ws = nullptr;
    void* impl = nullptr;
};

DeviceKSContext ks_context_create(const KeySwitchConstants& K);
DeviceKSWork ks_work_create(const DeviceKSContext& C);
void ks_context_destroy(DeviceKSContext& C);
void ks_work_destroy(DeviceKSWork& W);

/* Rescale one [towers][n] eval-form component in place: drop the last tower
 * into the first towers-1 (reference keyswitch_resident.h:52-55). s1/s2 are
 * qlInvModq / QlQlInvModqlDivqlModq at this level; d_scratch and d_drop are
 * n-word device buffers. Kernel launches only. */
void rescale_resident_raw(uint64_t* d_c, uint32_t towers, const DeviceKSContext& C, const std::vector<uint64_t>& s1,
                          const std::vector<uint64_t>& s2, uint64_t* d_scratch, uint64_t* d_drop, cudaStream_t s);

/* Hybrid keyswitch d_a ([sizeQl][n] eval) -> d_ba0, d_ba1 on stream s:
 * kernel launches only, no allocation, no host transfer, capturable in a CUDA
 * graph (reference keyswitch_resident.h:57-58). */
void keyswitch_resident(const uint64_t* d_a, uint64_t* d_ba0, uint64_t* d_ba1, const DeviceKSContext& C,
                        DeviceKSWork& W, cudaStream_t s);

}  // namespace gpufhe
