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
 * with its own DeviceKSWork. `impl` owns the device data. */
struct DeviceKSContext {
    uint32_t n = 0, sizeQl = 0, sizeP = 0, sizeQlP = 0, numPart = 0, fullQ = 0;
    std::vector<uint64_t> modList;
    std::vector<uint32_t> sizePart, sizeCompl, startIdx;
    std::vector<uint64_t> pInvModqHost, qModHost, pModHost;
    void* impl = nullptr;
};

/* Per-stream work buffers for one keyswitch in flight (reference
 * keyswitch_resident.h:32-39): the pipeline workspace, its job tables and a
 * device operation descriptor. */
struct DeviceKSWork {
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
