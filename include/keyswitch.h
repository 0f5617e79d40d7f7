#pragma once
#include <cstdint>
#include <vector>

namespace gpufhe {

/* Hybrid keyswitch constants and eval key as plain arrays; the seam between
 * parameter setup and the resident keyswitch. Same fields as the reference
 * include/keyswitch.h:11-55. */
struct KeySwitchConstants {
    uint32_t n = 0;
    uint32_t sizeQl = 0;
    uint32_t sizeP = 0;
    uint32_t numPart = 0;
    uint32_t alpha = 0;
    uint32_t fullQ = 0;

    std::vector<uint64_t> qMod;
    std::vector<uint64_t> pMod;

    std::vector<uint32_t> sizePart;
    std::vector<uint32_t> sizeCompl;
    std::vector<uint32_t> startIdx;
    std::vector<std::vector<uint64_t>> partQHatInv;
    std::vector<std::vector<uint64_t>> partQHatInvPrec;
    std::vector<std::vector<uint64_t>> partSrcMod;
    std::vector<std::vector<uint64_t>> partQHatModp;
    std::vector<std::vector<uint64_t>> partComplMod;
    std::vector<std::vector<uint64_t>> partBMuLo;
    std::vector<std::vector<uint64_t>> partBMuHi;

    /* eval key, per part [evalKeyTowers][n] over full QP; tower index of QlP
     * position i is (i >= sizeQl ? i + fullQ - sizeQl : i) */
    std::vector<std::vector<uint64_t>> av;
    std::vector<std::vector<uint64_t>> bv;
    uint32_t evalKeyTowers = 0;

    std::vector<uint64_t> pHatInv;
    std::vector<uint64_t> pHatInvPrec;
    std::vector<uint64_t> pHatModq;
    std::vector<uint64_t> mdBMuLo;
    std::vector<uint64_t> mdBMuHi;
    std::vector<uint64_t> pInvModq;

    std::vector<uint64_t> rootModList;
    std::vector<uint64_t> rootValList;
};

struct KeySwitchResult {
    std::vector<uint64_t> ba0;
    std::vector<uint64_t> ba1;
};

/* Fills every constant family from the moduli (reference
 * src/ks_constants.cpp:31-102): alpha = ceil(sizeQ/numPart). */
void compute_keyswitch_constants(KeySwitchConstants& K, const std::vector<uint64_t>& moduliQ,
                                 const std::vector<uint64_t>& moduliP, uint32_t numPart);

/* Host-vector keyswitch (reference include/keyswitch.h:71-72): uploads,
 * runs the resident keyswitch, downloads. */
KeySwitchResult keyswitch_core_resident(const std::vector<uint64_t>& aTowers, const KeySwitchConstants& K);

}  // namespace gpufhe
