/*
 * TEST INFRASTRUCTURE ONLY. C entry points over the reference's own host-only
 * sources (params.cpp, ks_constants.cpp, encode.cpp), compiled from the
 * read-only reference tree by oracle/build_ref.sh into oracle/_ref/. The
 * tests use them to pin the oracle's parameter and constant routines.
 */
#include "keyswitch.h"   /* reference include/keyswitch.h */
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace gpufhe {
void native_primes(std::vector<uint64_t>&, uint32_t, uint32_t, uint32_t, const std::vector<uint64_t>&);
uint64_t native_root(uint32_t, uint64_t);
void native_rescale_consts(std::vector<uint64_t>&, std::vector<uint64_t>&, const std::vector<uint64_t>&, uint32_t);
void encode_host(std::vector<int64_t>&, const std::vector<std::complex<double>>&, uint32_t, double);
void decode_host(std::vector<std::complex<double>>&, const std::vector<int64_t>&, uint32_t, double);
}

extern "C" {

int ref_native_primes(uint64_t* out, uint32_t count, uint32_t bits, uint32_t n,
                      const uint64_t* avoid, uint32_t navoid) {
    std::vector<uint64_t> o, av(avoid, avoid + navoid);
    try { gpufhe::native_primes(o, count, bits, n, av); } catch (...) { return -1; }
    std::memcpy(out, o.data(), o.size() * 8);
    return 0;
}

uint64_t ref_native_root(uint32_t n, uint64_t q) {
    try { return gpufhe::native_root(n, q); } catch (...) { return 0; }
}

void ref_rescale_consts(uint64_t* s1, uint64_t* s2, const uint64_t* mod, uint32_t nmod, uint32_t last) {
    std::vector<uint64_t> a, b, m(mod, mod + nmod);
    gpufhe::native_rescale_consts(a, b, m, last);
    std::memcpy(s1, a.data(), a.size() * 8);
    std::memcpy(s2, b.data(), b.size() * 8);
}

/* compute_keyswitch_constants flattened in the oracle's layout
 * (orc_ks_constants). Returns the alpha the reference derived. */
uint32_t ref_ks_constants(uint64_t* out, const uint64_t* Q, uint32_t L, const uint64_t* P,
                          uint32_t K, uint32_t numPart) {
    gpufhe::KeySwitchConstants C;
    std::vector<uint64_t> q(Q, Q + L), p(P, P + K);
    gpufhe::compute_keyswitch_constants(C, q, p, numPart);
    uint64_t* o = out;
    auto put = [&](const std::vector<uint64_t>& v) { std::memcpy(o, v.data(), v.size() * 8); o += v.size(); };
    for (uint32_t i = 0; i < C.numPart; ++i) {
        put(C.partQHatInv[i]); put(C.partQHatInvPrec[i]); put(C.partSrcMod[i]); put(C.partQHatModp[i]);
        put(C.partComplMod[i]); put(C.partBMuLo[i]); put(C.partBMuHi[i]);
    }
    put(C.pHatInv); put(C.pHatInvPrec); put(C.pHatModq); put(C.mdBMuLo); put(C.mdBMuHi); put(C.pInvModq);
    return C.alpha;
}

void ref_encode(int64_t* m, const double* zre, const double* zim, uint32_t N, double Delta) {
    std::vector<std::complex<double>> z(N / 2);
    for (uint32_t i = 0; i < N / 2; ++i) z[i] = {zre[i], zim[i]};
    std::vector<int64_t> o;
    gpufhe::encode_host(o, z, N, Delta);
    std::memcpy(m, o.data(), o.size() * 8);
}

void ref_decode(double* zre, double* zim, const int64_t* m, uint32_t N, double Delta) {
    std::vector<int64_t> mm(m, m + N);
    std::vector<std::complex<double>> z;
    gpufhe::decode_host(z, mm, N, Delta);
    for (uint32_t i = 0; i < N / 2; ++i) { zre[i] = z[i].real(); zim[i] = z[i].imag(); }
}

}  // extern "C"
