// Host-side exact modular helpers (setup only; never on a timed path).
#pragma once
#include <cstring>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "gf.cuh"

namespace hm {
typedef unsigned __int128 u128;

inline u64 mulmod(u64 a, u64 b, u64 q) { return (u64)(((u128)a * b) % q); }
inline u64 powmod(u64 b, u64 e, u64 q) {
    u128 r = 1, bb = b % q;
    while (e) { if (e & 1) r = (r * bb) % q; bb = (bb * bb) % q; e >>= 1; }
    return (u64)r;
}
inline u64 invmod(u64 a, u64 q) { return powmod(a % q, q - 2, q); }   // q prime
inline u64 precon(u64 w, u64 q) { return (u64)(((u128)w << 64) / q); }
inline uint32_t bitrev(uint32_t v, uint32_t bits) {
    uint32_t r = 0;
    for (uint32_t k = 0; k < bits; ++k) { r = (r << 1) | (v & 1); v >>= 1; }
    return r;
}
inline int ilog2(uint32_t n) { int l = 0; while ((1u << l) < n) ++l; return l; }
inline bool is_pow2(uint32_t n) { return n && !(n & (n - 1)); }

inline ModC modc(u64 q) {
    ModC m;
    m.q = q;
    m.two_q = 2 * q;
    u128 mu = (~(u128)0) / q;
    m.mu_lo = (u64)mu;
    m.mu_hi = (u64)(mu >> 64);
    m.r64 = (~0ull) / q;
    const double qinv = 1.0 / (double)q;   // RN(1/q), the FP64 NTT path's quotient scale
    std::memcpy(&m.qinv_bits, &qinv, 8);
    u64 inv = q;                            // q^-1 mod 2^64 by Newton (q odd): 3 -> 6 -> ... -> 96 bits
    for (int i = 0; i < 5; ++i) inv *= 2 - q * inv;
    m.qneg = 0 - inv;
    m.pad_ = 0;
    return m;
}

// Product of mods (skipping index `skip`) reduced mod q.
inline u64 prod_mod(const u64* mods, uint32_t cnt, u64 q, int skip = -1) {
    u64 r = 1 % q;
    for (uint32_t k = 0; k < cnt; ++k) if ((int)k != skip) r = mulmod(r, mods[k] % q, q);
    return r;
}

// Packed twiddle tables: fwd[i] = {psi^bitrev(i), precon}, inv from psi^-1.
inline void twiddles(uint32_t n, u64 q, u64 psi, std::vector<Tw>& fwd, std::vector<Tw>& inv) {
    const uint32_t logn = (uint32_t)ilog2(n);
    std::vector<u64> pw(n);
    auto fill = [&](u64 base, std::vector<Tw>& out) {
        out.resize(n);
        pw[0] = 1;
        for (uint32_t i = 1; i < n; ++i) pw[i] = mulmod(pw[i - 1], base, q);
        for (uint32_t i = 0; i < n; ++i) {
            u64 w = pw[bitrev(i, logn)];
            out[i] = Tw{w, precon(w, q)};
        }
    };
    fill(psi, fwd);
    fill(invmod(psi, q), inv);
}
}  // namespace hm
