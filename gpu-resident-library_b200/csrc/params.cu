// Native parameter generation (the reference's params.cpp:29-75 contract):
// NTT-friendly primes q = 1 mod 2n descending from 2^bits, the
// smallest-generator primitive 2n-th root, and the rescale constant pair.
// Exposed as the reference's C++ functions (namespace gpufhe, include/params.h)
// and as C entry points for non-C++ callers (include/gpufhe_b200.h).
#include <cstring>
#include <string>
#include <stdexcept>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "hostmath.hpp"
#include "params.h"

namespace {

bool is_prime(uint64_t x) {
    if (x < 2) return false;
    static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t a : bases) if (x % a == 0) return x == a;
    uint64_t d = x - 1;
    int s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    for (uint64_t a : bases) {   // deterministic for all 64-bit inputs
        uint64_t v = hm::powmod(a, d, x);
        if (v == 1 || v == x - 1) continue;
        bool composite = true;
        for (int i = 1; i < s && composite; ++i) {
            v = hm::mulmod(v, v, x);
            if (v == x - 1) composite = false;
        }
        if (composite) return false;
    }
    return true;
}

}  // namespace

namespace gpufhe {

void native_primes(std::vector<uint64_t>& out, uint32_t count, uint32_t bits, uint32_t n,
                   const std::vector<uint64_t>& avoid) {
    if (bits < 2 || bits > 62 || n == 0) throw std::invalid_argument("native_primes: bad bits or n");
    const uint64_t M = 2ull * n;
    uint64_t q = ((1ull << bits) / M) * M + 1;
    while (out.size() < count) {
        if (q < (1ull << (bits - 1)))
            throw std::runtime_error("native_primes: fewer than the requested count of " + std::to_string(bits) +
                                     "-bit primes q = 1 mod 2n outside the avoid list");
        bool skip = false;
        for (uint64_t a : avoid) if (a == q) skip = true;
        if (!skip && is_prime(q)) out.push_back(q);
        q -= M;
    }
}

uint64_t native_root(uint32_t n, uint64_t q) {
    const uint64_t M = 2ull * n;
    if (n == 0 || q < 3 || (q - 1) % M != 0)
        throw std::runtime_error("native_root: q - 1 is not a multiple of 2n, so q has no primitive 2n-th root");
    for (uint64_t g = 2; g < q; ++g) {
        uint64_t c = hm::powmod(g, (q - 1) / M, q);
        if (hm::powmod(c, n, q) == q - 1) return c;
    }
    throw std::runtime_error("native_root: no element of order 2n below q (q is not prime)");
}

// Rescale constants for dropping tower `last` of mod[0..last]. With
// Q_l = mod[0] * ... * mod[last-1], q_l = mod[last] and u = Q_l^-1 mod q_l,
// the reference defines s1[i] = q_l^-1 mod q_i and
// s2[i] = floor(Q_l * u / q_l) mod q_i. Because Q_l * u = 1 (mod q_l), the
// division is exact after subtracting one: floor(Q_l * u / q_l) =
// (Q_l * u - 1) / q_l. Every q_i with i < last divides Q_l, so modulo q_i the
// numerator is -1 and s2[i] = -q_l^-1 = q_i - s1[i]. The rescale
// a * s1 + b * s2 is then (a - b) * q_l^-1, as it must be.
void native_rescale_consts(std::vector<uint64_t>& s1, std::vector<uint64_t>& s2, const std::vector<uint64_t>& mod,
                           uint32_t last) {
    if (last >= mod.size()) throw std::invalid_argument("native_rescale_consts: tower index beyond the modulus list");
    const uint64_t ql = mod[last];
    s1.resize(last);
    s2.resize(last);
    for (uint32_t i = 0; i < last; ++i) {
        const uint64_t qi = mod[i];
        if (ql % qi == 0) throw std::invalid_argument("native_rescale_consts: moduli are not coprime");
        s1[i] = hm::invmod(ql % qi, qi);
        s2[i] = qi - s1[i];
    }
}

}  // namespace gpufhe

extern "C" {

int gpufhe_native_primes(uint64_t* out, uint32_t count, uint32_t bits, uint32_t n, const uint64_t* avoid,
                         uint32_t navoid) {
    if (!out) return GPUFHE_EINVAL;
    try {
        std::vector<uint64_t> o, av(avoid, avoid + (avoid ? navoid : 0));
        gpufhe::native_primes(o, count, bits, n, av);
        std::memcpy(out, o.data(), o.size() * 8);
        return GPUFHE_OK;
    } catch (const std::exception& e) {
        gfx::set_error(e.what());
        return GPUFHE_EINVAL;
    }
}

uint64_t gpufhe_native_root(uint32_t n, uint64_t q) {
    try { return gpufhe::native_root(n, q); } catch (...) { return 0; }
}

int gpufhe_rescale_consts(uint64_t* s1, uint64_t* s2, const uint64_t* mod, uint32_t last) {
    if (!s1 || !s2 || !mod) return GPUFHE_EINVAL;
    std::vector<uint64_t> a, b, m(mod, mod + last + 1);
    try {
        gpufhe::native_rescale_consts(a, b, m, last);
    } catch (const std::exception& e) {
        gfx::set_error(e.what());
        return GPUFHE_EINVAL;
    }
    std::memcpy(s1, a.data(), last * 8);
    std::memcpy(s2, b.data(), last * 8);
    return GPUFHE_OK;
}

}  // extern "C"
