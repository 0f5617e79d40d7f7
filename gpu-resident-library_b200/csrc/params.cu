// Native parameter generation (the reference's params.cpp:29-75 contract):
// NTT-friendly primes q = 1 mod 2n descending from 2^bits, the
// smallest-generator primitive 2n-th root, and the rescale constant pair.
// Exposed as the reference's C++ functions (namespace gpufhe, include/params.h)
// and as C entry points for non-C++ callers (include/gpufhe_b200.h).
#include <cstring>
#include <stdexcept>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "hostmath.hpp"
#include "params.h"

namespace {
using hm::u128;

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

u128 mulmod128(u128 a, u128 b, u128 m) {
    a %= m;
    u128 r = 0;
    while (b) {
        if (b & 1) { r += a; if (r >= m) r -= m; }
        a <<= 1; if (a >= m) a -= m;
        b >>= 1;
    }
    return r;
}
}  // namespace

namespace gpufhe {

void native_primes(std::vector<uint64_t>& out, uint32_t count, uint32_t bits, uint32_t n,
                   const std::vector<uint64_t>& avoid) {
    if (bits < 2 || bits > 62 || n == 0) throw std::invalid_argument("native_primes: bad bits or n");
    const uint64_t M = 2ull * n;
    uint64_t q = ((1ull << bits) / M) * M + 1;
    while (out.size() < count) {
        if (q < (1ull << (bits - 1))) throw std::runtime_error("prime search exhausted");
        bool skip = false;
        for (uint64_t a : avoid) if (a == q) skip = true;
        if (!skip && is_prime(q)) out.push_back(q);
        q -= M;
    }
}

uint64_t native_root(uint32_t n, uint64_t q) {
    const uint64_t M = 2ull * n;
    for (uint64_t g = 2; g < q; ++g) {
        uint64_t c = hm::powmod(g, (q - 1) / M, q);
        if (hm::powmod(c, n, q) == q - 1) return c;
    }
    throw std::runtime_error("no 2n-th root");
}

void native_rescale_consts(std::vector<uint64_t>& s1, std::vector<uint64_t>& s2, const std::vector<uint64_t>& mod,
                           uint32_t last) {
    const uint64_t ql = mod[last];
    s1.resize(last);
    s2.resize(last);
    uint64_t QlModql = 1 % ql;
    for (uint32_t t = 0; t < last; ++t) QlModql = hm::mulmod(QlModql, mod[t] % ql, ql);
    const uint64_t u = hm::invmod(QlModql, ql);
    for (uint32_t i = 0; i < last; ++i) {
        const uint64_t qi = mod[i];
        s1[i] = hm::invmod(ql % qi, qi);
        u128 m2 = (u128)ql * qi, Ql2 = 1 % m2;
        for (uint32_t t = 0; t < last; ++t) Ql2 = mulmod128(Ql2, mod[t], m2);
        u128 prod = mulmod128(Ql2, u, m2);
        u128 pm1 = prod == 0 ? m2 - 1 : prod - 1;
        s2[i] = (uint64_t)((pm1 / ql) % qi);
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
    gpufhe::native_rescale_consts(a, b, m, last);
    std::memcpy(s1, a.data(), last * 8);
    std::memcpy(s2, b.data(), last * 8);
    return GPUFHE_OK;
}

}  // extern "C"
