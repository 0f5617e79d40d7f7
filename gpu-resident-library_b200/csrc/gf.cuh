// Exact 64-bit modular arithmetic for RNS-CKKS on sm_100a.
//
// Moduli are odd primes q < 2^61. Values move through the transforms in
// "lazy" ranges ([0,2q) or [0,4q)) and are brought to the canonical range
// [0,q) wherever a result leaves a kernel, so every output is bit-identical
// to a fully reduced scalar computation of the same formula.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

typedef uint64_t u64;
typedef uint32_t u32;

// Twiddle with its Shoup precomputation floor(w * 2^64 / q).
struct __align__(16) Tw { u64 w, wp; };

// Per-modulus constants used by the kernels.
struct __align__(16) ModC {
    u64 q, two_q;
    u64 mu_lo, mu_hi;   // floor(2^128 / q)
    u64 r64;            // floor(2^64 / q)
    u64 qinv_bits;      // bits of the double RN(1/q) (FP64 NTT path)
    u64 qneg;           // -q^-1 mod 2^64 (Montgomery reduction)
    u64 pad_;
};

// Montgomery reduction: T = hi*2^64 + lo < q*2^64 -> T * 2^-64 mod q in [0, q).
// m = lo * (-q^-1) makes T + m*q divisible by 2^64; its low word sums to 0 or
// 2^64, carrying 1 exactly when lo != 0.
__device__ __forceinline__ u64 redc_lazy(u64 lo, u64 hi, const ModC& m) {   // result in [0, 2q)
    const u64 mm = lo * m.qneg;
    return hi + __umul64hi(mm, m.q) + (lo != 0 ? 1ull : 0ull);
}
__device__ __forceinline__ u64 redc(u64 lo, u64 hi, const ModC& m) {
    const u64 t = redc_lazy(lo, hi, m);
    return t >= m.q ? t - m.q : t;
}
// 2^64 mod q from r64 = floor(2^64 / q): 2^64 - q * r64, computed mod 2^64.
__device__ __forceinline__ u64 r_mod(const ModC& m) { return 0ull - m.q * m.r64; }

// Towers whose transforms may take the FP64 path (4q < 2^52).
__host__ __device__ __forceinline__ bool fp_tower(u64 q) { return q < (1ull << 50); }
__device__ __forceinline__ double qinv_of(const ModC& m) { return __longlong_as_double((long long)m.qinv_bits); }

__device__ __forceinline__ u64 csub(u64 a, u64 m) { return a >= m ? a - m : a; }

// a * w mod q in [0, 2q) for any a < 2^64 (Shoup, w < q).
__device__ __forceinline__ u64 shoup_lazy(u64 a, u64 w, u64 wp, u64 q) {
    return a * w - __umul64hi(a, wp) * q;
}
__device__ __forceinline__ u64 shoup(u64 a, u64 w, u64 wp, u64 q) {
    return csub(shoup_lazy(a, w, wp, q), q);
}

// 128-bit helpers (lo, hi).
__device__ __forceinline__ void mul_wide(u64 a, u64 b, u64& lo, u64& hi) {
    lo = a * b;
    hi = __umul64hi(a, b);
}
__device__ __forceinline__ void add_wide(u64& lo, u64& hi, u64 blo, u64 bhi) {
    asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;"
        : "+l"(lo), "+l"(hi) : "l"(blo), "l"(bhi));
}
__device__ __forceinline__ void mac_wide(u64& lo, u64& hi, u64 a, u64 b) {
    u64 plo, phi;
    mul_wide(a, b, plo, phi);
    add_wide(lo, hi, plo, phi);
}

// Barrett reduction of S = hi*2^64 + lo (S < 2^127) with mu = floor(2^128/q).
// The quotient estimate drops three fractional terms, so it is short by at
// most 3 and S - qhat*q lies in [0, 4q); that difference fits in 64 bits for
// q < 2^62, so it is computed mod 2^64. Lazy result in [0, 4q).
__device__ __forceinline__ u64 barrett_lazy(u64 lo, u64 hi, u64 q, u64 mu_lo, u64 mu_hi) {
    u64 qh = hi * mu_hi + __umul64hi(hi, mu_lo) + __umul64hi(lo, mu_hi);
    return lo - qh * q;
}
__device__ __forceinline__ u64 barrett(u64 lo, u64 hi, const ModC& m) {
    u64 r = barrett_lazy(lo, hi, m.q, m.mu_lo, m.mu_hi);
    r = csub(r, m.two_q);
    return csub(r, m.q);
}
__device__ __forceinline__ u64 mulmod(u64 a, u64 b, const ModC& m) {
    u64 lo, hi;
    mul_wide(a, b, lo, hi);
    return barrett(lo, hi, m);
}
// x mod q for any 64-bit x, using r64 = floor(2^64/q).
__device__ __forceinline__ u64 reduce64(u64 x, const ModC& m) {
    u64 r = x - __umul64hi(x, m.r64) * m.q;   // [0, 2q)
    return csub(r, m.q);
}

// Harvey forward (Cooley-Tukey) butterfly: x, y in [0,4q) -> [0,4q).
__device__ __forceinline__ void ct_bfly(u64& x, u64& y, u64 w, u64 wp, u64 q, u64 two_q) {
    u64 xx = csub(x, two_q);
    u64 t = shoup_lazy(y, w, wp, q);
    x = xx + t;
    y = xx - t + two_q;
}
// Inverse (Gentleman-Sande) butterfly: x, y in [0,2q) -> [0,2q).
__device__ __forceinline__ void gs_bfly(u64& x, u64& y, u64 w, u64 wp, u64 q, u64 two_q) {
    u64 s = csub(x + y, two_q);
    u64 d = x - y + two_q;
    x = s;
    y = shoup_lazy(d, w, wp, q);
}

// floor(2^128 / q) computed on the device for kernels that only receive a
// device array of moduli (reference ABI). q odd, 2^20 < q < 2^62.
__device__ __forceinline__ void barrett_mu_device(u64 q, u64& mu_lo, u64& mu_hi) {
    mu_hi = (~0ull) / q;                       // floor(2^64 / q) for odd q
    u64 rem = 0ull - mu_hi * q;                // 2^64 - mu_hi*q, in (0, q)
    // mu_lo = floor(rem * 2^64 / q): double estimate, then exact correction.
    double est = ((double)rem / (double)q) * 18446744073709551616.0;
    u64 e = est >= 18446744073709551615.0 ? ~0ull : (u64)est;
    for (int it = 0; it < 3; ++it) {
        // r = rem*2^64 - e*q as a signed 128-bit value (hi, lo)
        u64 plo, phi;
        mul_wide(e, q, plo, phi);
        u64 rlo = 0ull - plo;
        u64 rhi = rem - phi - (plo != 0 ? 1ull : 0ull);
        long long shi = (long long)rhi;
        double rd = (double)shi * 18446744073709551616.0 + (double)rlo;
        double corr = rd / (double)q;
        if (corr > -1.0 && corr < 2.0) break;
        e += (long long)corr;
    }
    for (int it = 0; it < 64; ++it) {
        u64 plo, phi;
        mul_wide(e, q, plo, phi);
        u64 rlo = 0ull - plo;
        u64 rhi = rem - phi - (plo != 0 ? 1ull : 0ull);
        if ((long long)rhi < 0) { --e; continue; }
        if (rhi == 0 && rlo < q) break;
        ++e;
    }
    mu_lo = e;
}
