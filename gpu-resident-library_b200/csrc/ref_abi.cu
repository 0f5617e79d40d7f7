// The reference library's 14 extern "C" Launch* entry points, same names,
// arguments and semantics (raw device pointers, async on the given stream,
// void return), rebuilt on this library's sm_100a kernels. Each function
// names the reference declaration it replaces in include/*.h.
//
// Every modular product is exact (Shoup for constants, 128-bit product +
// Barrett otherwise), so outputs are bit-identical to the reference's
// `(unsigned __int128) % q` and Montgomery forms.
#include <cstdint>

#include "gf.cuh"
#include "hostmath.hpp"
#include "xform.cuh"
#include "convert.hpp"
#include "devonce.hpp"

namespace {

constexpr int EW_THREADS = 256;

inline unsigned ew_blocks(uint32_t n, int per_thread = 1) {
    uint64_t b = ((uint64_t)n + (uint64_t)EW_THREADS * per_thread - 1) / ((uint64_t)EW_THREADS * per_thread);
    return (unsigned)(b ? b : 1);
}

// ---------------------------------------------------------------- fallback NTT
// Sizes outside the fast engine (n < 512 or n > 65536): one global kernel per
// stage, same butterflies.
__global__ void k_ct_stage(u64* x, const u64* w, const u64* wp, uint32_t n, uint32_t m, uint32_t t, u64 q) {
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n / 2; b += gridDim.x * blockDim.x) {
        uint32_t i = b / t, off = b % t, j1 = 2 * i * t + off;
        u64 W = w[m + i], Wp = wp[m + i];
        u64 of = shoup(x[j1 + t], W, Wp, q), lo = x[j1];
        u64 hi = lo + of; if (hi >= q) hi -= q;
        u64 lv = lo; if (lv < of) lv += q; lv -= of;
        x[j1] = hi; x[j1 + t] = lv;
    }
}
__global__ void k_gs_stage(u64* x, const u64* w, const u64* wp, uint32_t n, uint32_t m, uint32_t t, u64 q) {
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n / 2; b += gridDim.x * blockDim.x) {
        uint32_t i = b / t, off = b % t, j1 = 2 * i * t + off;
        u64 lo = x[j1], hi = x[j1 + t];
        u64 s = lo + hi; if (s >= q) s -= q;
        u64 d = lo; if (d < hi) d += q; d -= hi;
        x[j1] = s; x[j1 + t] = shoup(d, w[m + i], wp[m + i], q);
    }
}
__global__ void k_scale(u64* x, uint32_t n, u64 c, u64 cp, u64 q) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = shoup(x[i], c, cp, q);
}

// ---------------------------------------------------------------- elementwise
__global__ void k_rns_mult(const u64* __restrict__ a, const u64* __restrict__ b, u64* __restrict__ r,
                           ModC m, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = mulmod(a[i], b[i], m);
}

__global__ void k_switch_modulus(u64* __restrict__ v, u64 half, u64 diff, int larger, ModC mnew, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u64 x = v[i];
    u64 d = x > half ? diff : 0;
    if (larger) { v[i] = x + d; return; }
    u64 xm = reduce64(x, mnew);
    v[i] = xm >= d ? xm - d : xm + mnew.q - d;
}

__global__ void k_rescale_fuse(u64* __restrict__ a, const u64* __restrict__ b, u64 s1, u64 s1p, u64 s2,
                               u64 s2p, u64 q, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u64 t = shoup(a[i], s1, s1p, q) + shoup(b[i], s2, s2p, q);
    a[i] = csub(t, q);
}

__global__ void k_ks_macc(u64* __restrict__ out0, u64* __restrict__ out1, const u64* __restrict__ d,
                          const u64* __restrict__ b, const u64* __restrict__ a, ModC m, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u64 dv = d[i];
    out0[i] = csub(out0[i] + mulmod(dv, b[i], m), m.q);
    out1[i] = csub(out1[i] + mulmod(dv, a[i], m), m.q);
}

__global__ void k_ks_macc_batched(u64* __restrict__ out0, u64* __restrict__ out1,
                                  const u64* const* __restrict__ digits, const u64* __restrict__ bv,
                                  const u64* __restrict__ av, const uint32_t* __restrict__ keyRow,
                                  const u64* __restrict__ mods, uint32_t n) {
    const uint32_t t = blockIdx.y;
    ModC m;
    m.q = mods[t];
    m.two_q = 2 * m.q;
    barrett_mu_device(m.q, m.mu_lo, m.mu_hi);
    const u64* dg = digits[t];
    const size_t o = (size_t)t * n, kb = (size_t)keyRow[t] * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        u64 dv = dg[k];
        out0[o + k] = csub(out0[o + k] + mulmod(dv, bv[kb + k], m), m.q);
        out1[o + k] = csub(out1[o + k] + mulmod(dv, av[kb + k], m), m.q);
    }
}

__global__ void k_moddown_combine(u64* __restrict__ ans, const u64* __restrict__ a, const u64* __restrict__ b,
                                  u64 s, u64 sp, u64 q, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u64 x = a[i], y = b[i];
    u64 d = x >= y ? x - y : x + q - y;
    ans[i] = shoup(d, s, sp, q);
}

__global__ void k_tensor(const u64* __restrict__ c0a, const u64* __restrict__ c1a, const u64* __restrict__ c0b,
                         const u64* __restrict__ c1b, u64* __restrict__ t0, u64* __restrict__ t1,
                         u64* __restrict__ t2, const u64* __restrict__ mods, uint32_t n) {
    const uint32_t t = blockIdx.y;
    ModC m;
    m.q = mods[t];
    m.two_q = 2 * m.q;
    barrett_mu_device(m.q, m.mu_lo, m.mu_hi);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        size_t x = (size_t)t * n + k;
        u64 a0 = c0a[x], a1 = c1a[x], b0 = c0b[x], b1 = c1b[x];
        t0[x] = mulmod(a0, b0, m);
        u64 lo, hi;
        mul_wide(a0, b1, lo, hi);
        mac_wide(lo, hi, a1, b0);
        t1[x] = barrett(lo, hi, m);
        t2[x] = mulmod(a1, b1, m);
    }
}

__global__ void k_combine(u64* __restrict__ r0, u64* __restrict__ r1, const u64* __restrict__ t0,
                          const u64* __restrict__ t1, const u64* __restrict__ ba0, const u64* __restrict__ ba1,
                          const u64* __restrict__ mods, uint32_t n) {
    const uint32_t t = blockIdx.y;
    const u64 q = mods[t];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        size_t x = (size_t)t * n + k;
        r0[x] = csub(t0[x] + ba0[x], q);
        r1[x] = csub(t1[x] + ba1[x], q);
    }
}

// out[i] = +-in[j] with j*k = i (mod 2n) or i+n (mod 2n): gather form of the
// reference's scatter (every output index written once, coalesced stores).
__global__ void k_automorph(u64* __restrict__ out, const u64* __restrict__ in, uint32_t n, uint64_t kinv, u64 q) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t M = 2ull * n;
    uint64_t j = ((uint64_t)i * kinv) % M;
    if (j < n) out[i] = in[j];
    else { u64 v = in[j - n]; out[i] = v ? q - v : 0; }
}

__global__ void k_automorph_scatter(u64* __restrict__ out, const u64* __restrict__ in, uint32_t n, uint64_t k,
                                    u64 q) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint64_t M = 2ull * n;
    uint64_t idx = ((uint64_t)j * k) % M;
    u64 v = in[j];
    if (idx < n) out[idx] = v; else out[idx - n] = v ? q - v : 0;
}

__global__ void k_add_into(u64* __restrict__ a, const u64* __restrict__ b, u64 q, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = csub(a[i] + b[i], q);
}

__global__ void k_ptmulacc(u64* __restrict__ acc0, u64* __restrict__ acc1, const u64* __restrict__ b0,
                           const u64* __restrict__ b1, const u64* __restrict__ d, ModC m, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u64 dv = d[i];
    acc0[i] = csub(acc0[i] + mulmod(b0[i], dv, m), m.q);
    acc1[i] = csub(acc1[i] + mulmod(b1[i], dv, m), m.q);
}

// ApproxSwitchCRTBasis: x_i = a_i * QHatInv_i (Shoup) staged in shared memory
// per coefficient, then sum_i x_i * QHatModp[i][j] (128-bit) and Barrett.
__global__ void k_approx_switch(const u64* __restrict__ src, u64* __restrict__ dst, const u64* __restrict__ qhi,
                                const u64* __restrict__ qhip, const u64* __restrict__ qm,
                                const u64* __restrict__ qmp, const u64* __restrict__ p,
                                const u64* __restrict__ mulo, const u64* __restrict__ muhi,
                                uint32_t sizeQ, uint32_t sizeP, uint32_t n) {
    extern __shared__ u64 xs[];   // [sizeQ][blockDim]
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = k < n;
    for (uint32_t i = 0; i < sizeQ; ++i)
        xs[i * blockDim.x + threadIdx.x] = on ? shoup(src[(size_t)i * n + k], qhi[i], qhip[i], qm[i]) : 0;
    if (!on) return;
    for (uint32_t j = 0; j < sizeP; ++j) {
        u64 lo = 0, hi = 0;
        for (uint32_t i = 0; i < sizeQ; ++i) mac_wide(lo, hi, xs[i * blockDim.x + threadIdx.x], qmp[(size_t)i * sizeP + j]);
        ModC m;
        m.q = p[j]; m.two_q = 2 * m.q; m.mu_lo = mulo[j]; m.mu_hi = muhi[j];
        dst[(size_t)j * n + k] = barrett(lo, hi, m);
    }
}

void fallback_ntt(u64* x, const u64* w, const u64* wp, uint32_t n, u64 q, bool inv, u64 ninv, u64 ninvp,
                  cudaStream_t s) {
    const unsigned blocks = ew_blocks(n / 2 ? n / 2 : 1);
    if (!inv) {
        for (uint32_t m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1)
            k_ct_stage<<<blocks, EW_THREADS, 0, s>>>(x, w, wp, n, m, t, q);
    } else {
        for (uint32_t m = n >> 1, t = 1; m >= 1; m >>= 1, t <<= 1) {
            k_gs_stage<<<blocks, EW_THREADS, 0, s>>>(x, w, wp, n, m, t, q);
            if (m == 1) break;
        }
        k_scale<<<ew_blocks(n), EW_THREADS, 0, s>>>(x, n, ninv, ninvp, q);
    }
}

}  // namespace

namespace cv {

cudaError_t approx_switch_integer(const uint64_t* d_src, uint64_t* d_dst, const uint64_t* d_QHatInvModq,
                                  const uint64_t* d_QHatInvModqPrecon, const uint64_t* d_q, const uint64_t* d_QHatModp,
                                  const uint64_t* d_p, const uint64_t* d_mu_lo, const uint64_t* d_mu_hi, uint32_t sizeQ,
                                  uint32_t sizeP, uint32_t n, cudaStream_t s) {
    int threads = 128;
    size_t smem = (size_t)sizeQ * threads * 8;
    // the limit only caps what a launch may ask for: raise it once per device
    // to the opt-in maximum, so concurrent callers with different sizeQ never
    // lower it under one another
    static gfx::DeviceOnce attrs;
    attrs([] {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && optin > 0)
            cudaFuncSetAttribute(k_approx_switch, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    });
    unsigned blocks = (unsigned)(((uint64_t)n + threads - 1) / threads);
    k_approx_switch<<<blocks, threads, smem, s>>>(d_src, d_dst, d_QHatInvModq, d_QHatInvModqPrecon, d_q, d_QHatModp,
                                                  d_p, d_mu_lo, d_mu_hi, sizeQ, sizeP, n);
    return cudaGetLastError();
}

}  // namespace cv

extern "C" {

// include/ntt.h — reference ntt.h:8-10
void LaunchNTT_CT(uint64_t* d_x, const uint64_t* d_roots, const uint64_t* d_precon, uint32_t n, uint64_t q,
                  cudaStream_t s) {
    const int logn = hm::ilog2(n);
    if (hm::is_pow2(n) && xf_supported_logn(logn)) {
        xf::Job j{d_x, nullptr, d_roots, d_precon, q, 0, 0, nullptr, fp_tower(q) ? 1u : 0u, 0};
        xf_launch_ntt(nullptr, &j, 1, logn, false, s);
    } else if (n >= 2) {
        fallback_ntt(d_x, d_roots, d_precon, n, q, false, 0, 0, s);
    }
}

// include/intt.h — reference intt.h:7-10
void LaunchINTT_GS(uint64_t* d_x, const uint64_t* d_invroots, const uint64_t* d_invprecon, uint32_t n, uint64_t q,
                   uint64_t n_inv, uint64_t n_inv_precon, cudaStream_t s) {
    const int logn = hm::ilog2(n);
    if (hm::is_pow2(n) && xf_supported_logn(logn)) {
        xf::Job j{d_x, nullptr, d_invroots, d_invprecon, q, n_inv, n_inv_precon, nullptr, fp_tower(q) ? 1u : 0u, 0};
        xf_launch_ntt(nullptr, &j, 1, logn, true, s);
    } else if (n >= 2) {
        fallback_ntt(d_x, d_invroots, d_invprecon, n, q, true, n_inv, n_inv_precon, s);
    }
}

// include/rns_arith.h — reference rns_arith.h:7-9
void LaunchRNSMultTower(const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_r, uint64_t q, uint32_t n,
                        cudaStream_t stream) {
    k_rns_mult<<<ew_blocks(n), EW_THREADS, 0, stream>>>(d_a, d_b, d_r, hm::modc(q), n);
}

// include/switch_modulus.h — reference switch_modulus.h:7-8
void LaunchSwitchModulus(uint64_t* d_v, uint64_t q_old, uint64_t q_new, uint32_t n, cudaStream_t s) {
    const u64 half = q_old >> 1;
    const int larger = q_new > q_old;
    u64 diff = larger ? q_new - q_old : q_old - q_new;
    if (!larger) diff %= q_new;
    k_switch_modulus<<<ew_blocks(n), EW_THREADS, 0, s>>>(d_v, half, diff, larger, hm::modc(q_new), n);
}

// include/rescale.h — reference rescale.h:9-11
void LaunchRescaleFuse(uint64_t* d_a, const uint64_t* d_b, uint64_t s1, uint64_t s2, uint64_t q, uint32_t n,
                       cudaStream_t s) {
    s1 %= q; s2 %= q;
    k_rescale_fuse<<<ew_blocks(n), EW_THREADS, 0, s>>>(d_a, d_b, s1, hm::precon(s1, q), s2, hm::precon(s2, q), q, n);
}

// include/basis_convert.h — reference basis_convert.h:9-14. The tensor-core
// form (byte limbs on tcgen05, bit-identical) where its shape limits allow it:
// it measured 1.2-1.9x faster than the integer form at 3..8 source towers.
void LaunchApproxSwitchCRTBasis(const uint64_t* d_src, uint64_t* d_dst, const uint64_t* d_QHatInvModq,
                                const uint64_t* d_QHatInvModqPrecon, const uint64_t* d_q,
                                const uint64_t* d_QHatModp, const uint64_t* d_p, const uint64_t* d_mu_lo,
                                const uint64_t* d_mu_hi, uint32_t sizeQ, uint32_t sizeP, uint32_t n,
                                cudaStream_t s) {
    if (cv::tcgen05_shape(sizeQ, sizeP, n))
        cv::approx_switch_tcgen05(d_src, d_dst, d_QHatInvModq, d_QHatInvModqPrecon, d_q, d_QHatModp, d_p, d_mu_lo,
                                  d_mu_hi, sizeQ, sizeP, n, s);
    else
        cv::approx_switch_integer(d_src, d_dst, d_QHatInvModq, d_QHatInvModqPrecon, d_q, d_QHatModp, d_p, d_mu_lo,
                                  d_mu_hi, sizeQ, sizeP, n, s);
}

// include/ks_fastcore.h — reference ks_fastcore.h:9-12
void LaunchKSMultAcc(uint64_t* d_out0, uint64_t* d_out1, const uint64_t* d_digit, const uint64_t* d_b,
                     const uint64_t* d_a, uint64_t q, uint32_t n, cudaStream_t s) {
    k_ks_macc<<<ew_blocks(n), EW_THREADS, 0, s>>>(d_out0, d_out1, d_digit, d_b, d_a, hm::modc(q), n);
}

// include/ks_fastcore.h — reference ks_fastcore.h:13-18
void LaunchKSMultAccBatched(uint64_t* d_out0, uint64_t* d_out1, const uint64_t* const* d_digits,
                            const uint64_t* d_bv, const uint64_t* d_av, const uint32_t* d_keyRow,
                            const uint64_t* d_mods, uint32_t towers, uint32_t n, cudaStream_t s) {
    if (!towers) return;
    dim3 g(ew_blocks(n, 4), towers);
    k_ks_macc_batched<<<g, EW_THREADS, 0, s>>>(d_out0, d_out1, d_digits, d_bv, d_av, d_keyRow, d_mods, n);
}

// include/moddown.h — reference moddown.h:7-9
void LaunchModDownCombine(uint64_t* d_ans, const uint64_t* d_a, const uint64_t* d_b, uint64_t sc, uint64_t q,
                          uint32_t n, cudaStream_t st) {
    sc %= q;
    k_moddown_combine<<<ew_blocks(n), EW_THREADS, 0, st>>>(d_ans, d_a, d_b, sc, hm::precon(sc, q), q, n);
}

// include/tensor.h — reference kernels/tensor.cu:28-36 (headerless there)
void LaunchTensor(const uint64_t* c0a, const uint64_t* c1a, const uint64_t* c0b, const uint64_t* c1b,
                  uint64_t* t0, uint64_t* t1, uint64_t* t2, const uint64_t* d_mods, uint32_t sizeQ, uint32_t n,
                  cudaStream_t s) {
    if (!sizeQ) return;
    dim3 g(ew_blocks(n, 4), sizeQ);
    k_tensor<<<g, EW_THREADS, 0, s>>>(c0a, c1a, c0b, c1b, t0, t1, t2, d_mods, n);
}

// include/tensor.h — reference kernels/tensor.cu:53-61 (headerless there)
void LaunchCombine(uint64_t* r0, uint64_t* r1, const uint64_t* t0, const uint64_t* t1, const uint64_t* ba0,
                   const uint64_t* ba1, const uint64_t* d_mods, uint32_t sizeQ, uint32_t n, cudaStream_t s) {
    if (!sizeQ) return;
    dim3 g(ew_blocks(n, 4), sizeQ);
    k_combine<<<g, EW_THREADS, 0, s>>>(r0, r1, t0, t1, ba0, ba1, d_mods, n);
}

// include/automorph.h — reference automorph.h:4-6
void LaunchAutomorphPermute(uint64_t* d_out, const uint64_t* d_in, uint32_t n, uint64_t k, uint64_t q,
                            cudaStream_t s) {
    const uint64_t M = 2ull * n;
    // k^-1 mod 2n by extended Euclid; a k sharing a factor with 2n has no
    // inverse and takes the reference's scatter form instead.
    long long r0 = (long long)M, r1 = (long long)(k % M), t0 = 0, t1 = 1;
    while (r1) {
        long long qq = r0 / r1, tmp;
        tmp = r0 - qq * r1; r0 = r1; r1 = tmp;
        tmp = t0 - qq * t1; t0 = t1; t1 = tmp;
    }
    if (r0 != 1) {
        k_automorph_scatter<<<ew_blocks(n), EW_THREADS, 0, s>>>(d_out, d_in, n, k, q);
        return;
    }
    const uint64_t inv = (uint64_t)((t0 % (long long)M + (long long)M) % (long long)M);
    k_automorph<<<ew_blocks(n), EW_THREADS, 0, s>>>(d_out, d_in, n, inv, q);
}

// include/stage_acc.h — reference stage_acc.h:4-7
void LaunchPtMulAcc(uint64_t* d_acc0, uint64_t* d_acc1, const uint64_t* d_b0, const uint64_t* d_b1,
                    const uint64_t* d_d, uint64_t q, uint32_t n, cudaStream_t s) {
    k_ptmulacc<<<ew_blocks(n), EW_THREADS, 0, s>>>(d_acc0, d_acc1, d_b0, d_b1, d_d, hm::modc(q), n);
}

// include/stage_acc.h — reference stage_acc.h:8-9
void LaunchAddInto(uint64_t* d_a, const uint64_t* d_b, uint64_t q, uint32_t n, cudaStream_t s) {
    k_add_into<<<ew_blocks(n), EW_THREADS, 0, s>>>(d_a, d_b, q, n);
}

}  // extern "C"
