// Batched resident CKKS pipeline kernels: EvalMult+Rescale, Hybrid keyswitch,
// rotation and rescale for many independent ciphertexts of uneven level, one
// launch per phase for the whole batch.
//
// Reference algorithm (keyswitch_resident.cpp:139-244, tensor.cu, rescale.cu,
// rotate.cpp:118-132), restated with NTT linearity to fuse stages:
//   d2     = a1*b1                                     (tensor, eval)
//   x_i    = INTT(d2_i) * n^-1 * QHatInv_i              (ModUp input, coeff)
//   conv_j = sum_s x_s * QHatModp[s][j] mod m_j         (ApproxSwitchCRTBasis)
//   res_i  = sum_p digit_p[i] * key_p[row(i)]           (digit = NTT(conv) or d2_i)
//   ModDown + combine + rescale of tower l = L-1, for i < l:
//   out_i  = t_i*s1 + res_i*P^-1*s1 + NTT( sw_i(r_l)*s2 - conv'_i*P^-1*s1 )
//   r_l    = INTT(t_l + res_l*P^-1) - conv'_l*P^-1     (coeff, canonical)
// where conv' is the P->Q conversion of INTT(res_P)*n^-1*PHatInv and sw_i is
// SwitchModulus(q_l -> q_i). Every step is an exact residue computation, so
// each output equals the reference's bit for bit.
//
// Kernels (one launch each over all jobs of the batch; jobs are (pair, sub)):
//   K1 inv-row  (pair,i)        tensor / gather prologue, INTT row stages  -> X
//   K2 inv-col  (pair,i)        INTT column stages, * n^-1 QHatInv         -> X
//   K3 fwd-col  (pair,p,i)      ModUp conversion prologue, NTT columns     -> Y
//   K4 fwd-row  (pair,i<L+K)    NTT rows per digit + key MAC, epilogue     -> W / U / RP
//   K5 inv-col  (pair,c,t<=K)   INTT columns of U and RP, scaled           -> U / RP
//   K6 fwd-col  (pair,c,i)      ModDown + SwitchModulus prologue           -> Z
//   K7 fwd-row  (pair,c,i)      NTT rows, final combine                    -> out
#pragma once
#include "context.hpp"
#include "ntt.cuh"

namespace pl {

using gfx::DevCtx;
using gfx::Level;

constexpr int MAXA = 16;   // digit width supported by the fused ModUp prologue

enum Mode : u32 {
    EMR = 0,       // EvalMult + Rescale: in = c0a,c1a,c0b,c1b [L]; out0,out1 [L-1]
    KS = 1,        // keyswitch: in[0] = a [L]; out0,out1 = ba0, ba1 [L]
    ROT = 2,       // rotation: in = c0, c1 [L]; out = sigma(c0)+ba0, ba1 [L]
    RESCALE = 3,   // rescale: in[0] = comp [L]; out0 = [L-1] (may alias in[0])
};

struct PairDesc {
    u32 L;
    u32 mode;
    u64 galois;            // ROT: Galois element k (odd, < 2n)
    const u64* in[4];
    u64* out[2];
    u64* ws;
    const u64* kav;        // key [dnum][fullQ+K][n]
    const u64* kbv;
};

// Workspace layout (tower-polys of n words) for level L.
struct WsLayout {
    u32 X, Y, W, U, RP, Z, total;
};
__host__ __device__ __forceinline__ WsLayout ws_layout(u32 L, u32 K, u32 alpha) {
    const u32 beta = (L + alpha - 1) / alpha;
    WsLayout w;
    w.X = 0;
    w.Y = w.X + L;
    w.W = w.Y + beta * (L + K);
    w.U = w.W + 2 * L;
    w.RP = w.U + 2;
    w.Z = w.RP + 2 * K;
    w.total = w.Z + 2 * L;
    return w;
}

// QP-table index of QlP position i at level L.
__host__ __device__ __forceinline__ u32 qp_of(u32 i, u32 L, u32 fullQ) { return i < L ? i : fullQ + (i - L); }

// Eval-slot permutation of the Galois automorphism X -> X^k: slot j of the
// bit-reversed NTT output holds the evaluation at psi^(2*brv(j)+1), so
// sigma_k(a)[j] = a[brv(((2*brv(j)+1)*k mod 2n - 1)/2)].
template <int LOGN>
__device__ __forceinline__ u32 galois_slot(u32 j, u64 k) {
    const u32 e = 2 * (__brev(j) >> (32 - LOGN)) + 1;
    const u32 t = (u32)(((u64)e * k) & ((2ull << LOGN) - 1));
    return __brev((t - 1) >> 1) >> (32 - LOGN);
}

template <int LOGN>
struct PG {
    using G = ntt::Geo<LOGN>;
    static constexpr int MAC_RB = ntt::cmin(G::R1, 8);          // K4 row tile rows
    static constexpr int MAC_TILE = MAC_RB * 256;
    static constexpr int MAC_THREADS = MAC_TILE / 8;            // 8 values per thread
    static constexpr int MAC_TILES = G::R1 / MAC_RB;
    static constexpr int MAC_SMEM = MAC_RB * G::ROW_STRIDE * 8;
};

// Digit source value at element e of tower i (eval form, canonical).
template <int LOGN>
__device__ __forceinline__ u64 digit_src(const PairDesc& P, u32 i, u32 e, const ModC& m) {
    const size_t o = ((size_t)i << LOGN);
    if (P.mode == EMR) return mulmod(P.in[1][o + e], P.in[3][o + e], m);
    if (P.mode == ROT) return P.in[1][o + galois_slot<LOGN>(e, P.galois)];
    return P.in[0][o + e];
}

// ------------------------------------------------------------------ K1
template <int LOGN>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS)
k1_inv_row(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const uint2 jb = jobs[blockIdx.x / G::ROW_TILES];
    const u32 R0 = (blockIdx.x % G::ROW_TILES) * G::RB;
    const PairDesc& P = pairs[jb.x];
    const u32 i = jb.y;
    const ModC m = D.mod[i];
    const WsLayout w = ws_layout(P.L, D.K, D.alpha);
    u64* X = P.ws + ((size_t)(w.X + i) << LOGN) + (size_t)R0 * 256;
    ntt::row_tile_walk<G::RB, G::ROW_THREADS>([&](int rl, int c) {
        sm[rl * G::ROW_STRIDE + ntt::rowpad(c)] = digit_src<LOGN>(P, i, (R0 + rl) * 256 + c, m);
    });
    __syncthreads();
    auto st = [&](int rl, int c, u64 v) { X[rl * 256 + c] = v; };
    ntt::inv_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 8>(sm, ntt::TwPacked{D.twi + ((size_t)i << LOGN)}, R0,
                                                           m.q, m.two_q, st);
}

// ------------------------------------------------------------------ K2
template <int LOGN>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS)
k2_inv_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const uint2 jb = jobs[blockIdx.x / G::COL_TILES];
    const int c0 = (blockIdx.x % G::COL_TILES) * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 i = jb.y;
    const ModC m = D.mod[i];
    const Level& lv = D.lvl[P.L];
    const u64 sc = P.mode == RESCALE ? D.ninv[i] : lv.up_scale[i];
    const u64 scp = P.mode == RESCALE ? D.ninvp[i] : lv.up_scale_p[i];
    const WsLayout w = ws_layout(P.L, D.K, D.alpha);
    u64* X = P.ws + ((size_t)(w.X + i) << LOGN) + c0;
    auto ld = [&](int r, int cl) { return X[r * 256 + cl]; };
    auto st = [&](int r, int cl, u64 v) { X[r * 256 + cl] = shoup(v, sc, scp, m.q); };
    ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A>(sm, ntt::TwPacked{D.twi + ((size_t)i << LOGN)}, m.q,
                                                          m.two_q, ld, st);
}

// ------------------------------------------------------------------ K3
template <int LOGN>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS)
k3_modup_fwd_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    __shared__ u64 cst[MAXA];
    const uint2 jb = jobs[blockIdx.x / G::COL_TILES];
    const int c0 = (blockIdx.x % G::COL_TILES) * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K, QlP = L + K;
    const u32 p = jb.y / QlP, i = jb.y % QlP;
    const Level& lv = D.lvl[L];
    const u32 st0 = lv.part_st[p], sp = lv.part_sp[p];
    const u32 qp = qp_of(i, L, D.fullQ);
    const ModC m = D.mod[qp];
    if (threadIdx.x < sp) cst[threadIdx.x] = D.pool[lv.qmp_off + (st0 + threadIdx.x) * QlP + i];
    __syncthreads();
    const WsLayout w = ws_layout(L, K, D.alpha);
    const u64* X = P.ws + ((size_t)(w.X + st0) << LOGN) + c0;
    u64* Y = P.ws + ((size_t)(w.Y + p * QlP + i) << LOGN) + c0;
    auto ld = [&](int r, int cl) {
        const u64* x = X + r * 256 + cl;
        u64 lo = 0, hi = 0;
#pragma unroll 4
        for (u32 s = 0; s < sp; ++s) mac_wide(lo, hi, x[(size_t)s << LOGN], cst[s]);
        return barrett_lazy(lo, hi, m.q, m.mu_lo, m.mu_hi);
    };
    auto st = [&](int r, int cl, u64 v) { Y[r * 256 + cl] = v; };
    ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0>(sm, ntt::TwPacked{D.twf + ((size_t)qp << LOGN)}, m.q,
                                                       m.two_q, ld, st);
}

// ------------------------------------------------------------------ K4
template <int LOGN>
__global__ void __launch_bounds__(PG<LOGN>::MAC_THREADS)
k4_mac_fwd_row(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    using G = ntt::Geo<LOGN>;
    using PGL = PG<LOGN>;
    constexpr int NT = PGL::MAC_THREADS, RB = PGL::MAC_RB;
    extern __shared__ __align__(16) u64 sm[];
    const uint2 jb = jobs[blockIdx.x / PGL::MAC_TILES];
    const u32 R0 = (blockIdx.x % PGL::MAC_TILES) * RB;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K, QlP = L + K, i = jb.y;
    const Level& lv = D.lvl[L];
    const u32 qp = qp_of(i, L, D.fullQ);
    const ModC m = D.mod[qp];
    const WsLayout w = ws_layout(L, K, D.alpha);
    const size_t tile0 = (size_t)R0 * 256;
    const ntt::TwPacked twf{D.twf + ((size_t)qp << LOGN)};
    const size_t krow = (size_t)qp;   // full-QP key row of QlP position i

    u64 a0l[8], a0h[8], a1l[8], a1h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a0l[k] = a0h[k] = a1l[k] = a1h[k] = 0;

    for (u32 p = 0; p < lv.nparts; ++p) {
        const u32 st0 = lv.part_st[p], sp = lv.part_sp[p];
        const bool in_range = i >= st0 && i < st0 + sp;
        const size_t kofs = (((size_t)p * D.QP + krow) << LOGN) + tile0;
        const u64* kb = P.kbv + kofs;
        const u64* ka = P.kav + kofs;
        if (in_range) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const u32 e = threadIdx.x + k * NT;
                const u64 v = digit_src<LOGN>(P, i, (u32)tile0 + e, m);
                mac_wide(a0l[k], a0h[k], v, kb[e]);
                mac_wide(a1l[k], a1h[k], v, ka[e]);
            }
        } else {
            const u64* Y = P.ws + ((size_t)(w.Y + p * QlP + i) << LOGN) + tile0;
            auto ld = [&](int rl, int c) { return Y[rl * 256 + c]; };
            ntt::fwd_row_rounds<G::A, RB, NT, 3, 0>(sm, twf, R0, m.q, m.two_q, ld);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const u32 e = threadIdx.x + k * NT;
                const u64 v = csub(sm[(e >> 8) * G::ROW_STRIDE + ntt::rowpad(e & 255)], m.two_q);
                mac_wide(a0l[k], a0h[k], v, kb[e]);
                mac_wide(a1l[k], a1h[k], v, ka[e]);
            }
            __syncthreads();
        }
    }
    u64 r0[8], r1[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        r0[k] = barrett(a0l[k], a0h[k], m);
        r1[k] = barrett(a1l[k], a1h[k], m);
    }

    const bool is_q = i < L;
    const bool drop = P.mode == EMR && i == L - 1;
    if (is_q && !drop) {
        // W = (t + res*P^-1)*s1 (EvalMult+Rescale) or res*P^-1 (keyswitch)
        u64* W0 = P.ws + ((size_t)(w.W + i) << LOGN) + tile0;
        u64* W1 = P.ws + ((size_t)(w.W + L + i) << LOGN) + tile0;
        const u64 q = m.q;
        if (P.mode == EMR) {
            const u64 s1 = lv.s1[i], s1p = lv.s1p[i], ps1 = lv.ps1[i], ps1p = lv.ps1p[i];
            const size_t o = ((size_t)i << LOGN) + tile0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const u32 e = threadIdx.x + k * NT;
                const u64 x0 = P.in[0][o + e], x1 = P.in[1][o + e], y0 = P.in[2][o + e], y1 = P.in[3][o + e];
                const u64 t0 = mulmod(x0, y0, m);
                u64 lo, hi;
                mul_wide(x0, y1, lo, hi);
                mac_wide(lo, hi, x1, y0);
                const u64 t1 = barrett(lo, hi, m);
                W0[e] = csub(csub(shoup_lazy(t0, s1, s1p, q) + shoup_lazy(r0[k], ps1, ps1p, q), m.two_q), q);
                W1[e] = csub(csub(shoup_lazy(t1, s1, s1p, q) + shoup_lazy(r1[k], ps1, ps1p, q), m.two_q), q);
            }
        } else {
            const u64 pv = D.pinv[i], pvp = D.pinvp[i];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const u32 e = threadIdx.x + k * NT;
                W0[e] = shoup(r0[k], pv, pvp, q);
                W1[e] = shoup(r1[k], pv, pvp, q);
            }
        }
        return;
    }
    // dropped tower (u = t + res*P^-1) or P tower (res): INTT row stages
    if (drop) {
        const u64 pv = D.pinv[i], pvp = D.pinvp[i];
        const size_t o = ((size_t)i << LOGN) + tile0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const u32 e = threadIdx.x + k * NT;
            const u64 x0 = P.in[0][o + e], x1 = P.in[1][o + e], y0 = P.in[2][o + e], y1 = P.in[3][o + e];
            const u64 t0 = mulmod(x0, y0, m);
            u64 lo, hi;
            mul_wide(x0, y1, lo, hi);
            mac_wide(lo, hi, x1, y0);
            const u64 t1 = barrett(lo, hi, m);
            r0[k] = csub(t0 + shoup(r0[k], pv, pvp, m.q), m.q);
            r1[k] = csub(t1 + shoup(r1[k], pv, pvp, m.q), m.q);
        }
    }
    const ntt::TwPacked twi{D.twi + ((size_t)qp << LOGN)};
    for (int c = 0; c < 2; ++c) {
        u64* dst = drop ? P.ws + ((size_t)(w.U + c) << LOGN) + tile0
                        : P.ws + ((size_t)(w.RP + c * K + (i - L)) << LOGN) + tile0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const u32 e = threadIdx.x + k * NT;
            sm[(e >> 8) * G::ROW_STRIDE + ntt::rowpad(e & 255)] = c ? r1[k] : r0[k];
        }
        __syncthreads();
        auto st = [&](int rl, int cc, u64 v) { dst[rl * 256 + cc] = v; };
        ntt::inv_row_rounds<G::A, RB, NT, 3, 8>(sm, twi, R0, m.q, m.two_q, st);
        __syncthreads();
    }
}

// ------------------------------------------------------------------ K5
template <int LOGN>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS)
k5_moddown_inv_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const uint2 jb = jobs[blockIdx.x / G::COL_TILES];
    const int c0 = (blockIdx.x % G::COL_TILES) * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K;
    const u32 c = jb.y / (K + 1), t = jb.y % (K + 1);
    const WsLayout w = ws_layout(L, K, D.alpha);
    u32 qp, slot;
    u64 sc, scp;
    if (t == 0) { qp = L - 1; slot = w.U + c; sc = D.ninv[qp]; scp = D.ninvp[qp]; }
    else { qp = D.fullQ + t - 1; slot = w.RP + c * K + (t - 1); sc = D.pdn[t - 1]; scp = D.pdnp[t - 1]; }
    const ModC m = D.mod[qp];
    u64* X = P.ws + ((size_t)slot << LOGN) + c0;
    auto ld = [&](int r, int cl) { return X[r * 256 + cl]; };
    auto st = [&](int r, int cl, u64 v) { X[r * 256 + cl] = shoup(v, sc, scp, m.q); };
    ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A>(sm, ntt::TwPacked{D.twi + ((size_t)qp << LOGN)}, m.q,
                                                          m.two_q, ld, st);
}

// ------------------------------------------------------------------ K6
template <int LOGN>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS)
k6_moddown_fwd_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    __shared__ u64 ci[gfx::MAXP], cl_[gfx::MAXP];
    const uint2 jb = jobs[blockIdx.x / G::COL_TILES];
    const int c0 = (blockIdx.x % G::COL_TILES) * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K, mode = P.mode;
    const u32 c = jb.y / L, i = jb.y % L;
    const u32 l = L - 1;
    const WsLayout w = ws_layout(L, K, D.alpha);
    const Level& lv = D.lvl[L];
    const ModC m = D.mod[i];
    const ModC ml = D.mod[l];
    if (threadIdx.x < K) {
        ci[threadIdx.x] = D.phatmodq[threadIdx.x * D.fullQ + i];
        cl_[threadIdx.x] = D.phatmodq[threadIdx.x * D.fullQ + l];
    }
    __syncthreads();
    const u64* XP = P.ws + ((size_t)(w.RP + c * K) << LOGN) + c0;
    const u64* UC = mode == RESCALE ? P.ws + ((size_t)(w.X + l) << LOGN) + c0
                                    : P.ws + ((size_t)(w.U + c) << LOGN) + c0;
    u64* Z = P.ws + ((size_t)(w.Z + c * L + i) << LOGN) + c0;
    const u64 q = m.q;
    // SwitchModulus q_l -> q_i (switch_modulus.cu:11-27)
    const u64 half = ml.q >> 1;
    const bool larger = q > ml.q;
    const u64 diff = larger ? q - ml.q : (ml.q - q) % q;
    auto swm = [&](u64 r) -> u64 {
        const u64 d = r > half ? diff : 0;
        if (larger) return r + d;
        const u64 xm = reduce64(r, m);
        return xm >= d ? xm - d : xm + q - d;
    };
    auto conv = [&](const u64* x, const u64* cst, const ModC& mm) {
        u64 lo = 0, hi = 0;
        for (u32 j = 0; j < K; ++j) mac_wide(lo, hi, x[(size_t)j << LOGN], cst[j]);
        return barrett_lazy(lo, hi, mm.q, mm.mu_lo, mm.mu_hi);
    };
    auto ld = [&](int r, int cl) -> u64 {
        const int e = r * 256 + cl;
        if (mode == RESCALE) return shoup_lazy(swm(UC[e]), lv.s2[i], lv.s2p[i], q);
        const u64 cvi = conv(XP + e, ci, m);
        if (mode != EMR) return 2 * q - shoup_lazy(cvi, D.pinv[i], D.pinvp[i], q);
        const u64 cvl = conv(XP + e, cl_, ml);
        const u64 tmp = shoup(cvl, D.pinv[l], D.pinvp[l], ml.q);
        const u64 u = UC[e];
        const u64 rl = u >= tmp ? u - tmp : u + ml.q - tmp;
        return shoup_lazy(swm(rl), lv.s2[i], lv.s2p[i], q) + 2 * q - shoup_lazy(cvi, lv.ps1[i], lv.ps1p[i], q);
    };
    auto st = [&](int r, int cl, u64 v) { Z[r * 256 + cl] = v; };
    ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0>(sm, ntt::TwPacked{D.twf + ((size_t)i << LOGN)}, q,
                                                       m.two_q, ld, st);
}

// ------------------------------------------------------------------ K7
template <int LOGN>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS)
k7_final_fwd_row(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const uint2 jb = jobs[blockIdx.x / G::ROW_TILES];
    const u32 R0 = (blockIdx.x % G::ROW_TILES) * G::RB;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K, mode = P.mode;
    const u32 c = jb.y / L, i = jb.y % L;
    const WsLayout w = ws_layout(L, K, D.alpha);
    const ModC m = D.mod[i];
    const size_t tile0 = (size_t)R0 * 256;
    const u64* Z = P.ws + ((size_t)(w.Z + c * L + i) << LOGN) + tile0;
    auto ld = [&](int rl, int cc) { return Z[rl * 256 + cc]; };
    ntt::fwd_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 0>(sm, ntt::TwPacked{D.twf + ((size_t)i << LOGN)}, R0, m.q,
                                                           m.two_q, ld);
    const size_t o = ((size_t)i << LOGN) + tile0;
    u64* out = P.out[c] + o;
    const u64* Wt = P.ws + ((size_t)(w.W + c * L + i) << LOGN) + tile0;
    const Level& lv = D.lvl[L];
    const u64 s1 = lv.s1[i], s1p = lv.s1p[i];
    ntt::row_tile_walk<G::RB, G::ROW_THREADS>([&](int rl, int cc) {
        const int e = rl * 256 + cc;
        const u64 v = csub(csub(sm[rl * G::ROW_STRIDE + ntt::rowpad(cc)], m.two_q), m.q);
        u64 r;
        if (mode == RESCALE) {
            r = csub(shoup(P.in[0][o + e], s1, s1p, m.q) + v, m.q);
        } else {
            r = csub(Wt[e] + v, m.q);
            if (mode == ROT && c == 0)
                r = csub(r + P.in[0][((size_t)i << LOGN) + galois_slot<LOGN>((u32)(tile0 + e), P.galois)], m.q);
        }
        out[e] = r;
    });
}

}  // namespace pl
