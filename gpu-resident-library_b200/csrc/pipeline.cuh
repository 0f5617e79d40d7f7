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
// Pass-to-pass intermediates (X after P1, Y after P3, Z after P8) are kept in
// the arithmetic path's own word format; every other slot holds u64 residues.
//
// Phases (one launch each per arithmetic path; jobs are (pair, sub) unless noted):
//   P1 inv-row  (pair,i)       tensor / gather prologue, INTT row stages     -> X
//   P2 inv-col  (pair,i)       INTT column stages, * n^-1 QHatInv            -> X
//   P3 fwd-col  (pair,p,i)     ModUp conversion prologue, NTT column stages  -> Y
//   P4 fwd-row  (pair,p,i)     NTT row stages                               -> Y (eval digit)
//   P5 MAC      (row,group)    key-stationary inner product over the batch:
//                              one CTA keeps a key-row tile of every digit in
//                              shared memory and streams all pairs using it -> W / U / RP
//   P6 inv-row  (pair,c,t)     INTT row stages of U (dropped tower) and RP   -> U / RP
//   P7 inv-col  (pair,c,t)     INTT columns of RP, scaled; then (pair,c) U and r_l -> RP / U
//   P8 fwd-col  (pair,c,i)     ModDown conversion + SwitchModulus prologue   -> Z
//   P9 fwd-row  (pair,c,i)     NTT row stages, final combine                -> out
#pragma once
#include <type_traits>

#include "context.hpp"
#include "ntt.cuh"

namespace pl {

using gfx::DevCtx;
using gfx::Level;

constexpr int NPHASE = 9;
constexpr int MAXA = 16;       // digit width supported by the fused ModUp prologue
constexpr int MAC_TILE = 512;  // P5 elements per CTA
constexpr int MAC_NT = 128;    // P5 threads of the 4-word form (the 2-word form has 256)
constexpr int MAC_GROUP = 16;  // P5 pairs streamed per CTA

enum Mode : u32 {
    EMR = 0,       // EvalMult + Rescale: in = c0a,c1a,c0b,c1b [L]; out0,out1 [L-1]
    KS = 1,        // keyswitch: in[0] = a [L]; out0,out1 = ba0, ba1 [L]
    ROT = 2,       // rotation: in = c0, c1 [L]; out = sigma(c0)+ba0, ba1 [L]
    RESCALE = 3,   // rescale: in[0] = comp [L]; out0 = [L-1] (may alias in[0])
    HROT = 4,      // hoisted rotation: as ROT, but operations of one batch with the same
                   // c1 buffer and level share one ModUp of c1 (computed by the first of
                   // them); each applies sigma_k to the shared digits in eval form
};

struct PairDesc {
    u32 L;
    u32 mode;
    u64 galois;            // ROT: Galois element k (odd, < 2n)
    const u64* in[4];
    u64* out[2];
    u64* ws;
    const u64* ysrc;       // workspace holding the ModUp digits (own ws; HROT: the group's first)
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

// Digit source value at element e of Q tower i (eval form, canonical).
template <int LOGN>
__device__ __forceinline__ u64 digit_src(const PairDesc& P, u32 i, u32 e, const ModC& m) {
    const size_t o = ((size_t)i << LOGN);
    if (P.mode == EMR) return mulmod(P.in[1][o + e], P.in[3][o + e], m);
    if (P.mode == ROT) return P.in[1][o + galois_slot<LOGN>(e, P.galois)];
    if (P.mode == HROT) return P.in[1][o + e];   // ModUp source of a hoisted group: c1 itself
    return P.in[0][o + e];
}

__device__ __forceinline__ u64* slot_ptr(const PairDesc& P, u32 slot, int logn) {
    return P.ws + ((size_t)slot << logn);
}

// Arithmetic policy and twiddle accessors of the integer (FP = false) or the
// FP64 (FP = true, towers with q < 2^50) instantiation of a phase kernel.
template <bool FP>
__device__ __forceinline__ auto ar_of(const ModC& m) {
    if constexpr (FP) return ntt::FpArS{ntt::u2d(m.q), qinv_of(m)};
    else return ntt::IntAr{m.q, m.two_q};
}
template <bool FP>
__device__ __forceinline__ auto twf_of(const DevCtx& D, u32 qp, int logn) {
    if constexpr (FP) return ntt::TwD{D.twfd + ((size_t)qp << logn)};
    else return ntt::TwPacked{D.twf + ((size_t)qp << logn)};
}
template <bool FP>
__device__ __forceinline__ auto twi_of(const DevCtx& D, u32 qp, int logn) {
    if constexpr (FP) return ntt::TwD{D.twid + ((size_t)qp << logn)};
    else return ntt::TwPacked{D.twi + ((size_t)qp << logn)};
}

// Arithmetic path of a transform kernel launch: PATH 0 = integer jobs only,
// 1 = FP64 jobs only, 2 = a mixed job list whose FP64 jobs carry bit 31 of
// job.y (integer- and FP64-bound CTAs then share each SM's pipes).
constexpr u32 JOB_FP = 0x80000000u;
template <int PATH, class F>
__device__ __forceinline__ void on_path(uint2& jb, F&& f) {
    if constexpr (PATH == 2) {
        const bool fp = (jb.y & JOB_FP) != 0;
        jb.y &= ~JOB_FP;
        if (fp) f(std::true_type{});
        else f(std::false_type{});
    } else {
        f(std::integral_constant<bool, PATH == 1>{});
    }
}

// Column-tile staging: the prologue of a column pass (a basis conversion)
// is computed for the whole tile into shared memory before the first round,
// reading its inputs as 16-byte column pairs with the loads of CS_VB pairs
// (and up to four conversion terms) in flight together. Thread t covers
// pairs t + k * COL_THREADS, k < PER; pair v sits at row v / (C/2), column
// 2 * (v % (C/2)), so a warp reads whole 128-byte row segments.
constexpr int CS_VB = 2;
constexpr int P8_VB = 1;   // P8 carries more live state per pair (three modes inlined)

template <int LOGN>
struct ColStage {
    using G = ntt::Geo<LOGN>;
    static constexpr int VPR = G::C / 2;
    static constexpr int PER = G::R1 * VPR / G::COL_THREADS;
    static_assert(PER * G::COL_THREADS == G::R1 * VPR && PER % CS_VB == 0, "column staging geometry");
    __device__ static __forceinline__ void pos(int k, int& r, int& cl) {
        const int v = threadIdx.x + k * G::COL_THREADS;
        r = v / VPR;
        cl = 2 * (v % VPR);
    }
};

__device__ __forceinline__ ulonglong2 ld2(const u64* p) { return *reinterpret_cast<const ulonglong2*>(p); }

// One key-switch accumulator -> res (P rows) or res * P^-1 (Q rows), canonical:
// the stored key carries P^-1 on Q rows and, with D.mont, the factor 2^64
// that the Montgomery reduction removes.
__device__ __forceinline__ u64 acc_reduce(u64 lo, u64 hi, const ModC& m, u32 mont) {
    return mont ? redc(lo, hi, m) : barrett(lo, hi, m);
}
// A basis-conversion sum whose constants carry 2^64 when `mont` (else plain):
// lazy residue in [0, 4q).
__device__ __forceinline__ u64 conv_reduce(u64 lo, u64 hi, const ModC& m, u32 mont) {
    return mont ? redc_lazy(lo, hi, m) : barrett_lazy(lo, hi, m.q, m.mu_lo, m.mu_hi);
}

// lo/hi[b][j] += sum_{t < nterms} base[t * stride + e[b] + j] * coef[t] (128-bit).
template <int VB>
__device__ __forceinline__ void mac_terms(u64 (&lo)[VB][2], u64 (&hi)[VB][2], const u64* base, size_t stride,
                                          u32 nterms, const u64* coef, const size_t (&e)[VB]) {
    for (u32 t0 = 0; t0 < nterms; t0 += 4) {
        ulonglong2 xv[4][VB];
#pragma unroll
        for (int tt = 0; tt < 4; ++tt)
            if (t0 + tt < nterms)
#pragma unroll
                for (int b = 0; b < VB; ++b) xv[tt][b] = ld2(base + (t0 + tt) * stride + e[b]);
#pragma unroll
        for (int tt = 0; tt < 4; ++tt)
            if (t0 + tt < nterms) {
                const u64 c = coef[t0 + tt];
#pragma unroll
                for (int b = 0; b < VB; ++b) {
                    mac_wide(lo[b][0], hi[b][0], xv[tt][b].x, c);
                    mac_wide(lo[b][1], hi[b][1], xv[tt][b].y, c);
                }
            }
    }
}

// ------------------------------------------------------------------ P1
template <int LOGN, bool FP>
__device__ __forceinline__ void p1_inv_row_body(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint2 jb,
                                              const u32 tile) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const u32 R0 = tile * G::RB;
    const PairDesc& P = pairs[jb.x];
    const u32 i = jb.y;
    const ModC m = D.mod[i];
    const auto ar = ar_of<FP>(m);
    const WsLayout w = ws_layout(P.L, D.K, D.alpha);
    u64* X = slot_ptr(P, w.X + i, LOGN) + (size_t)R0 * 256;
    if (P.mode == EMR) {   // d2 = a1 * b1: both operands of a batch loaded before the products
        const size_t o = ((size_t)i << LOGN) + (size_t)R0 * 256;
        ntt::row_tile_stage2<G::RB, G::ROW_THREADS>(
            [&](int rl, int c) { return P.in[1][o + rl * 256 + c]; },
            [&](int rl, int c) { return P.in[3][o + rl * 256 + c]; },
            [&](int rl, int c, u64 a, u64 b) {
                u64 v;
                if constexpr (FP) {   // canonical operands: the product exactly on the FP64 pipe
                    if (a < m.q && b < m.q) {
                        const ntt::FpAr ua{ntt::u2d(m.q), qinv_of(m)};
                        v = ar.bits(ua.norm(ua.mulq<true>(ntt::u2d(a), ntt::u2d(b))));
                    } else {
                        v = ar.stage_in(mulmod(a, b, m));
                    }
                } else {
                    v = ar.stage_in(mulmod(a, b, m));
                }
                sm[rl * G::ROW_STRIDE + ntt::rowpad(c)] = v;
            });
    } else {
        ntt::row_tile_stage<G::RB, G::ROW_THREADS>(
            [&](int rl, int c) { return digit_src<LOGN>(P, i, (R0 + rl) * 256 + c, m); },
            [&](int rl, int c, u64 v) { sm[rl * G::ROW_STRIDE + ntt::rowpad(c)] = ar.stage_in(v); });
    }
    __syncthreads();
    auto st = [&](int rl, int c, u64 v) { X[rl * 256 + c] = v; };
    ntt::inv_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 8, true>(sm, twi_of<FP>(D, i, LOGN), R0, ar, st);
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS, 4)
p1_inv_row(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::ROW_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::ROW_TILES;
    on_path<PATH>(jb, [&](auto fp) { p1_inv_row_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

// ------------------------------------------------------------------ P2
template <int LOGN, bool FP>
__device__ __forceinline__ void p2_inv_col_body(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint2 jb,
                                              const u32 tile) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const int c0 = tile * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 i = jb.y;
    const ModC m = D.mod[i];
    const Level& lv = D.lvl[P.L];
    const u64 sc = P.mode == RESCALE ? D.ninv[i] : lv.up_scale[i];
    const u64 scp = P.mode == RESCALE ? D.ninvp[i] : lv.up_scale_p[i];
    const WsLayout w = ws_layout(P.L, D.K, D.alpha);
    u64* X = slot_ptr(P, w.X + i, LOGN) + c0;
    auto ld = [&](int r, int cl) { return X[r * 256 + cl]; };
    if constexpr (FP) {   // the scale as an exact FP64 product (v, sc < q < 2^50), canonical
        const ntt::FpAr ua{ntt::u2d(m.q), qinv_of(m)};
        const double scd = ntt::u2d(sc);
        auto st = [&](int r, int cl, u64 v) { X[r * 256 + cl] = ua.out(ua.norm(ua.mulq<true>(ntt::u2d(v), scd))); };
        ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A, true>(sm, twi_of<FP>(D, i, LOGN), ar_of<FP>(m), ld, st);
    } else {
        auto st = [&](int r, int cl, u64 v) { X[r * 256 + cl] = shoup(v, sc, scp, m.q); };
        ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A, true>(sm, twi_of<FP>(D, i, LOGN), ar_of<FP>(m), ld, st);
    }
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
p2_inv_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::COL_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::COL_TILES;
    on_path<PATH>(jb, [&](auto fp) { p2_inv_col_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

// ------------------------------------------------------------------ P3
template <int LOGN, bool FP>
__device__ __forceinline__ void p3_modup_fwd_col_body(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint2 jb,
                                              const u32 tile) {
    using G = ntt::Geo<LOGN>;
    using CS = ColStage<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    __shared__ u64 cst[MAXA];
    const int c0 = tile * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K, QlP = L + K;
    const u32 p = jb.y / QlP, i = jb.y % QlP;
    const Level& lv = D.lvl[L];
    const u32 st0 = lv.part_st[p], sp = lv.part_sp[p];
    const u32 qp = qp_of(i, L, D.fullQ);
    const ModC m = D.mod[qp];
    const WsLayout w = ws_layout(L, K, D.alpha);
    const u64* X = slot_ptr(P, w.X + st0, LOGN) + c0;
    u64* Y = slot_ptr(P, w.Y + p * QlP + i, LOGN) + c0;
    // A 50-bit target whose digit has at most three sources, all below 2^50,
    // converts on the FP64 pipe: every term x_s * QHatModp[s][i] is an exact
    // FP64 modular product of unsigned operands (|r| <= 2q), their sum stays
    // below 6q < 2^53, and one normalisation gives the canonical residue.
    bool fpc = false;
    if constexpr (FP) {
        fpc = sp <= 3;
        for (u32 s = 0; s < sp; ++s) fpc = fpc && fp_tower(D.mod[st0 + s].q);
    }
    const u64* pool = D.pool + (fpc ? lv.qmpp_off : lv.qmp_off) + (size_t)st0 * QlP + i;
    if (threadIdx.x < sp) {
        const u64 c = pool[(size_t)threadIdx.x * QlP];
        cst[threadIdx.x] = fpc ? (u64)__double_as_longlong(ntt::u2d(c)) : c;
    }
    __syncthreads();
    if (fpc) {
        const ntt::FpAr ua{ntt::u2d(m.q), qinv_of(m)};
#pragma unroll 1
        for (int k0 = 0; k0 < CS::PER; k0 += CS_VB) {
            int r[CS_VB], cl[CS_VB];
            size_t e[CS_VB];
            ulonglong2 xv[3][CS_VB];
#pragma unroll
            for (int b = 0; b < CS_VB; ++b) {
                CS::pos(k0 + b, r[b], cl[b]);
                e[b] = (size_t)r[b] * 256 + cl[b];
            }
#pragma unroll
            for (int t = 0; t < 3; ++t)
                if ((u32)t < sp)
#pragma unroll
                    for (int b = 0; b < CS_VB; ++b) xv[t][b] = ld2(X + ((size_t)t << LOGN) + e[b]);
#pragma unroll
            for (int b = 0; b < CS_VB; ++b) {
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int t = 0; t < 3; ++t)
                    if ((u32)t < sp) {
                        const double c = __longlong_as_double((long long)cst[t]);
                        a0 = __dadd_rn(a0, ua.mulq<true>(ntt::u2d(xv[t][b].x), c));
                        a1 = __dadd_rn(a1, ua.mulq<true>(ntt::u2d(xv[t][b].y), c));
                    }
                ulonglong2 v;
                v.x = ua.out(ua.norm(a0));
                v.y = ua.out(ua.norm(a1));
                *reinterpret_cast<ulonglong2*>(sm + r[b] * G::C + cl[b]) = v;
            }
        }
        __syncthreads();
        auto ld = [&](int r, int cl) { return sm[r * G::C + cl]; };
        auto stf = [&](int r, int cl, u64 v) { Y[r * 256 + cl] = v; };
        ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0, true>(sm, twf_of<FP>(D, qp, LOGN), ar_of<FP>(m), ld, stf);
        return;
    }
    // conv_i = sum_s x_s * QHatModp[s][i] (ApproxSwitchCRTBasis), lazy in [0, 4q)
#pragma unroll 1
    for (int k0 = 0; k0 < CS::PER; k0 += CS_VB) {
        int r[CS_VB], cl[CS_VB];
        size_t e[CS_VB];
        u64 lo[CS_VB][2] = {}, hi[CS_VB][2] = {};
#pragma unroll
        for (int b = 0; b < CS_VB; ++b) {
            CS::pos(k0 + b, r[b], cl[b]);
            e[b] = (size_t)r[b] * 256 + cl[b];
        }
        mac_terms<CS_VB>(lo, hi, X, (size_t)1 << LOGN, sp, cst, e);
#pragma unroll
        for (int b = 0; b < CS_VB; ++b) {
            ulonglong2 v;
            v.x = conv_reduce(lo[b][0], hi[b][0], m, D.mont_up);
            v.y = conv_reduce(lo[b][1], hi[b][1], m, D.mont_up);
            *reinterpret_cast<ulonglong2*>(sm + r[b] * G::C + cl[b]) = v;
        }
    }
    __syncthreads();
    auto ld = [&](int r, int cl) { return sm[r * G::C + cl]; };
    auto stf = [&](int r, int cl, u64 v) { Y[r * 256 + cl] = v; };
    ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0, true>(sm, twf_of<FP>(D, qp, LOGN), ar_of<FP>(m), ld, stf);
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
p3_modup_fwd_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::COL_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::COL_TILES;
    on_path<PATH>(jb, [&](auto fp) { p3_modup_fwd_col_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

// P3, warp-specialised form: a persistent CTA of COL_THREADS transform threads
// and NP conversion threads over a double-buffered tile ring (MINB CTAs per SM). While the
// transform warps run the column NTT of tile k (FP64 or integer butterflies),
// the NP conversion threads compute the ApproxSwitchCRTBasis prologue of tile k+1
// (integer 128-bit MACs) into the other buffer, so the two pipes overlap.
// Hand-over uses named barriers: FULL[b] (conversion -> transform) and
// EMPTY[b] (transform -> conversion); both sides walk the same tile sequence,
// and a transform warp releases a buffer only if a later tile will refill it.
// Results equal p3_modup_fwd_col's word for word.
constexpr unsigned BAR_FULL = 1, BAR_EMPTY = 3, BAR_XFORM = 5, BAR_CONV = 6;

__device__ __forceinline__ void nb_sync(unsigned id, unsigned count) {
    asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void nb_arrive(unsigned id, unsigned count) {
    asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}

template <int LOGN, int NP>
struct P3WS {
    using G = ntt::Geo<LOGN>;
    static constexpr int NC = G::COL_THREADS;                // transform threads
    static constexpr int NT = NC + NP;                       // NP conversion threads
    static constexpr int SMEM = 2 * G::COL_SMEM;
    static constexpr int VPR = G::C / 2;
    static constexpr int PPER = G::R1 * VPR / NP;            // 16-byte pairs per conversion thread
    static_assert(PPER * NP == G::R1 * VPR && PPER % CS_VB == 0, "conversion geometry");
};

struct XformSync {
    unsigned count;
    __device__ __forceinline__ void operator()() const { nb_sync(BAR_XFORM, count); }
};

template <int LOGN, int PATH, int NP, int MINB>
__global__ void __launch_bounds__(P3WS<LOGN, NP>::NT, MINB)
p3ws_modup_fwd_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs,
                   const u32 ntiles) {
    using G = ntt::Geo<LOGN>;
    using W = P3WS<LOGN, NP>;
    extern __shared__ __align__(16) u64 sm[];   // [2][COL_TILE]
    __shared__ u64 cst[2][MAXA];
    const bool conv = threadIdx.x >= W::NC;
    const u32 ctid = threadIdx.x - W::NC;
    u32 k = 0;
    for (u32 t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
        const int b = (int)(k & 1);
        uint2 jb = jobs[t / G::COL_TILES];
        const int c0 = (int)(t % G::COL_TILES) * G::C;
        bool fp = PATH == 1;
        if constexpr (PATH == 2) {
            fp = (jb.y & JOB_FP) != 0;
            jb.y &= ~JOB_FP;
        }
        const PairDesc& P = pairs[jb.x];
        const u32 L = P.L, K = D.K, QlP = L + K;
        const u32 p = jb.y / QlP, i = jb.y % QlP;
        const Level& lv = D.lvl[L];
        const u32 st0 = lv.part_st[p], sp = lv.part_sp[p];
        const u32 qp = qp_of(i, L, D.fullQ);
        const ModC m = D.mod[qp];
        const WsLayout w = ws_layout(L, K, D.alpha);
        u64* buf = sm + (size_t)b * G::COL_TILE;
        if (conv) {
            if (k >= 2) nb_sync(BAR_EMPTY + b, W::NT);      // transform warps released buffer b
            const u64* pool = D.pool + lv.qmp_off + (size_t)st0 * QlP + i;
            if (ctid < sp) cst[b][ctid] = pool[(size_t)ctid * QlP];
            nb_sync(BAR_CONV, NP);
            const u64* X = slot_ptr(P, w.X + st0, LOGN) + c0;
#pragma unroll 1
            for (int k0 = 0; k0 < W::PPER; k0 += CS_VB) {
                int r[CS_VB], cl[CS_VB];
                size_t e[CS_VB];
                u64 lo[CS_VB][2] = {}, hi[CS_VB][2] = {};
#pragma unroll
                for (int bb = 0; bb < CS_VB; ++bb) {
                    const int v = (int)ctid + (k0 + bb) * NP;
                    r[bb] = v / W::VPR;
                    cl[bb] = 2 * (v % W::VPR);
                    e[bb] = (size_t)r[bb] * 256 + cl[bb];
                }
                mac_terms<CS_VB>(lo, hi, X, (size_t)1 << LOGN, sp, cst[b], e);
#pragma unroll
                for (int bb = 0; bb < CS_VB; ++bb) {
                    ulonglong2 v;
                    v.x = conv_reduce(lo[bb][0], hi[bb][0], m, D.mont_up);
                    v.y = conv_reduce(lo[bb][1], hi[bb][1], m, D.mont_up);
                    *reinterpret_cast<ulonglong2*>(buf + r[bb] * G::C + cl[bb]) = v;
                }
            }
            nb_arrive(BAR_FULL + b, W::NT);                 // buffer b staged
        } else {
            nb_sync(BAR_FULL + b, W::NT);
            u64* Y = slot_ptr(P, w.Y + p * QlP + i, LOGN) + c0;
            auto ld = [&](int r, int cl) { return buf[r * G::C + cl]; };
            auto stf = [&](int r, int cl, u64 v) { Y[r * 256 + cl] = v; };
            const XformSync xs{(unsigned)W::NC};
            if (fp)
                ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0, true>(buf, twf_of<true>(D, qp, LOGN),
                                                                         ar_of<true>(m), ld, stf, xs);
            else
                ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0, true>(buf, twf_of<false>(D, qp, LOGN),
                                                                         ar_of<false>(m), ld, stf, xs);
            if (t + 2 * gridDim.x < ntiles) nb_arrive(BAR_EMPTY + b, W::NT);   // a later tile refills b
        }
    }
}

// ------------------------------------------------------------------ P4
// NTT row stages of one digit tower; output reduced to [0, 2q).
template <int LOGN, bool FP>
__device__ __forceinline__ void p4_modup_fwd_row_body(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint2 jb,
                                              const u32 tile) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const u32 R0 = tile * G::RB;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, QlP = L + D.K;
    const u32 p = jb.y / QlP, i = jb.y % QlP;
    const u32 qp = qp_of(i, L, D.fullQ);
    const ModC m = D.mod[qp];
    const WsLayout w = ws_layout(L, D.K, D.alpha);
    u64* Y = slot_ptr(P, w.Y + p * QlP + i, LOGN) + (size_t)R0 * 256;
    auto ld = [&](int rl, int c) { return Y[rl * 256 + c]; };
    const auto ar = ar_of<FP>(m);
    ntt::fwd_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 0, true>(sm, twf_of<FP>(D, qp, LOGN), R0, ar, ld);
    ntt::row_tile_walk<G::RB, G::ROW_THREADS>([&](int rl, int c) {
        Y[rl * 256 + c] = ar.final_2q(sm[rl * G::ROW_STRIDE + ntt::rowpad(c)]);
    });
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS, 4)
p4_modup_fwd_row(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::ROW_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::ROW_TILES;
    on_path<PATH>(jb, [&](auto fp) { p4_modup_fwd_row_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

// ------------------------------------------------------------------ P5
// Job: {key row r (QP index), offset into the pair-index list, pair count}.
// The CTA loads the key tile of row r for every digit (av and bv) into
// shared memory once, then for each listed pair accumulates
//   res_c = sum_p digit_p * key_p   (128-bit, one Barrett at the end)
// over that pair's digits and writes the epilogue for its QlP position.
// A thread owns MAC_TILE / MAC_NT elements as 16-byte pairs; for each pair it
// issues every load first (the pair's own-digit source and, for
// EvalMult+Rescale, the four tensor inputs; then the digits in chunks of
// MAC_PCH) so that many loads are in flight before the first multiply.
constexpr int MAC_PCH = 4;

__device__ __forceinline__ u64 v2get(const ulonglong2& v, int j) { return j ? v.y : v.x; }
__device__ __forceinline__ void v2set(ulonglong2& v, int j, u64 x) { if (j) v.y = x; else v.x = x; }


template <int LOGN, int NT>
__global__ void __launch_bounds__(NT, NT == 128 ? 4 : 3)
p5_mac(const DevCtx D, const PairDesc* __restrict__ pairs, const uint4* __restrict__ jobs,
       const u32* __restrict__ plist) {
    constexpr int TILES = (1 << LOGN) / MAC_TILE;
    constexpr int NV = MAC_TILE / (2 * NT);   // 16-byte vectors per thread
    extern __shared__ __align__(16) u64 sm[];     // [dnum][2][MAC_TILE]
    const uint4 jb = jobs[blockIdx.x / TILES];
    const u32 tile0 = (blockIdx.x % TILES) * MAC_TILE;
    const u32 r = jb.x;
    const ModC m = D.mod[r];
    const u32 dnum = D.dnum;
    // every listed pair uses the same key (checked on the host)
    const PairDesc& P0 = pairs[plist[jb.y]];
    for (u32 k = threadIdx.x; k < dnum * (MAC_TILE / 2); k += NT) {
        const u32 p = k / (MAC_TILE / 2), e = 2 * (k % (MAC_TILE / 2));
        const size_t off = (((size_t)p * D.QP + r) << LOGN) + tile0 + e;
        *reinterpret_cast<ulonglong2*>(sm + (2 * p) * MAC_TILE + e) = *reinterpret_cast<const ulonglong2*>(P0.kbv + off);
        *reinterpret_cast<ulonglong2*>(sm + (2 * p + 1) * MAC_TILE + e) =
            *reinterpret_cast<const ulonglong2*>(P0.kav + off);
    }
    __syncthreads();
    const bool is_p = r >= D.fullQ;
    const u64 q = m.q;
    for (u32 g = 0; g < jb.z; ++g) {
        const PairDesc& P = pairs[plist[jb.y + g]];
        const u32 L = P.L, K = D.K, QlP = L + K;
        const u32 i = is_p ? L + (r - D.fullQ) : r;       // QlP position of row r
        const Level& lv = D.lvl[L];
        const WsLayout w = ws_layout(L, K, D.alpha);
        const u32 nparts = lv.nparts;
        const u32 pin = is_p ? 0xffffffffu : i / D.alpha; // digit holding tower i
        const bool emr = P.mode == EMR;
        const size_t o = ((size_t)i << LOGN) + tile0;
        // own-digit source s (eval form) and, for EvalMult+Rescale, tensor t0, t1
        ulonglong2 s[NV], t0[NV], t1[NV];
        if (!is_p) {
            if (emr) {
                ulonglong2 x0[NV], x1[NV], y0[NV], y1[NV];
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    const u32 e = 2 * (threadIdx.x + k * NT);
                    x0[k] = *reinterpret_cast<const ulonglong2*>(P.in[0] + o + e);
                    x1[k] = *reinterpret_cast<const ulonglong2*>(P.in[1] + o + e);
                    y0[k] = *reinterpret_cast<const ulonglong2*>(P.in[2] + o + e);
                    y1[k] = *reinterpret_cast<const ulonglong2*>(P.in[3] + o + e);
                }
#pragma unroll
                for (int k = 0; k < NV; ++k)
#pragma unroll
                    for (int j = 0; j < 2; ++j) {   // tensor (Montgomery products with D.mont, see Key)
                        const u64 a0 = v2get(x0[k], j), a1 = v2get(x1[k], j);
                        const u64 b0 = v2get(y0[k], j), b1 = v2get(y1[k], j);
                        u64 lo, hi;
                        mul_wide(a1, b1, lo, hi);
                        v2set(s[k], j, acc_reduce(lo, hi, m, D.mont));
                        mul_wide(a0, b0, lo, hi);
                        v2set(t0[k], j, acc_reduce(lo, hi, m, D.mont));
                        mul_wide(a0, b1, lo, hi);
                        mac_wide(lo, hi, a1, b0);
                        v2set(t1[k], j, acc_reduce(lo, hi, m, D.mont));
                    }
            } else {
                if (P.mode == ROT || P.mode == HROT) {
                    const u64* src = P.in[1] + ((size_t)i << LOGN);
#pragma unroll
                    for (int k = 0; k < NV; ++k)
#pragma unroll
                        for (int j = 0; j < 2; ++j)
                            v2set(s[k], j, src[galois_slot<LOGN>(tile0 + 2 * (threadIdx.x + k * NT) + j, P.galois)]);
                } else {
#pragma unroll
                    for (int k = 0; k < NV; ++k)
                        s[k] = *reinterpret_cast<const ulonglong2*>(P.in[0] + o + 2 * (threadIdx.x + k * NT));
                }
                if (D.mont) {   // own-digit source times R^-1 (Key)
#pragma unroll
                    for (int k = 0; k < NV; ++k)
#pragma unroll
                        for (int j = 0; j < 2; ++j) v2set(s[k], j, redc(v2get(s[k], j), 0, m));
                }
            }
        }
        u64 a0l[2 * NV], a0h[2 * NV], a1l[2 * NV], a1h[2 * NV];
#pragma unroll
        for (int k = 0; k < 2 * NV; ++k) a0l[k] = a0h[k] = a1l[k] = a1h[k] = 0;
        for (u32 p0 = 0; p0 < nparts; p0 += MAC_PCH) {
            ulonglong2 v[MAC_PCH][NV];
#pragma unroll
            for (int pp = 0; pp < MAC_PCH; ++pp) {
                const u32 p = p0 + pp;
                if (p < nparts && p != pin) {
                    const u64* Yt = P.ysrc + ((size_t)(w.Y + p * QlP + i) << LOGN);
                    if (P.mode == HROT) {   // sigma_k of the shared digit: eval-slot gather
#pragma unroll
                        for (int k = 0; k < NV; ++k)
#pragma unroll
                            for (int j = 0; j < 2; ++j)
                                v2set(v[pp][k], j,
                                      Yt[galois_slot<LOGN>(tile0 + 2 * (threadIdx.x + k * NT) + j, P.galois)]);
                    } else {
                        const ulonglong2* Y = reinterpret_cast<const ulonglong2*>(Yt + tile0);
#pragma unroll
                        for (int k = 0; k < NV; ++k) v[pp][k] = __ldcs(Y + threadIdx.x + k * NT);
                    }
                }
            }
#pragma unroll
            for (int pp = 0; pp < MAC_PCH; ++pp) {
                const u32 p = p0 + pp;
                if (p >= nparts) break;
                const u64* kb = sm + (2 * p) * MAC_TILE;
                const u64* ka = sm + (2 * p + 1) * MAC_TILE;
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    const u32 e = 2 * (threadIdx.x + k * NT);
                    const ulonglong2 kbv = *reinterpret_cast<const ulonglong2*>(kb + e);
                    const ulonglong2 kav = *reinterpret_cast<const ulonglong2*>(ka + e);
                    const ulonglong2 dv = p == pin ? s[k] : v[pp][k];
                    mac_wide(a0l[2 * k], a0h[2 * k], dv.x, kbv.x);
                    mac_wide(a0l[2 * k + 1], a0h[2 * k + 1], dv.y, kbv.y);
                    mac_wide(a1l[2 * k], a1h[2 * k], dv.x, kav.x);
                    mac_wide(a1l[2 * k + 1], a1h[2 * k + 1], dv.y, kav.y);
                }
            }
        }
        // P rows and EvalMult Q rows carry R^-1 after Montgomery; keyswitch /
        // rotation Q rows are plain sums (Key)
        const u32 use_redc = D.mont && (is_p || emr);
        ulonglong2 r0[NV], r1[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                v2set(r0[k], j, acc_reduce(a0l[2 * k + j], a0h[2 * k + j], m, use_redc));
                v2set(r1[k], j, acc_reduce(a1l[2 * k + j], a1h[2 * k + j], m, use_redc));
            }
        u64 *d0, *d1;
        if (is_p) {
            d0 = slot_ptr(P, w.RP + (i - L), LOGN) + tile0;
            d1 = slot_ptr(P, w.RP + K + (i - L), LOGN) + tile0;
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const u32 e = 2 * (threadIdx.x + k * NT);
                *reinterpret_cast<ulonglong2*>(d0 + e) = r0[k];
                *reinterpret_cast<ulonglong2*>(d1 + e) = r1[k];
            }
            continue;
        }
        if (!emr) {   // keyswitch / rotation: W = res * P^-1 (the reduced accumulator)
            d0 = slot_ptr(P, w.W + i, LOGN) + tile0;
            d1 = slot_ptr(P, w.W + L + i, LOGN) + tile0;
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const u32 e = 2 * (threadIdx.x + k * NT);
                *reinterpret_cast<ulonglong2*>(d0 + e) = r0[k];
                *reinterpret_cast<ulonglong2*>(d1 + e) = r1[k];
            }
            continue;
        }
        const bool drop = i == L - 1;
        const u64 s1 = lv.s1r[i], s1p = lv.s1rp[i];
        d0 = drop ? slot_ptr(P, w.U, LOGN) + tile0 : slot_ptr(P, w.W + i, LOGN) + tile0;
        d1 = drop ? slot_ptr(P, w.U + 1, LOGN) + tile0 : slot_ptr(P, w.W + L + i, LOGN) + tile0;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const u32 e = 2 * (threadIdx.x + k * NT);
            ulonglong2 o0, o1;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                // u = t + res * P^-1 (eval, INTT'd in P6/P7); W = (t + res * P^-1) * s1
                const u64 ua = csub(v2get(t0[k], j) + v2get(r0[k], j), q);
                const u64 ub = csub(v2get(t1[k], j) + v2get(r1[k], j), q);
                v2set(o0, j, drop ? ua : shoup(ua, s1, s1p, q));
                v2set(o1, j, drop ? ub : shoup(ub, s1, s1p, q));
            }
            *reinterpret_cast<ulonglong2*>(d0 + e) = o0;
            *reinterpret_cast<ulonglong2*>(d1 + e) = o1;
        }
    }
}

// P5 on the FP64 pipe, for the key rows of Q towers with q < 2^50 (the
// integer forms above take P rows and 60-bit Q rows). The integer forms keep
// the FP64 pipe idle and are bound by integer issue; here every product
// digit * key is an exact FP64 modular product (FpArS::mulq: h, l by
// multiply and FMA, quotient by the magic-constant rounding, remainder by
// FMA) and the inner product is a plain FP64 sum of those remainders.
// Canonical quantities throughout, no Montgomery scale:
//   key tile: key_p * P^-1 mod q for every digit (the own digit's stored key
//     carries an extra R = 2^64 with DevCtx mont: one redc removes it on
//     load), as signed doubles in (-q/2, q/2];
//   own source: EvalMult a1 * b1, keyswitch input, rotation sigma_k(c1);
//   res' = sum_p src_p * key'_p = res * P^-1 (mod q);
//   EvalMult: W = (t + res') * s1 with t0 = a0 b0, t1 = a0 b1 + a1 b0; the
//     dropped tower gets (t + res') times R^-1 (one redc) with mont, the
//     scale the integer form writes for P7; keyswitch / rotation: W = res'.
// Bounds (q < 2^50, digits and inputs in [0, 2q), keys and s1 signed):
// every product |r| <= 0.75 q, the accumulator is normalised every eight
// digits (|acc| < 6.1 q < 2^53), t0 and t1 stay below 1.25 q, t + res' below
// 1.75 q + 1 before the final product, so every value is an exact integer
// below 2^53 and the canonical outputs equal the integer form's word for
// word.
// Two occupancy forms: PCH digits' loads in flight per batch and MINB CTAs
// per SM (4 digits / 4 CTAs at 128 registers, or 2 digits / 5 CTAs at 94).
constexpr int MACF_NT = 128;

template <int LOGN, int PCH, int MINB>
__global__ void __launch_bounds__(MACF_NT, MINB)
p5_mac_fp(const DevCtx D, const PairDesc* __restrict__ pairs, const uint4* __restrict__ jobs,
          const u32* __restrict__ plist) {
    constexpr int NT = MACF_NT;
    constexpr int TILES = (1 << LOGN) / MAC_TILE;
    constexpr int NV = MAC_TILE / (2 * NT);   // 16-byte vectors per thread
    extern __shared__ __align__(16) u64 sm[];     // [dnum][2][MAC_TILE] signed doubles
    double* smd = reinterpret_cast<double*>(sm);
    const uint4 jb = jobs[blockIdx.x / TILES];
    const u32 tile0 = (blockIdx.x % TILES) * MAC_TILE;
    const u32 r = jb.x;                           // a Q row (r < fullQ), q < 2^50
    const ModC m = D.mod[r];
    const u32 dnum = D.dnum;
    const double qd = ntt::u2d(m.q), hq = ntt::u2d(m.q >> 1);
    const ntt::FpArS ar{qd, qinv_of(m)};
    const u32 pin = r / D.alpha;                  // digit holding tower r
    auto sgn = [&](u64 x) {                       // canonical -> signed double in (-q/2, q/2]
        const double d = ntt::u2d(x);
        return d > hq ? __dsub_rn(d, qd) : d;
    };
    const PairDesc& P0 = pairs[plist[jb.y]];
    for (u32 k = threadIdx.x; k < dnum * MAC_TILE; k += NT) {
        const u32 p = k / MAC_TILE, e = k % MAC_TILE;
        const size_t off = (((size_t)p * D.QP + r) << LOGN) + tile0 + e;
        u64 kb = P0.kbv[off], ka = P0.kav[off];
        if (D.mont && p == pin) {
            kb = redc(kb, 0, m);
            ka = redc(ka, 0, m);
        }
        smd[(2 * p) * MAC_TILE + e] = sgn(kb);
        smd[(2 * p + 1) * MAC_TILE + e] = sgn(ka);
    }
    __syncthreads();
    const u64 q = m.q;
    auto canon = [&](double z) { return ar.out(ar.norm(z)); };   // |z| < 2^52 -> [0, q)
    for (u32 g = 0; g < jb.z; ++g) {
        const PairDesc& P = pairs[plist[jb.y + g]];
        const u32 L = P.L, K = D.K, QlP = L + K;
        const u32 i = r;                          // QlP position of a Q row
        const Level& lv = D.lvl[L];
        const WsLayout w = ws_layout(L, K, D.alpha);
        const u32 nparts = lv.nparts;
        const bool emr = P.mode == EMR;
        const size_t o = ((size_t)i << LOGN) + tile0;
        double s[2 * NV], t0[2 * NV], t1[2 * NV];
        if (emr) {
            ulonglong2 x0[NV], x1[NV], y0[NV], y1[NV];
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const u32 e = 2 * (threadIdx.x + k * NT);
                x0[k] = *reinterpret_cast<const ulonglong2*>(P.in[0] + o + e);
                x1[k] = *reinterpret_cast<const ulonglong2*>(P.in[1] + o + e);
                y0[k] = *reinterpret_cast<const ulonglong2*>(P.in[2] + o + e);
                y1[k] = *reinterpret_cast<const ulonglong2*>(P.in[3] + o + e);
            }
#pragma unroll
            for (int k = 0; k < NV; ++k)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const double a0 = ntt::u2d(v2get(x0[k], j)), a1 = ntt::u2d(v2get(x1[k], j));
                    const double b0 = sgn(v2get(y0[k], j)), b1 = sgn(v2get(y1[k], j));
                    s[2 * k + j] = ar.mulq<false>(a1, b1);
                    t0[2 * k + j] = ar.mulq<false>(a0, b0);
                    t1[2 * k + j] = __dadd_rn(ar.mulq<false>(a0, b1), ar.mulq<false>(a1, b0));
                }
        } else {
#pragma unroll
            for (int k = 0; k < NV; ++k)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const u32 e = tile0 + 2 * (threadIdx.x + k * NT) + j;
                    const u64 x = (P.mode == ROT || P.mode == HROT)
                                      ? P.in[1][((size_t)i << LOGN) + galois_slot<LOGN>(e, P.galois)]
                                      : P.in[0][((size_t)i << LOGN) + e];
                    s[2 * k + j] = ntt::u2d(x);
                }
        }
        double acc_b[2 * NV], acc_a[2 * NV];
#pragma unroll
        for (int k = 0; k < 2 * NV; ++k) acc_b[k] = acc_a[k] = 0.0;
        for (u32 p0 = 0; p0 < nparts; p0 += PCH) {
            ulonglong2 v[PCH][NV];
#pragma unroll
            for (int pp = 0; pp < PCH; ++pp) {
                const u32 p = p0 + pp;
                if (p < nparts && p != pin) {
                    const u64* Yt = P.ysrc + ((size_t)(w.Y + p * QlP + i) << LOGN);
                    if (P.mode == HROT) {   // sigma_k of the shared digit: eval-slot gather
#pragma unroll
                        for (int k = 0; k < NV; ++k)
#pragma unroll
                            for (int j = 0; j < 2; ++j)
                                v2set(v[pp][k], j,
                                      Yt[galois_slot<LOGN>(tile0 + 2 * (threadIdx.x + k * NT) + j, P.galois)]);
                    } else {
                        const ulonglong2* Y = reinterpret_cast<const ulonglong2*>(Yt + tile0);
#pragma unroll
                        for (int k = 0; k < NV; ++k) v[pp][k] = __ldcs(Y + threadIdx.x + k * NT);
                    }
                }
            }
#pragma unroll
            for (int pp = 0; pp < PCH; ++pp) {
                const u32 p = p0 + pp;
                if (p >= nparts) break;
                const double* kb = smd + (2 * p) * MAC_TILE;
                const double* ka = smd + (2 * p + 1) * MAC_TILE;
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    const u32 e = 2 * (threadIdx.x + k * NT);
                    const double2 kbv = *reinterpret_cast<const double2*>(kb + e);
                    const double2 kav = *reinterpret_cast<const double2*>(ka + e);
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const double y = p == pin ? s[2 * k + j] : ntt::u2d(v2get(v[pp][k], j));
                        acc_b[2 * k + j] = __dadd_rn(acc_b[2 * k + j], ar.mulq<false>(y, j ? kbv.y : kbv.x));
                        acc_a[2 * k + j] = __dadd_rn(acc_a[2 * k + j], ar.mulq<false>(y, j ? kav.y : kav.x));
                    }
                }
            }
            if ((p0 & 7u) == 4u) {   // after every eighth digit: keep |acc| below 2^53
#pragma unroll
                for (int k = 0; k < 2 * NV; ++k) {
                    acc_b[k] = ar.norm(acc_b[k]);
                    acc_a[k] = ar.norm(acc_a[k]);
                }
            }
        }
        u64 *d0, *d1;
        if (!emr) {   // keyswitch / rotation: W = res * P^-1
            d0 = slot_ptr(P, w.W + i, LOGN) + tile0;
            d1 = slot_ptr(P, w.W + L + i, LOGN) + tile0;
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const u32 e = 2 * (threadIdx.x + k * NT);
                *reinterpret_cast<ulonglong2*>(d0 + e) = make_ulonglong2(canon(acc_b[2 * k]), canon(acc_b[2 * k + 1]));
                *reinterpret_cast<ulonglong2*>(d1 + e) = make_ulonglong2(canon(acc_a[2 * k]), canon(acc_a[2 * k + 1]));
            }
            continue;
        }
        const bool drop = i == L - 1;
        const double s1 = sgn(lv.s1[i]);
        d0 = drop ? slot_ptr(P, w.U, LOGN) + tile0 : slot_ptr(P, w.W + i, LOGN) + tile0;
        d1 = drop ? slot_ptr(P, w.U + 1, LOGN) + tile0 : slot_ptr(P, w.W + L + i, LOGN) + tile0;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const u32 e = 2 * (threadIdx.x + k * NT);
            ulonglong2 o0, o1;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const double ua = __dadd_rn(t0[2 * k + j], ar.norm(acc_b[2 * k + j]));
                const double ub = __dadd_rn(t1[2 * k + j], ar.norm(acc_a[2 * k + j]));
                u64 wa, wb;
                if (drop) {   // U: the integer form's scale, (t + res') * R^-1 with mont
                    wa = canon(ua);
                    wb = canon(ub);
                    if (D.mont) {
                        wa = redc(wa, 0, m);
                        wb = redc(wb, 0, m);
                    }
                } else {
                    wa = canon(ar.mulq<true>(ua, s1));
                    wb = canon(ar.mulq<true>(ub, s1));
                }
                v2set(o0, j, wa);
                v2set(o1, j, wb);
            }
            *reinterpret_cast<ulonglong2*>(d0 + e) = o0;
            *reinterpret_cast<ulonglong2*>(d1 + e) = o1;
        }
    }
    (void)q;
}

// P5, pipelined form (dnum small enough for the staging buffers): 256
// threads, each owning one 16-byte pair of the 512-element tile. While a
// pair is multiplied, the tiles of the next pair (the four tensor inputs or
// the keyswitch input, and every other digit of tower i) are already in
// flight into the other shared-memory stage with cp.async; each thread copies
// and later reads only its own 16 bytes, so the stages need no barrier.
// Results equal p5_mac's word for word.
constexpr int MACA_NT = 256;
constexpr int MACA_IN = 4;   // stage slots for tensor / keyswitch inputs
__host__ __device__ constexpr int maca_slots(int dnum) { return MACA_IN + dnum; }
__host__ __device__ constexpr int maca_smem(int dnum) {
    return (2 * dnum + 2 * maca_slots(dnum)) * MAC_TILE * 8;
}

__device__ __forceinline__ void cp_async16(u64* smem, const u64* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(u64* smem, const u64* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int LOGN>
__global__ void __launch_bounds__(MACA_NT)
p5_mac_async(const DevCtx D, const PairDesc* __restrict__ pairs, const uint4* __restrict__ jobs,
             const u32* __restrict__ plist) {
    constexpr int TILES = (1 << LOGN) / MAC_TILE;
    extern __shared__ __align__(16) u64 sm[];   // key [dnum][2][TILE] | stage [2][slots][TILE]
    const uint4 jb = jobs[blockIdx.x / TILES];
    const u32 tile0 = (blockIdx.x % TILES) * MAC_TILE;
    const u32 r = jb.x;
    const ModC m = D.mod[r];
    const u32 dnum = D.dnum, slots = maca_slots((int)dnum);
    u64* stage = sm + 2 * dnum * MAC_TILE;
    const PairDesc& P0 = pairs[plist[jb.y]];
    for (u32 k = threadIdx.x; k < dnum * (MAC_TILE / 2); k += MACA_NT) {
        const u32 p = k / (MAC_TILE / 2), e = 2 * (k % (MAC_TILE / 2));
        const size_t off = (((size_t)p * D.QP + r) << LOGN) + tile0 + e;
        *reinterpret_cast<ulonglong2*>(sm + (2 * p) * MAC_TILE + e) = ld2(P0.kbv + off);
        *reinterpret_cast<ulonglong2*>(sm + (2 * p + 1) * MAC_TILE + e) = ld2(P0.kav + off);
    }
    __syncthreads();
    const bool is_p = r >= D.fullQ;
    const u32 e = 2 * threadIdx.x;               // this thread's pair within the tile
    const u32 K = D.K;
    // queue the copies of pair g into stage buffer b (one commit group per pair)
    auto issue = [&](u32 g, int b) {
        const PairDesc& P = pairs[plist[jb.y + g]];
        const u32 L = P.L, QlP = L + K;
        const u32 i = is_p ? L + (r - D.fullQ) : r;
        const u32 pin = is_p ? 0xffffffffu : i / D.alpha;
        const WsLayout w = ws_layout(L, K, D.alpha);
        u64* sb = stage + (size_t)b * slots * MAC_TILE + e;
        const size_t o = ((size_t)i << LOGN) + tile0 + e;
        if (!is_p) {
            if (P.mode == EMR) {
#pragma unroll
                for (int k = 0; k < 4; ++k) cp_async16(sb + k * MAC_TILE, P.in[k] + o);
            } else if (P.mode == KS) {
                cp_async16(sb + MAC_TILE, P.in[0] + o);
            }
        }
        const u32 nparts = D.lvl[L].nparts;
        for (u32 p = 0; p < nparts; ++p) {
            if (p == pin) continue;
            const u64* Yt = P.ysrc + ((size_t)(w.Y + p * QlP + i) << LOGN);
            if (P.mode == HROT) {   // sigma_k of the shared digit: two 8-byte gathers
#pragma unroll
                for (int j = 0; j < 2; ++j)
                    cp_async8(sb + (MACA_IN + p) * MAC_TILE + j, Yt + galois_slot<LOGN>(tile0 + e + j, P.galois));
            } else {
                cp_async16(sb + (MACA_IN + p) * MAC_TILE, Yt + tile0 + e);
            }
        }
        cp_async_commit();
    };
    issue(0, 0);
    for (u32 g = 0; g < jb.z; ++g) {
        if (g + 1 < jb.z) issue(g + 1, (int)((g + 1) & 1));
        else cp_async_commit();                  // empty group keeps the wait count uniform
        cp_async_wait1();                        // pair g's copies have landed
        const PairDesc& P = pairs[plist[jb.y + g]];
        const u32 L = P.L;
        const u32 i = is_p ? L + (r - D.fullQ) : r;
        const Level& lv = D.lvl[L];
        const WsLayout w = ws_layout(L, K, D.alpha);
        const u32 nparts = lv.nparts;
        const u32 pin = is_p ? 0xffffffffu : i / D.alpha;
        const bool emr = P.mode == EMR;
        const u64* sb = stage + (size_t)(g & 1) * slots * MAC_TILE + e;
        ulonglong2 s{0, 0}, t0{0, 0}, t1{0, 0};
        if (!is_p) {
            if (emr) {
                const ulonglong2 x0 = ld2(sb), x1 = ld2(sb + MAC_TILE);
                const ulonglong2 y0 = ld2(sb + 2 * MAC_TILE), y1 = ld2(sb + 3 * MAC_TILE);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const u64 a0 = v2get(x0, j), a1 = v2get(x1, j), b0 = v2get(y0, j), b1 = v2get(y1, j);
                    u64 lo, hi;
                    mul_wide(a1, b1, lo, hi);
                    v2set(s, j, acc_reduce(lo, hi, m, D.mont));
                    mul_wide(a0, b0, lo, hi);
                    v2set(t0, j, acc_reduce(lo, hi, m, D.mont));
                    mul_wide(a0, b1, lo, hi);
                    mac_wide(lo, hi, a1, b0);
                    v2set(t1, j, acc_reduce(lo, hi, m, D.mont));
                }
            } else {
                if (P.mode == ROT || P.mode == HROT) {
                    const u64* src = P.in[1] + ((size_t)i << LOGN);
#pragma unroll
                    for (int j = 0; j < 2; ++j) v2set(s, j, src[galois_slot<LOGN>(tile0 + e + j, P.galois)]);
                } else {
                    s = ld2(sb + MAC_TILE);
                }
                if (D.mont) {
#pragma unroll
                    for (int j = 0; j < 2; ++j) v2set(s, j, redc(v2get(s, j), 0, m));
                }
            }
        }
        u64 a0l[2] = {0, 0}, a0h[2] = {0, 0}, a1l[2] = {0, 0}, a1h[2] = {0, 0};
        for (u32 p = 0; p < nparts; ++p) {
            const ulonglong2 dv = p == pin ? s : ld2(sb + (MACA_IN + p) * MAC_TILE);
            const ulonglong2 kbv = ld2(sm + (2 * p) * MAC_TILE + e);
            const ulonglong2 kav = ld2(sm + (2 * p + 1) * MAC_TILE + e);
            mac_wide(a0l[0], a0h[0], dv.x, kbv.x);
            mac_wide(a0l[1], a0h[1], dv.y, kbv.y);
            mac_wide(a1l[0], a1h[0], dv.x, kav.x);
            mac_wide(a1l[1], a1h[1], dv.y, kav.y);
        }
        const u32 use_redc = D.mont && (is_p || emr);
        ulonglong2 r0, r1;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            v2set(r0, j, acc_reduce(a0l[j], a0h[j], m, use_redc));
            v2set(r1, j, acc_reduce(a1l[j], a1h[j], m, use_redc));
        }
        const u64 q = m.q;
        if (is_p) {
            *reinterpret_cast<ulonglong2*>(slot_ptr(P, w.RP + (i - L), LOGN) + tile0 + e) = r0;
            *reinterpret_cast<ulonglong2*>(slot_ptr(P, w.RP + K + (i - L), LOGN) + tile0 + e) = r1;
            continue;
        }
        ulonglong2 o0, o1;
        u64 *d0, *d1;
        if (!emr) {   // keyswitch / rotation: W = res * P^-1 (the reduced accumulator)
            d0 = slot_ptr(P, w.W + i, LOGN);
            d1 = slot_ptr(P, w.W + L + i, LOGN);
            o0 = r0;
            o1 = r1;
        } else {
            const bool drop = i == L - 1;
            const u64 s1 = lv.s1r[i], s1p = lv.s1rp[i];
            d0 = drop ? slot_ptr(P, w.U, LOGN) : slot_ptr(P, w.W + i, LOGN);
            d1 = drop ? slot_ptr(P, w.U + 1, LOGN) : slot_ptr(P, w.W + L + i, LOGN);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const u64 ua = csub(v2get(t0, j) + v2get(r0, j), q);
                const u64 ub = csub(v2get(t1, j) + v2get(r1, j), q);
                v2set(o0, j, drop ? ua : shoup(ua, s1, s1p, q));
                v2set(o1, j, drop ? ub : shoup(ub, s1, s1p, q));
            }
        }
        *reinterpret_cast<ulonglong2*>(d0 + tile0 + e) = o0;
        *reinterpret_cast<ulonglong2*>(d1 + tile0 + e) = o1;
    }
}

// P5, TMA form. One producer thread streams every pair's tiles (the four
// tensor inputs or the keyswitch input, and each other digit of tower i: rows
// of P5T_TILE contiguous words) into a ring of P5T_STAGES shared-memory stages
// with cp.async.bulk; each stage completes on its own mbarrier by transaction
// count. P5T_NC consumer threads own one 16-byte pair of the tile each,
// release a stage by arriving on its empty mbarrier as soon as they hold its
// words in registers, and then write the epilogue. The key tile of row r
// arrives the same way, once per CTA. Hoisted-rotation digits (an eval-slot
// gather) and the rotation source are read by the consumers directly.
// Every wait is bounded in time (mbar_wait): when one expires the thread ORs
// a code into D.err and leaves, and the producer waits (bounded again) for
// its copies in flight to land before it leaves, so no copy outlives the CTA.
// A CTA that starts with D.err set leaves before issuing anything.
// Results equal p5_mac's word for word.
constexpr int P5T_TILE = 256;
constexpr int P5T_NC = P5T_TILE / 2;        // consumer threads
constexpr int P5T_NT = P5T_NC + 32;         // + one producer warp
constexpr int P5T_STAGES = 3;
constexpr int P5T_BAR_WORDS = 16;           // mbarriers: key, full[S], empty[S] (padded)
static_assert(1 + 2 * P5T_STAGES <= P5T_BAR_WORDS, "mbarrier area");
__host__ __device__ constexpr int p5t_smem(int dnum, int stages = P5T_STAGES, bool compact = false) {
    return (P5T_BAR_WORDS + (2 * dnum + stages * (maca_slots(dnum) - (compact ? 1 : 0))) * P5T_TILE) * 8;
}

__device__ __forceinline__ u32 smem_addr(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u32 bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(u32 bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(u32 bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_test(u32 bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ u64 global_ns() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase of `bar` with parity `parity` to complete; false once
// about two seconds have passed without it.
__device__ __forceinline__ bool mbar_wait(u32 bar, u32 parity) {
    if (mbar_test(bar, parity)) return true;
    const u64 t0 = global_ns();
    for (u32 k = 1;; ++k) {
        if (mbar_test(bar, parity)) return true;
        if ((k & 63) == 0 && global_ns() - t0 > 2000000000ull) return false;
    }
}
// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing on mbarrier `bar`.
__device__ __forceinline__ void bulk_load(u32 dst, const void* src, u32 bytes, u32 bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Ring of the TMA forms: mbarriers at the start of dynamic shared memory
// (key, full[S], empty[S]), then the key tile [dnum][2][P5T_TILE], then
// S stages of `slots` rows: MACA_IN input rows, then a row per digit. A
// compact ring (Q rows only) leaves out the row of the digit that holds the
// tower itself, which is never copied.
template <int S>
struct P5Ring {
    u64* keys;
    u64* stage;
    u32 kbar;
    u32 slots;
    bool compact;
    __device__ __forceinline__ u32 slot(u32 p, u32 pin) const { return MACA_IN + p - (compact && p > pin ? 1u : 0u); }
    __device__ __forceinline__ u32 full(u32 b) const { return kbar + 8 * (1 + b); }
    __device__ __forceinline__ u32 empty(u32 b) const { return kbar + 8 * (1 + S + b); }
};

// Thread 0 initialises the mbarriers; every thread learns whether an earlier
// CTA's wait expired (then the CTA leaves before issuing anything).
template <int S>
__device__ __forceinline__ bool p5t_setup(const DevCtx& D, u64* sm, P5Ring<S>& R, bool compact = false) {
    static_assert(1 + 2 * S <= P5T_BAR_WORDS, "mbarrier area");
    __shared__ u32 failed;
    R.compact = compact;
    R.slots = (u32)maca_slots((int)D.dnum) - (compact ? 1u : 0u);
    R.keys = sm + P5T_BAR_WORDS;
    R.stage = R.keys + 2 * D.dnum * P5T_TILE;
    R.kbar = smem_addr(sm);
    if (threadIdx.x == 0) {
        failed = *reinterpret_cast<volatile u32*>(D.err);
        mbar_init(R.kbar, 1);
        for (u32 b = 0; b < (u32)S; ++b) {
            mbar_init(R.full(b), 1);
            mbar_init(R.empty(b), P5T_NC);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();                            // the only CTA-wide barrier
    return failed == 0;
}

// The producer (one thread): the key tile of row r once, then per listed
// pair the tensor inputs (EvalMult+Rescale, slots 0-3) or the keyswitch input
// (slot 1) of a Q row and every other digit of its tower (slot MACA_IN + p),
// into stage g % S after the consumers have released it; finally it waits
// (bounded) for every copy in flight.
template <int LOGN, int S>
__device__ __forceinline__ void p5t_produce(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint4 jb,
                                            const u32* __restrict__ plist, const u32 tile0, const P5Ring<S>& R) {
    constexpr u32 ROW = P5T_TILE * 8;           // bytes of one staged row
    const u32 r = jb.x, dnum = D.dnum, slots = R.slots, K = D.K;
    const bool is_p = r >= D.fullQ;
    const PairDesc& P0 = pairs[plist[jb.y]];
    mbar_arrive_expect_tx(R.kbar, 2 * dnum * ROW);
    for (u32 p = 0; p < dnum; ++p) {
        const size_t off = (((size_t)p * D.QP + r) << LOGN) + tile0;
        bulk_load(smem_addr(R.keys + (2 * p) * P5T_TILE), P0.kbv + off, ROW, R.kbar);
        bulk_load(smem_addr(R.keys + (2 * p + 1) * P5T_TILE), P0.kav + off, ROW, R.kbar);
    }
    u32 issued = 0;
    for (u32 g = 0; g < jb.z; ++g) {
        const u32 b = g % S;
        if (g >= S && !mbar_wait(R.empty(b), (g / S - 1) & 1)) {
            atomicOr(D.err, 4u);
            break;
        }
        const PairDesc& P = pairs[plist[jb.y + g]];
        const u32 L = P.L, QlP = L + K;
        const u32 i = is_p ? L + (r - D.fullQ) : r;
        const u32 pin = is_p ? 0xffffffffu : i / D.alpha;
        const WsLayout w = ws_layout(L, K, D.alpha);
        const u32 nparts = D.lvl[L].nparts;
        const u32 nin = is_p ? 0u : (P.mode == EMR ? 4u : (P.mode == KS ? 1u : 0u));
        const u32 ndig = P.mode == HROT ? 0u : nparts - (pin < nparts ? 1u : 0u);
        u64* sb = R.stage + (size_t)b * slots * P5T_TILE;
        const size_t o = ((size_t)i << LOGN) + tile0;
        mbar_arrive_expect_tx(R.full(b), (nin + ndig) * ROW);
        if (nin == 4) {
            for (u32 k = 0; k < 4; ++k) bulk_load(smem_addr(sb + k * P5T_TILE), P.in[k] + o, ROW, R.full(b));
        } else if (nin == 1) {
            bulk_load(smem_addr(sb + P5T_TILE), P.in[0] + o, ROW, R.full(b));
        }
        if (ndig)
            for (u32 p = 0; p < nparts; ++p) {
                if (p == pin) continue;
                const u64* Yt = P.ysrc + ((size_t)(w.Y + p * QlP + i) << LOGN) + tile0;
                bulk_load(smem_addr(sb + R.slot(p, pin) * P5T_TILE), Yt, ROW, R.full(b));
            }
        issued = g + 1;
    }
    // every issued stage's copies must land before this thread leaves
    const u32 first = issued > (u32)S ? issued - S : 0u;
    for (u32 g = first; g < issued; ++g)
        if (!mbar_wait(R.full(g % S), (g / S) & 1)) atomicOr(D.err, 4u);
    if (!mbar_wait(R.kbar, 0)) atomicOr(D.err, 1u);
}

// Consumer of the TMA forms for an integer key row (a P row, or a Q row of
// any width): p5_mac's arithmetic on one 16-byte pair of the tile per thread.
template <int LOGN, int S>
__device__ __forceinline__ void p5t_consume_int(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint4 jb,
                                                const u32* __restrict__ plist, const u32 tile0, const P5Ring<S>& R) {
    const u32 r = jb.x, slots = R.slots;
    const bool is_p = r >= D.fullQ;
    const u32 K = D.K;
    const u32 e = 2 * threadIdx.x;              // this thread's pair within the tile
    const ModC m = D.mod[r];
    if (!mbar_wait(R.kbar, 0)) {
        atomicOr(D.err, 1u);
        return;
    }
    for (u32 g = 0; g < jb.z; ++g) {
        const u32 b = g % S;
        if (!mbar_wait(R.full(b), (g / S) & 1)) {
            atomicOr(D.err, 2u);
            return;
        }
        const PairDesc& P = pairs[plist[jb.y + g]];
        const u32 L = P.L, QlP = L + K;
        const u32 i = is_p ? L + (r - D.fullQ) : r;
        const Level& lv = D.lvl[L];
        const WsLayout w = ws_layout(L, K, D.alpha);
        const u32 nparts = lv.nparts;
        const u32 pin = is_p ? 0xffffffffu : i / D.alpha;
        const bool emr = P.mode == EMR;
        const u64* sb = R.stage + (size_t)b * slots * P5T_TILE + e;
        ulonglong2 s{0, 0}, t0{0, 0}, t1{0, 0};
        if (!is_p) {
            if (emr) {
                const ulonglong2 x0 = ld2(sb), x1 = ld2(sb + P5T_TILE);
                const ulonglong2 y0 = ld2(sb + 2 * P5T_TILE), y1 = ld2(sb + 3 * P5T_TILE);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const u64 a0 = v2get(x0, j), a1 = v2get(x1, j), b0 = v2get(y0, j), b1 = v2get(y1, j);
                    u64 lo, hi;
                    mul_wide(a1, b1, lo, hi);
                    v2set(s, j, acc_reduce(lo, hi, m, D.mont));
                    mul_wide(a0, b0, lo, hi);
                    v2set(t0, j, acc_reduce(lo, hi, m, D.mont));
                    mul_wide(a0, b1, lo, hi);
                    mac_wide(lo, hi, a1, b0);
                    v2set(t1, j, acc_reduce(lo, hi, m, D.mont));
                }
            } else {
                if (P.mode == ROT || P.mode == HROT) {
                    const u64* src = P.in[1] + ((size_t)i << LOGN);
#pragma unroll
                    for (int j = 0; j < 2; ++j) v2set(s, j, src[galois_slot<LOGN>(tile0 + e + j, P.galois)]);
                } else {
                    s = ld2(sb + P5T_TILE);
                }
                if (D.mont) {
#pragma unroll
                    for (int j = 0; j < 2; ++j) v2set(s, j, redc(v2get(s, j), 0, m));
                }
            }
        }
        u64 a0l[2] = {0, 0}, a0h[2] = {0, 0}, a1l[2] = {0, 0}, a1h[2] = {0, 0};
        for (u32 p = 0; p < nparts; ++p) {
            ulonglong2 dv;
            if (p == pin) {
                dv = s;
            } else if (P.mode == HROT) {            // sigma_k of the shared digit: eval-slot gather
                const u64* Yt = P.ysrc + ((size_t)(w.Y + p * QlP + i) << LOGN);
#pragma unroll
                for (int j = 0; j < 2; ++j) v2set(dv, j, Yt[galois_slot<LOGN>(tile0 + e + j, P.galois)]);
            } else {
                dv = ld2(sb + R.slot(p, pin) * P5T_TILE);
            }
            const ulonglong2 kbv = ld2(R.keys + (2 * p) * P5T_TILE + e);
            const ulonglong2 kav = ld2(R.keys + (2 * p + 1) * P5T_TILE + e);
            mac_wide(a0l[0], a0h[0], dv.x, kbv.x);
            mac_wide(a0l[1], a0h[1], dv.y, kbv.y);
            mac_wide(a1l[0], a1h[0], dv.x, kav.x);
            mac_wide(a1l[1], a1h[1], dv.y, kav.y);
        }
        mbar_arrive(R.empty(b));                  // every word of stage b is in registers
        const u32 use_redc = D.mont && (is_p || emr);
        ulonglong2 r0, r1;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            v2set(r0, j, acc_reduce(a0l[j], a0h[j], m, use_redc));
            v2set(r1, j, acc_reduce(a1l[j], a1h[j], m, use_redc));
        }
        const u64 q = m.q;
        if (is_p) {
            *reinterpret_cast<ulonglong2*>(slot_ptr(P, w.RP + (i - L), LOGN) + tile0 + e) = r0;
            *reinterpret_cast<ulonglong2*>(slot_ptr(P, w.RP + K + (i - L), LOGN) + tile0 + e) = r1;
            continue;
        }
        ulonglong2 o0, o1;
        u64 *d0, *d1;
        if (!emr) {   // keyswitch / rotation: W = res * P^-1 (the reduced accumulator)
            d0 = slot_ptr(P, w.W + i, LOGN);
            d1 = slot_ptr(P, w.W + L + i, LOGN);
            o0 = r0;
            o1 = r1;
        } else {
            const bool drop = i == L - 1;
            const u64 s1 = lv.s1r[i], s1p = lv.s1rp[i];
            d0 = drop ? slot_ptr(P, w.U, LOGN) : slot_ptr(P, w.W + i, LOGN);
            d1 = drop ? slot_ptr(P, w.U + 1, LOGN) : slot_ptr(P, w.W + L + i, LOGN);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const u64 ua = csub(v2get(t0, j) + v2get(r0, j), q);
                const u64 ub = csub(v2get(t1, j) + v2get(r1, j), q);
                v2set(o0, j, drop ? ua : shoup(ua, s1, s1p, q));
                v2set(o1, j, drop ? ub : shoup(ub, s1, s1p, q));
            }
        }
        *reinterpret_cast<ulonglong2*>(d0 + tile0 + e) = o0;
        *reinterpret_cast<ulonglong2*>(d1 + tile0 + e) = o1;
    }
}

template <int LOGN>
__global__ void __launch_bounds__(P5T_NT)
p5_mac_tma(const DevCtx D, const PairDesc* __restrict__ pairs, const uint4* __restrict__ jobs,
           const u32* __restrict__ plist) {
    constexpr int TILES = (1 << LOGN) / P5T_TILE;
    extern __shared__ __align__(128) u64 sm[];  // mbarriers | key [dnum][2][TILE] | stage [S][slots][TILE]
    const uint4 jb = jobs[blockIdx.x / TILES];
    const u32 tile0 = (blockIdx.x % TILES) * P5T_TILE;
    P5Ring<P5T_STAGES> R;
    if (!p5t_setup(D, sm, R)) return;
    if (threadIdx.x >= P5T_NC) {                // producer warp: lane 0 issues every copy
        if (threadIdx.x == P5T_NC) p5t_produce<LOGN>(D, pairs, jb, plist, tile0, R);
        return;
    }
    p5t_consume_int<LOGN>(D, pairs, jb, plist, tile0, R);
}

// Consumer of the TMA forms for an FP64 key row (P5 on the FP64 pipe, TMA
// form, the kernel below): p5_mac_tma's ring (the same producer,
// bounded waits and error codes) with p5_mac_fp's arithmetic in the
// consumers, for the key rows of Q towers with q < 2^50. The key tile lands
// as stored words; each consumer turns its own two words of every key row
// into signed doubles in place (a Montgomery reduction first for the own
// digit's key under DevCtx mont), so no barrier is needed. The bounds are
// p5_mac_fp's: products |r| <= 0.75 q, the sums normalised after every
// eighth digit, every value an exact integer below 2^53. Results equal
// p5_mac's word for word.
template <int LOGN, int S>
__device__ __forceinline__ void p5t_consume_fp(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint4 jb,
                                               const u32* __restrict__ plist, const u32 tile0, const P5Ring<S>& R) {
    const u32 r = jb.x, dnum = D.dnum, slots = R.slots;   // a Q row, q < 2^50
    const u32 e = 2 * threadIdx.x;              // this thread's pair within the tile
    const u32 K = D.K, pin = r / D.alpha;       // digit holding tower r
    const ModC m = D.mod[r];
    const double qd = ntt::u2d(m.q), hq = ntt::u2d(m.q >> 1);
    const ntt::FpArS ar{qd, qinv_of(m)};
    auto sgn = [&](u64 x) {                     // canonical -> signed double in (-q/2, q/2]
        const double d = ntt::u2d(x);
        return d > hq ? __dsub_rn(d, qd) : d;
    };
    auto canon = [&](double z) { return ar.out(ar.norm(z)); };   // |z| < 2^52 -> [0, q)
    if (!mbar_wait(R.kbar, 0)) {
        atomicOr(D.err, 1u);
        return;
    }
    for (u32 p = 0; p < 2 * dnum; ++p) {        // own words of key row p / 2 (b, then a) -> doubles
        u64* kw = R.keys + p * P5T_TILE + e;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            u64 k = kw[j];
            if (D.mont && p / 2 == pin) k = redc(k, 0, m);
            kw[j] = (u64)__double_as_longlong(sgn(k));
        }
    }
    const double* kd = reinterpret_cast<const double*>(R.keys);
    for (u32 g = 0; g < jb.z; ++g) {
        const u32 b = g % S;
        if (!mbar_wait(R.full(b), (g / S) & 1)) {
            atomicOr(D.err, 2u);
            return;
        }
        const PairDesc& P = pairs[plist[jb.y + g]];
        const u32 L = P.L, QlP = L + K;
        const u32 i = r;                        // QlP position of a Q row
        const Level& lv = D.lvl[L];
        const WsLayout w = ws_layout(L, K, D.alpha);
        const u32 nparts = lv.nparts;
        const bool emr = P.mode == EMR;
        const u64* sb = R.stage + (size_t)b * slots * P5T_TILE + e;
        double s[2], t0[2] = {0.0, 0.0}, t1[2] = {0.0, 0.0};
        if (emr) {
            const ulonglong2 x0 = ld2(sb), x1 = ld2(sb + P5T_TILE);
            const ulonglong2 y0 = ld2(sb + 2 * P5T_TILE), y1 = ld2(sb + 3 * P5T_TILE);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const double a0 = ntt::u2d(v2get(x0, j)), a1 = ntt::u2d(v2get(x1, j));
                const double b0 = sgn(v2get(y0, j)), b1 = sgn(v2get(y1, j));
                s[j] = ar.mulq<false>(a1, b1);
                t0[j] = ar.mulq<false>(a0, b0);
                t1[j] = __dadd_rn(ar.mulq<false>(a0, b1), ar.mulq<false>(a1, b0));
            }
        } else if (P.mode == ROT || P.mode == HROT) {
            const u64* src = P.in[1] + ((size_t)i << LOGN);
#pragma unroll
            for (int j = 0; j < 2; ++j) s[j] = ntt::u2d(src[galois_slot<LOGN>(tile0 + e + j, P.galois)]);
        } else {
            const ulonglong2 x = ld2(sb + P5T_TILE);
            s[0] = ntt::u2d(x.x);
            s[1] = ntt::u2d(x.y);
        }
        double acc_b[2] = {0.0, 0.0}, acc_a[2] = {0.0, 0.0};
        for (u32 p = 0; p < nparts; ++p) {
            double y[2];
            if (p == pin) {
                y[0] = s[0];
                y[1] = s[1];
            } else if (P.mode == HROT) {        // sigma_k of the shared digit: eval-slot gather
                const u64* Yt = P.ysrc + ((size_t)(w.Y + p * QlP + i) << LOGN);
#pragma unroll
                for (int j = 0; j < 2; ++j) y[j] = ntt::u2d(Yt[galois_slot<LOGN>(tile0 + e + j, P.galois)]);
            } else {
                const ulonglong2 dv = ld2(sb + R.slot(p, pin) * P5T_TILE);
                y[0] = ntt::u2d(dv.x);
                y[1] = ntt::u2d(dv.y);
            }
            const double2 kbv = *reinterpret_cast<const double2*>(kd + (2 * p) * P5T_TILE + e);
            const double2 kav = *reinterpret_cast<const double2*>(kd + (2 * p + 1) * P5T_TILE + e);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                acc_b[j] = __dadd_rn(acc_b[j], ar.mulq<false>(y[j], j ? kbv.y : kbv.x));
                acc_a[j] = __dadd_rn(acc_a[j], ar.mulq<false>(y[j], j ? kav.y : kav.x));
            }
            if ((p & 7u) == 7u) {               // after every eighth digit: keep |acc| below 2^53
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    acc_b[j] = ar.norm(acc_b[j]);
                    acc_a[j] = ar.norm(acc_a[j]);
                }
            }
        }
        mbar_arrive(R.empty(b));                // every word of stage b is in registers
        ulonglong2 o0, o1;
        u64 *d0, *d1;
        if (!emr) {   // keyswitch / rotation: W = res * P^-1
            d0 = slot_ptr(P, w.W + i, LOGN);
            d1 = slot_ptr(P, w.W + L + i, LOGN);
            o0 = make_ulonglong2(canon(acc_b[0]), canon(acc_b[1]));
            o1 = make_ulonglong2(canon(acc_a[0]), canon(acc_a[1]));
        } else {
            const bool drop = i == L - 1;
            const double s1 = sgn(lv.s1[i]);
            d0 = drop ? slot_ptr(P, w.U, LOGN) : slot_ptr(P, w.W + i, LOGN);
            d1 = drop ? slot_ptr(P, w.U + 1, LOGN) : slot_ptr(P, w.W + L + i, LOGN);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const double ua = __dadd_rn(t0[j], ar.norm(acc_b[j]));
                const double ub = __dadd_rn(t1[j], ar.norm(acc_a[j]));
                u64 wa, wb;
                if (drop) {   // U: the integer form's scale, (t + res') * R^-1 with mont
                    wa = canon(ua);
                    wb = canon(ub);
                    if (D.mont) {
                        wa = redc(wa, 0, m);
                        wb = redc(wb, 0, m);
                    }
                } else {
                    wa = canon(ar.mulq<true>(ua, s1));
                    wb = canon(ar.mulq<true>(ub, s1));
                }
                v2set(o0, j, wa);
                v2set(o1, j, wb);
            }
        }
        *reinterpret_cast<ulonglong2*>(d0 + tile0 + e) = o0;
        *reinterpret_cast<ulonglong2*>(d1 + tile0 + e) = o1;
    }
}

// S = 3 stages (65.7 KB at dnum 4, three CTAs per SM), or 2 stages in the
// compact ring (44.1 KB, five CTAs per SM at up to 81 registers).
template <int LOGN, int S>
__global__ void __launch_bounds__(P5T_NT, S == 2 ? 5 : 3)
p5_mac_fp_tma(const DevCtx D, const PairDesc* __restrict__ pairs, const uint4* __restrict__ jobs,
              const u32* __restrict__ plist) {
    constexpr int TILES = (1 << LOGN) / P5T_TILE;
    extern __shared__ __align__(128) u64 sm[];  // mbarriers | key [dnum][2][TILE] | stage [S][slots][TILE]
    const uint4 jb = jobs[blockIdx.x / TILES];
    const u32 tile0 = (blockIdx.x % TILES) * P5T_TILE;
    P5Ring<S> R;
    if (!p5t_setup(D, sm, R, S == 2)) return;
    if (threadIdx.x >= P5T_NC) {                // producer warp: lane 0 issues every copy
        if (threadIdx.x == P5T_NC) p5t_produce<LOGN>(D, pairs, jb, plist, tile0, R);
        return;
    }
    p5t_consume_fp<LOGN>(D, pairs, jb, plist, tile0, R);
}

// ------------------------------------------------------------------ P6
// INTT row stages of U[c] (t = 0, EvalMult+Rescale only) and RP[c][t-1].
template <int LOGN, bool FP>
__device__ __forceinline__ void p6_moddown_inv_row_body(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint2 jb,
                                              const u32 tile) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const u32 R0 = tile * G::RB;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K;
    const u32 c = jb.y / (K + 1), t = jb.y % (K + 1);
    const WsLayout w = ws_layout(L, K, D.alpha);
    const u32 qp = t == 0 ? L - 1 : D.fullQ + t - 1;
    const u32 slot = t == 0 ? w.U + c : w.RP + c * K + (t - 1);
    const ModC m = D.mod[qp];
    const auto ar = ar_of<FP>(m);
    u64* X = slot_ptr(P, slot, LOGN) + (size_t)R0 * 256;
    ntt::row_tile_stage<G::RB, G::ROW_THREADS>(
        [&](int rl, int cc) { return X[rl * 256 + cc]; },
        [&](int rl, int cc, u64 v) { sm[rl * G::ROW_STRIDE + ntt::rowpad(cc)] = ar.stage_in(v); });
    __syncthreads();
    auto st = [&](int rl, int cc, u64 v) { X[rl * 256 + cc] = v; };
    ntt::inv_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 8, true>(sm, twi_of<FP>(D, qp, LOGN), R0, ar, st);
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS, 4)
p6_moddown_inv_row(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::ROW_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::ROW_TILES;
    on_path<PATH>(jb, [&](auto fp) { p6_moddown_inv_row_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

// ------------------------------------------------------------------ P7
// Two launches. P7a (pair, c, t >= 1): INTT columns of P tower t-1 of RP[c],
// scaled by n^-1 * PHatInv. P7b (pair, c), EvalMult+Rescale only, after P7a:
// INTT columns of U[c] scaled by n^-1 (times R: U carries R^-1 from P5, see
// Key), then r_l = u - conv'_l * P^-1 mod q_l into U[c], with the P->q_l
// constants folding P^-1 (and 2^64 for a Montgomery reduction when
// D.mont_down). Both read P6's output in the path's own word format.
template <int LOGN, bool FP>
__device__ __forceinline__ void p7a_moddown_inv_col_body(const DevCtx& D, const PairDesc* __restrict__ pairs,
                                                         const uint2 jb, const u32 tile) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const int c0 = tile * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K;
    const u32 c = jb.y / (K + 1), t = jb.y % (K + 1);
    const WsLayout w = ws_layout(L, K, D.alpha);
    const u32 qp = D.fullQ + t - 1;
    const ModC m = D.mod[qp];
    const u64 sc = D.pdn[t - 1], scp = D.pdnp[t - 1];
    u64* X = slot_ptr(P, w.RP + c * K + (t - 1), LOGN) + c0;
    auto ld = [&](int r, int cl) { return X[r * 256 + cl]; };
    auto st = [&](int r, int cl, u64 v) { X[r * 256 + cl] = shoup(v, sc, scp, m.q); };
    ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A, true>(sm, twi_of<FP>(D, qp, LOGN), ar_of<FP>(m), ld, st);
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
p7a_moddown_inv_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::COL_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::COL_TILES;
    on_path<PATH>(jb, [&](auto fp) { p7a_moddown_inv_col_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

template <int LOGN, bool FP>
__device__ __forceinline__ void p7b_moddown_inv_col_body(const DevCtx& D, const PairDesc* __restrict__ pairs,
                                                         const uint2 jb, const u32 tile) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    __shared__ u64 cl_[gfx::MAXP];
    const int c0 = tile * G::C;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K, c = jb.y / (K + 1), l = L - 1;
    const WsLayout w = ws_layout(L, K, D.alpha);
    const ModC m = D.mod[l];
    if (threadIdx.x < K) {   // PHatModq[j][l] * P^-1 (* 2^64 with mont_down)
        u64 v = mulmod(D.phatmodq[threadIdx.x * D.fullQ + l], D.pinv[l], m);
        if (D.mont_down) v = mulmod(v, r_mod(m), m);
        cl_[threadIdx.x] = v;
    }
    __syncthreads();
    const u64 ni = D.ninvu[l], nip = D.ninvup[l];
    u64* U = slot_ptr(P, w.U + c, LOGN) + c0;
    const u64* XP = slot_ptr(P, w.RP + c * K, LOGN) + c0;
    auto ld = [&](int r, int cl) { return U[r * 256 + cl]; };
    auto st = [&](int r, int cl, u64 v) {
        const int e = r * 256 + cl;
        const u64 u = shoup(v, ni, nip, m.q);
        u64 lo = 0, hi = 0;
        for (u32 j = 0; j < K; ++j) mac_wide(lo, hi, XP[((size_t)j << LOGN) + e], cl_[j]);
        const u64 tmp = D.mont_down ? redc(lo, hi, m) : barrett(lo, hi, m);
        U[e] = u >= tmp ? u - tmp : u + m.q - tmp;
    };
    ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A, true>(sm, twi_of<FP>(D, l, LOGN), ar_of<FP>(m), ld, st);
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
p7b_moddown_inv_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::COL_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::COL_TILES;
    on_path<PATH>(jb, [&](auto fp) { p7b_moddown_inv_col_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

// ------------------------------------------------------------------ P8
template <int LOGN, u32 MODE, bool FP>
__device__ __forceinline__ void p8_body(const DevCtx& D, const PairDesc& P, u32 c, u32 i, int c0, u64* sm,
                                        const u64* ci) {
    using G = ntt::Geo<LOGN>;
    using CS = ColStage<LOGN>;
    const u32 L = P.L, K = D.K, l = L - 1;
    const WsLayout w = ws_layout(L, K, D.alpha);
    const Level& lv = D.lvl[L];
    const ModC m = D.mod[i];
    const u64 q = m.q;
    const u64* XP = slot_ptr(P, w.RP + c * K, LOGN) + c0;
    const u64* R = MODE == RESCALE ? slot_ptr(P, w.X + l, LOGN) + c0 : slot_ptr(P, w.U + c, LOGN) + c0;
    u64* Z = slot_ptr(P, w.Z + c * L + i, LOGN) + c0;
    // SwitchModulus q_l -> q_i (switch_modulus.cu:11-27)
    const u64 ql = D.mod[l].q;
    const u64 half = ql >> 1;
    const bool larger = q > ql;
    const u64 diff = larger ? q - ql : (ql - q) % q;
    const u64 s2 = lv.s2[i], s2p = lv.s2p[i];

    // v = sw_i(r_l) * s2 - conv'_i * cm, lazy in [0, 4q)
    auto finish = [&](u64 x, u64 lo, u64 hi) -> u64 {
        u64 v = 0;
        if constexpr (MODE == EMR || MODE == RESCALE) {
            const u64 d = x > half ? diff : 0;
            u64 sw;
            if (larger) sw = x + d;
            else { const u64 xm = reduce64(x, m); sw = xm >= d ? xm - d : xm + q - d; }
            v = shoup_lazy(sw, s2, s2p, q);
        }
        if constexpr (MODE != RESCALE) {   // conv'_i * cm, folded into the constants
            u64 c = conv_reduce(lo, hi, m, D.mont_down);   // [0, 4q)
            c = csub(c, 2 * q);                            // [0, 2q)
            v += 2 * q - c;
        }
        return v;
    };
#pragma unroll 1
    for (int k0 = 0; k0 < CS::PER; k0 += P8_VB) {
        int r[P8_VB], cl[P8_VB];
        size_t e[P8_VB];
#pragma unroll
        for (int b = 0; b < P8_VB; ++b) {
            CS::pos(k0 + b, r[b], cl[b]);
            e[b] = (size_t)r[b] * 256 + cl[b];
        }
        ulonglong2 xr[P8_VB];
        if constexpr (MODE == EMR || MODE == RESCALE) {
#pragma unroll
            for (int b = 0; b < P8_VB; ++b) xr[b] = ld2(R + e[b]);
        }
        u64 lo[P8_VB][2] = {}, hi[P8_VB][2] = {};
        if constexpr (MODE != RESCALE) mac_terms<P8_VB>(lo, hi, XP, (size_t)1 << LOGN, K, ci, e);
#pragma unroll
        for (int b = 0; b < P8_VB; ++b) {
            const bool has_r = MODE == EMR || MODE == RESCALE;
            ulonglong2 v;
            v.x = finish(has_r ? xr[b].x : 0, lo[b][0], hi[b][0]);
            v.y = finish(has_r ? xr[b].y : 0, lo[b][1], hi[b][1]);
            *reinterpret_cast<ulonglong2*>(sm + r[b] * G::C + cl[b]) = v;
        }
    }
    __syncthreads();
    auto ld = [&](int r, int cl) { return sm[r * G::C + cl]; };
    auto st = [&](int r, int cl, u64 v) { Z[r * 256 + cl] = v; };
    ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0, true>(sm, twf_of<FP>(D, i, LOGN), ar_of<FP>(m), ld, st);
}

template <int LOGN, bool FP>
__device__ __forceinline__ void p8_moddown_fwd_col_body(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint2 jb,
                                              const u32 tile) {
    extern __shared__ __align__(16) u64 sm[];
    __shared__ u64 ci[gfx::MAXP];
    const int c0 = tile * ntt::Geo<LOGN>::C;
    const PairDesc& P = pairs[jb.x];
    const u32 c = jb.y / P.L, i = jb.y % P.L;
    if (threadIdx.x < D.K) {
        // PHatModq[j][i] times the combine factor cm (P^-1 * s1 for EvalMult+Rescale,
        // P^-1 otherwise) and, with mont_down, 2^64: the staged sum then reduces
        // straight to conv'_i * cm
        const ModC mi = D.mod[i];
        const u64 cm = P.mode == EMR ? D.lvl[P.L].ps1[i] : D.pinv[i];
        u64 v = mulmod(D.phatmodq[threadIdx.x * D.fullQ + i], cm, mi);
        if (D.mont_down) v = mulmod(v, r_mod(mi), mi);
        ci[threadIdx.x] = v;
    }
    __syncthreads();
    if (P.mode == EMR) p8_body<LOGN, EMR, FP>(D, P, c, i, c0, sm, ci);
    else if (P.mode == RESCALE) p8_body<LOGN, RESCALE, FP>(D, P, c, i, c0, sm, ci);
    else p8_body<LOGN, KS, FP>(D, P, c, i, c0, sm, ci);
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
p8_moddown_fwd_col(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::COL_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::COL_TILES;
    on_path<PATH>(jb, [&](auto fp) { p8_moddown_fwd_col_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

// ------------------------------------------------------------------ P9
template <int LOGN, bool FP>
__device__ __forceinline__ void p9_final_fwd_row_body(const DevCtx& D, const PairDesc* __restrict__ pairs, const uint2 jb,
                                              const u32 tile) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const u32 R0 = tile * G::RB;
    const PairDesc& P = pairs[jb.x];
    const u32 L = P.L, K = D.K, mode = P.mode;
    const u32 c = jb.y / L, i = jb.y % L;
    const WsLayout w = ws_layout(L, K, D.alpha);
    const ModC m = D.mod[i];
    const size_t tile0 = (size_t)R0 * 256;
    const u64* Z = slot_ptr(P, w.Z + c * L + i, LOGN) + tile0;
    auto ld = [&](int rl, int cc) { return Z[rl * 256 + cc]; };
    const auto ar = ar_of<FP>(m);
    ntt::fwd_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 0, true>(sm, twf_of<FP>(D, i, LOGN), R0, ar, ld);
    const size_t o = ((size_t)i << LOGN) + tile0;
    u64* out = P.out[c] + o;
    const u64* Wt = slot_ptr(P, w.W + c * L + i, LOGN) + tile0;
    const Level& lv = D.lvl[L];
    const u64 s1 = lv.s1[i], s1p = lv.s1p[i];
    // every W (or rescale input) word of the thread is loaded before the sums
    const u64* addend = mode == RESCALE ? P.in[0] + o : Wt;
    ntt::row_tile_stage<G::RB, G::ROW_THREADS>(
        [&](int rl, int cc) { return addend[rl * 256 + cc]; },
        [&](int rl, int cc, u64 a) {
            const int e = rl * 256 + cc;
            const u64 v = ar.final_canon(sm[rl * G::ROW_STRIDE + ntt::rowpad(cc)]);
            u64 r;
            if (mode == RESCALE) {
                r = csub(shoup(a, s1, s1p, m.q) + v, m.q);
            } else {
                r = csub(a + v, m.q);
                if ((mode == ROT || mode == HROT) && c == 0)
                    r = csub(r + P.in[0][((size_t)i << LOGN) + galois_slot<LOGN>((u32)(tile0 + e), P.galois)], m.q);
            }
            out[e] = r;
        });
}

template <int LOGN, int PATH>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS, 4)
p9_final_fwd_row(const DevCtx D, const PairDesc* __restrict__ pairs, const uint2* __restrict__ jobs) {
    uint2 jb = jobs[blockIdx.x / ntt::Geo<LOGN>::ROW_TILES];
    const u32 tile = blockIdx.x % ntt::Geo<LOGN>::ROW_TILES;
    on_path<PATH>(jb, [&](auto fp) { p9_final_fwd_row_body<LOGN, decltype(fp)::value>(D, pairs, jb, tile); });
}

}  // namespace pl
