// Two-pass negacyclic NTT engine for N = 2^LOGN, 9 <= LOGN <= 16.
//
// The transform is the reference's: forward Cooley-Tukey with twiddle
// roots[m+i] = psi^bitrev(m+i) (standard order in, bit-reversed out) and the
// inverse Gentleman-Sande with the same indexing (bit-reversed in, standard
// out). The coefficient vector is viewed as a matrix x[r*256 + c] with
// R1 = 2^(LOGN-8) rows of 256 columns:
//   * the first A = LOGN-8 forward stages only couple rows (fixed column):
//     the "column pass", tile = all R1 rows x C columns;
//   * the last 8 stages only couple columns inside one row: the "row pass",
//     tile = RB rows x 256.
// Each pass runs radix-2^K rounds held in registers (K <= 4, 16 values per
// thread), exchanging through shared memory between rounds, so a pass reads
// and writes global memory once.
//
// Two arithmetic policies run the same rounds. IntAr: 64-bit integer
// Harvey lazy butterflies with Shoup twiddles (forward values in [0,4q),
// inverse in [0,2q)), any q < 2^62. FpAr (q < 2^50): residues held as signed
// FP64 integers and multiplied exactly with FMA (see FpAr), which runs on
// the FP64 pipe at about twice the integer path's butterfly rate. Both give
// the same canonical residues, so callers pick per tower.
//
// Twiddle index of line-local stage j: a round that starts at stage J0 with
// group base B = 2^(goff+J0) + HB uses twiddle (B << l) + (u >> (K-l)) at its
// local stage l for register slot u (see ct_reg / gs_reg).
#pragma once
#include "gf.cuh"

namespace ntt {

struct TwPacked {
    const Tw* t;
    __device__ __forceinline__ Tw operator()(u32 i) const { return t[i]; }
};
struct TwSplit {
    const u64* w;
    const u64* wp;
    __device__ __forceinline__ Tw operator()(u32 i) const { return Tw{__ldg(w + i), __ldg(wp + i)}; }
};

// FP64 twiddle accessors: a library double table, or the reference's u64
// table converted on load.
__device__ __forceinline__ double u2d(u64 x) {   // exact for x < 2^52
    return __dsub_rn(__longlong_as_double((long long)(x | 0x4330000000000000ull)), 4503599627370496.0);
}
__device__ __forceinline__ u64 d2u(double z) {   // integer 0 <= z < 2^52
    return (u64)__double_as_longlong(__dadd_rn(z, 4503599627370496.0)) & 0xFFFFFFFFFFFFFull;
}
struct TwD {
    const double* t;
    __device__ __forceinline__ double operator()(u32 i) const { return __ldg(t + i); }
};

// The 2^L twiddles tw(base + g), g < 2^L, of one butterfly group at local
// stage L (base = B << L, so the run is aligned to 2^L entries). The
// library's double tables (TwD, 16-byte aligned per modulus) load them as
// 16-byte vectors; other tables load word by word.
template <int L, class TW>
__device__ __forceinline__ void tw_run(const TW& tw, u32 base, double (&w)[1 << L]) {
#pragma unroll
    for (int g = 0; g < (1 << L); ++g) w[g] = tw(base + (u32)g);
}
template <int L>
__device__ __forceinline__ void tw_run(const TwD& tw, u32 base, double (&w)[1 << L]) {
    if constexpr (L == 0) {
        w[0] = __ldg(tw.t + base);
    } else {
        const double2* p = reinterpret_cast<const double2*>(tw.t + base);
#pragma unroll
        for (int h = 0; h < (1 << (L - 1)); ++h) {
            const double2 v = __ldg(p + h);
            w[2 * h] = v.x;
            w[2 * h + 1] = v.y;
        }
    }
}
struct TwDConv {
    const u64* w;
    __device__ __forceinline__ double operator()(u32 i) const { return u2d(__ldg(w + i)); }
};

// One radix-2 stage (local stage L of K) on the register slots; recursion
// over L keeps every index a compile-time constant so v stays in registers.
template <int K, int L, class TW>
__device__ __forceinline__ void ct_stage(u64 (&v)[1 << K], const TW& tw, u32 B, u64 q, u64 two_q) {
    constexpr int half = 1 << (K - 1 - L);
#pragma unroll
    for (int g = 0; g < (1 << L); ++g) {
        const Tw t = tw((B << L) + g);
#pragma unroll
        for (int o = 0; o < half; ++o)
            ct_bfly(v[g * 2 * half + o], v[g * 2 * half + o + half], t.w, t.wp, q, two_q);
    }
    if constexpr (L + 1 < K) ct_stage<K, L + 1>(v, tw, B, q, two_q);
}

template <int K, int L, class TW>
__device__ __forceinline__ void gs_stage(u64 (&v)[1 << K], const TW& tw, u32 B, u64 q, u64 two_q) {
    constexpr int half = 1 << (K - 1 - L);
#pragma unroll
    for (int g = 0; g < (1 << L); ++g) {
        const Tw t = tw((B << L) + g);
#pragma unroll
        for (int o = 0; o < half; ++o)
            gs_bfly(v[g * 2 * half + o], v[g * 2 * half + o + half], t.w, t.wp, q, two_q);
    }
    if constexpr (L > 0) gs_stage<K, L - 1>(v, tw, B, q, two_q);
}

// K forward stages (local 0..K-1) / K inverse stages (local K-1..0).
template <int K, class TW>
__device__ __forceinline__ void ct_reg(u64 (&v)[1 << K], const TW& tw, u32 B, u64 q, u64 two_q) {
    ct_stage<K, 0>(v, tw, B, q, two_q);
}
template <int K, class TW>
__device__ __forceinline__ void gs_reg(u64 (&v)[1 << K], const TW& tw, u32 B, u64 q, u64 two_q) {
    gs_stage<K, K - 1>(v, tw, B, q, two_q);
}

// ------------------------------------------------------------------ FP64 arithmetic
// Residues as FP64 integers for q < 2^50 (so 8q < 2^53). With
// M2 = 1.5*2^53 and M1 = 1.5*2^52 ("magic" constants whose addition rounds
// to the nearest even / nearest integer) and qinv = RN(1/q) (relative error
// at most 2^-53):
//   mul(y, w): h = RN(y*w); l = y*w - h exactly (FMA); k = RN(h*qinv) by M1
//     or RN2(h*qinv) (even) by M2; r = (h - k*q) + l. h, l, h - k*q and r are
//     exact integers (|h| >= 2^53 makes h an integer, h - k*q and r are
//     integers below 2^52), so r = y*w (mod q). With |h| <= c*q*|w|:
//     |l| <= |h| 2^-53 and |k - h/q| <= e + |h/q| 2^-53, e = 1/2 (M1) or 1 (M2).
//   norm(z), |z| < 2^53: k = RN(z*qinv) by M1; z - k*q in [-q/2 - 1, q/2 + 1].
//
// Unsigned twiddles 0 <= w < q (FpArT<false>, tables converted on load): mul
// by M2 for |y| <= 4q gives |r| <= 2q. A round keeps every value normalised
// at its start and end and normalises after every second stage: forward (CT)
// values stay below 4.5q + 1 and multiplier inputs below 2.5q + 1; inverse
// (GS) values below 3q + 2, multiplier inputs below 3q + 2.
//
// Signed twiddles |w| <= (q-1)/2 (FpArT<true>, the library's double tables):
// |h/q| <= |y|/2, so with c = |y|/q and q < 2^50, |l| <= (c/16) q and
//   M1 (needs |y| < 2^52):  |r| <= (1/2 + c/8) q,
//   M2 (needs |y| < 2^53):  |r| <= (1 + c/8) q,
// and a round of up to four stages needs one normalisation, at its end:
//   CT from |x| <= q/2 + 1, M1 in every stage: stage outputs below 1.07q,
//     1.70q, 2.41q, 3.21q; multiplier inputs below 2.41q < 4q.
//   GS from |x| <= q/2 + 1: stages one to three by M1 (multiplier inputs
//     below q + 2, 2q + 4, 4q + 8 < 2^52, since an NTT prime below 2^50 has
//     q = 1 mod 2n with n >= 2^9, so q <= 2^50 - 2^10 + 1), values below
//     q + 2, 2q + 4, 4q + 8; stage four
//     by M2 (input below 8q + 16 < 2^53, |r| <= 2q + 2), sums below 8q + 16.
// Every value stays an exact integer below 2^53, so the results equal the
// integer path's canonical residues.
constexpr double FP_M1 = 6755399441055744.0;    // 1.5 * 2^52
constexpr double FP_M2 = 13510798882111488.0;   // 1.5 * 2^53

template <bool SIGNED_TW>
struct FpArT {
    using T = double;
    double q, qinv;
    __device__ __forceinline__ double norm(double z) const {
        const double k = __dsub_rn(__fma_rn(z, qinv, FP_M1), FP_M1);
        return __fma_rn(-k, q, z);
    }
    template <bool EVEN = true>
    __device__ __forceinline__ double mulq(double y, double w) const {
        constexpr double M = EVEN ? FP_M2 : FP_M1;
        const double h = __dmul_rn(y, w);
        const double l = __fma_rn(y, w, -h);
        const double k = __dsub_rn(__fma_rn(h, qinv, M), M);
        return __dadd_rn(__fma_rn(-k, q, h), l);
    }
    __device__ __forceinline__ double mul(double y, double w) const { return mulq<true>(y, w); }
    // x < 4q (any lazy residue of the integer kernels)
    __device__ __forceinline__ double in(u64 x) const { return norm(u2d(x)); }
    // normalised z -> canonical [0, q)
    __device__ __forceinline__ u64 out(double z) const { return d2u(z < 0.0 ? __dadd_rn(z, q) : z); }
    __device__ __forceinline__ u64 bits(double z) const { return (u64)__double_as_longlong(z); }
    __device__ __forceinline__ double unbits(u64 b) const { return __longlong_as_double((long long)b); }
    __device__ __forceinline__ u64 stage_in(u64 x) const { return bits(in(x)); }
    __device__ __forceinline__ u64 final_out(u64 b) const { return out(unbits(b)); }
    // final words already canonical: no lazy-range correction needed
    __device__ __forceinline__ u64 final_canon(u64 b) const { return out(unbits(b)); }
    __device__ __forceinline__ u64 final_2q(u64 b) const { return out(unbits(b)); }
    // pass-to-pass intermediates stay in the policy's own representation
    __device__ __forceinline__ double from_raw(u64 b) const { return unbits(b); }
    __device__ __forceinline__ u64 to_raw(double z) const { return bits(z); }

    template <int K, int L, class TW>
    __device__ __forceinline__ void ct_stage(double (&v)[1 << K], const TW& tw, u32 B) const {
        static_assert(K <= 4, "bounds are proven for rounds of at most four stages");
        constexpr int half = 1 << (K - 1 - L);
        double wr[1 << L];
        tw_run<L>(tw, B << L, wr);
#pragma unroll
        for (int g = 0; g < (1 << L); ++g) {
            const double w = wr[g];
#pragma unroll
            for (int o = 0; o < half; ++o) {
                double& x = v[g * 2 * half + o];
                double& y = v[g * 2 * half + o + half];
                const double r = mulq<!SIGNED_TW>(y, w), xx = x;
                x = __dadd_rn(xx, r);
                y = __dsub_rn(xx, r);
            }
        }
        if constexpr ((!SIGNED_TW && L % 2 == 1) || L == K - 1) {
#pragma unroll
            for (int u = 0; u < (1 << K); ++u) v[u] = norm(v[u]);
        }
        if constexpr (L + 1 < K) ct_stage<K, L + 1>(v, tw, B);
    }
    template <int K, int L, class TW>
    __device__ __forceinline__ void gs_stage(double (&v)[1 << K], const TW& tw, u32 B) const {
        static_assert(K <= 4, "bounds are proven for rounds of at most four stages");
        constexpr int half = 1 << (K - 1 - L);
        constexpr bool EVEN = !SIGNED_TW || (K - 1 - L) >= 3;
        double wr[1 << L];
        tw_run<L>(tw, B << L, wr);
#pragma unroll
        for (int g = 0; g < (1 << L); ++g) {
            const double w = wr[g];
#pragma unroll
            for (int o = 0; o < half; ++o) {
                double& x = v[g * 2 * half + o];
                double& y = v[g * 2 * half + o + half];
                const double xx = x, yy = y;
                x = __dadd_rn(xx, yy);
                y = mulq<EVEN>(__dsub_rn(xx, yy), w);
            }
        }
        if constexpr ((!SIGNED_TW && (K - L) % 2 == 0) || L == 0) {
#pragma unroll
            for (int u = 0; u < (1 << K); ++u) v[u] = norm(v[u]);
        }
        if constexpr (L > 0) gs_stage<K, L - 1>(v, tw, B);
    }
    template <int K, class TW>
    __device__ __forceinline__ void fwd(double (&v)[1 << K], const TW& tw, u32 B) const { ct_stage<K, 0>(v, tw, B); }
    template <int K, class TW>
    __device__ __forceinline__ void inv(double (&v)[1 << K], const TW& tw, u32 B) const { gs_stage<K, K - 1>(v, tw, B); }
};
// Unsigned twiddles (the reference's u64 tables converted on load).
using FpAr = FpArT<false>;
// Signed twiddles in (-q/2, q/2) (the library's double tables).
using FpArS = FpArT<true>;

// Integer path: the lazy Harvey/Shoup butterflies above, values as-is.
struct IntAr {
    using T = u64;
    u64 q, two_q;
    __device__ __forceinline__ u64 in(u64 x) const { return x; }
    __device__ __forceinline__ u64 out(u64 x) const { return x; }
    __device__ __forceinline__ u64 bits(u64 x) const { return x; }
    __device__ __forceinline__ u64 unbits(u64 b) const { return b; }
    __device__ __forceinline__ u64 stage_in(u64 x) const { return x; }
    __device__ __forceinline__ u64 final_out(u64 b) const { return b; }
    // lazy [0, 4q) -> canonical [0, q), or -> [0, 2q)
    __device__ __forceinline__ u64 final_canon(u64 b) const { return csub(csub(b, two_q), q); }
    __device__ __forceinline__ u64 final_2q(u64 b) const { return csub(b, two_q); }
    __device__ __forceinline__ u64 from_raw(u64 b) const { return b; }
    __device__ __forceinline__ u64 to_raw(u64 v) const { return v; }
    template <int K, class TW>
    __device__ __forceinline__ void fwd(u64 (&v)[1 << K], const TW& tw, u32 B) const { ct_reg<K>(v, tw, B, q, two_q); }
    template <int K, class TW>
    __device__ __forceinline__ void inv(u64 (&v)[1 << K], const TW& tw, u32 B) const { gs_reg<K>(v, tw, B, q, two_q); }
};

__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Geometry of the two passes for one LOGN.
template <int LOGN>
struct Geo {
    static_assert(LOGN >= 9 && LOGN <= 16, "LOGN out of range");
    static constexpr int N = 1 << LOGN;
    static constexpr int A = LOGN - 8;               // column stages
    static constexpr int R1 = 1 << A;                // rows
    static constexpr int COLS = 256;
    // column pass: all rows x C columns, <= 4096 elements, >= 16 columns
    static constexpr int C = cmin(256, cmax(16, 4096 >> A));
    static constexpr int COL_TILE = R1 * C;
    static constexpr int COL_TILES = COLS / C;
    static constexpr int COL_THREADS = COL_TILE / 16;
    // row pass: RB rows x 256 (padded rows in shared memory)
    static constexpr int RB = cmin(R1, 16);
    static constexpr int ROW_TILE = RB * COLS;
    static constexpr int ROW_TILES = R1 / RB;
    static constexpr int ROW_THREADS = ROW_TILE / 16;
    static constexpr int ROW_STRIDE = COLS + COLS / 16;      // one pad word per 16
    static constexpr int COL_SMEM = COL_TILE * 8;
    static constexpr int ROW_SMEM = RB * ROW_STRIDE * 8;
};

__device__ __forceinline__ int rowpad(int c) { return c + (c >> 4); }

// ------------------------------------------------------------------ column pass
// Round (J0, K) over a column tile: thread groups index gi -> (cl, lo, hidx).
// LD(r, cl) -> u64 and ST(r, cl, v) address tile-local column cl, global row r.
template <int A, int C, int NT, int J0, int K, bool FWD, class AR, class TW, class LD, class ST>
__device__ __forceinline__ void col_round(const AR& ar, const TW& tw, LD&& ld, ST&& st) {
    constexpr int SH = A - J0 - K;
    constexpr int GROUPS = ((1 << A) * C) >> K;
    static_assert(GROUPS % NT == 0, "groups must divide evenly");
#pragma unroll 1
    for (int gi = threadIdx.x; gi < GROUPS; gi += NT) {
        const int cl = gi % C;
        const int rest = gi / C;
        const int lo = rest & ((1 << SH) - 1);
        const int hidx = rest >> SH;
        const int hi = hidx << (A - J0);
        typename AR::T v[1 << K];
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) v[u] = ld(hi + (u << SH) + lo, cl);
        const u32 B = (1u << J0) + (u32)hidx;
        if constexpr (FWD) ar.template fwd<K>(v, tw, B);
        else ar.template inv<K>(v, tw, B);
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) st(hi + (u << SH) + lo, cl, v[u]);
    }
}

// Forward column pass: stages 0..A-1. First round loads via `ld`, last round
// stores via `st`; intermediate rounds go through shared memory `sm`.
// Barrier between rounds: the whole CTA by default; a warp-specialised
// kernel passes a named barrier over its transform warps.
struct CtaSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// `ld` returns u64 residues below 4q; `st` receives the policy's output
// (IntAr: lazy [0,4q); FpAr: canonical [0,q)), or with RAW_OUT the policy's
// own word (ar.to_raw), for a following row pass that reads it with RAW_IN.
template <int A, int C, int NT, int J0, bool RAW_OUT = false, class AR, class TW, class LD, class ST,
          class SY = CtaSync>
__device__ __forceinline__ void fwd_col_rounds(u64* sm, const TW& tw, const AR& ar, LD&& ld, ST&& st,
                                               const SY& sync = SY{}) {
    constexpr int K = cmin(4, A - J0);
    constexpr bool FIRST = (J0 == 0);
    constexpr bool LAST = (J0 + K == A);
    using T = typename AR::T;
    auto gld = [&](int r, int cl) { return ar.in(ld(r, cl)); };
    auto gst = [&](int r, int cl, T v) {
        if constexpr (RAW_OUT) st(r, cl, ar.to_raw(v));
        else st(r, cl, ar.out(v));
    };
    auto sld = [&](int r, int cl) { return ar.unbits(sm[r * C + cl]); };
    auto sst = [&](int r, int cl, T v) { sm[r * C + cl] = ar.bits(v); };
    if constexpr (FIRST && LAST) col_round<A, C, NT, J0, K, true>(ar, tw, gld, gst);
    else if constexpr (FIRST) col_round<A, C, NT, J0, K, true>(ar, tw, gld, sst);
    else if constexpr (LAST) col_round<A, C, NT, J0, K, true>(ar, tw, sld, gst);
    else col_round<A, C, NT, J0, K, true>(ar, tw, sld, sst);
    if constexpr (!LAST) {
        sync();
        fwd_col_rounds<A, C, NT, J0 + K, RAW_OUT>(sm, tw, ar, ld, st, sync);
    }
}

// Inverse column pass: stages A-1..0 (GS). Rounds run from the top stage
// group down; JE is the exclusive end of the current round's stage range.
// RAW_IN: `ld` returns the policy's own words written by a RAW_OUT row pass.
template <int A, int C, int NT, int JE, bool RAW_IN = false, class AR, class TW, class LD, class ST>
__device__ __forceinline__ void inv_col_rounds(u64* sm, const TW& tw, const AR& ar, LD&& ld, ST&& st) {
    // partition identical to the forward one: rounds [0,4),[4,8),... last ragged
    constexpr int J0 = ((JE - 1) / 4) * 4;
    constexpr int K = JE - J0;
    constexpr bool FIRST = (JE == A);
    constexpr bool LAST = (J0 == 0);
    using T = typename AR::T;
    auto gld = [&](int r, int cl) {
        if constexpr (RAW_IN) return ar.from_raw(ld(r, cl));
        else return ar.in(ld(r, cl));
    };
    auto gst = [&](int r, int cl, T v) { st(r, cl, ar.out(v)); };
    auto sld = [&](int r, int cl) { return ar.unbits(sm[r * C + cl]); };
    auto sst = [&](int r, int cl, T v) { sm[r * C + cl] = ar.bits(v); };
    if constexpr (FIRST && LAST) col_round<A, C, NT, J0, K, false>(ar, tw, gld, gst);
    else if constexpr (FIRST) col_round<A, C, NT, J0, K, false>(ar, tw, gld, sst);
    else if constexpr (LAST) col_round<A, C, NT, J0, K, false>(ar, tw, sld, gst);
    else col_round<A, C, NT, J0, K, false>(ar, tw, sld, sst);
    if constexpr (!LAST) {
        __syncthreads();
        inv_col_rounds<A, C, NT, J0, RAW_IN>(sm, tw, ar, ld, st);
    }
}

// ------------------------------------------------------------------ row pass
// Round (J0, K) over a row tile of RB rows; global row of tile row 0 is R0.
// Twiddle base B = 2^(A+J0) + ((R0+rl) << J0) + hidx.
template <int A, int RB, int NT, int J0, int K, bool FWD, class AR, class TW, class LD, class ST>
__device__ __forceinline__ void row_round(const AR& ar, const TW& tw, u32 R0, LD&& ld, ST&& st) {
    constexpr int SH = 8 - J0 - K;
    constexpr int GROUPS = (RB * 256) >> K;
    static_assert(GROUPS % NT == 0, "groups must divide evenly");
#pragma unroll 1
    for (int gi = threadIdx.x; gi < GROUPS; gi += NT) {
        const int lo = gi & ((1 << SH) - 1);
        const int rest = gi >> SH;
        const int hidx = rest & ((1 << J0) - 1);
        const int rl = rest >> J0;
        const int cb = (hidx << (8 - J0)) + lo;
        typename AR::T v[1 << K];
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) v[u] = ld(rl, cb + (u << SH));
        const u32 B = (1u << (A + J0)) + ((R0 + (u32)rl) << J0) + (u32)hidx;
        if constexpr (FWD) ar.template fwd<K>(v, tw, B);
        else ar.template inv<K>(v, tw, B);
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) st(rl, cb + (u << SH), v[u]);
    }
}

template <int KMAX, int J0>
struct RowK { static constexpr int K = cmin(KMAX, 8 - J0); };

// Forward row pass: stages A..A+7, rounds of KMAX. The first round reads with
// `ld` (u64 below 4q) directly; the last round writes shared memory, and the
// caller then reads the tile row-contiguously (coalesced) and converts each
// word with ar.final_out.
// RAW_IN: `ld` returns the policy's own words written by a RAW_OUT column pass.
template <int A, int RB, int NT, int KMAX, int J0, bool RAW_IN = false, class AR, class TW, class LD>
__device__ __forceinline__ void fwd_row_rounds(u64* sm, const TW& tw, u32 R0, const AR& ar, LD&& ld) {
    constexpr int K = RowK<KMAX, J0>::K;
    constexpr bool LAST = (J0 + K == 8);
    constexpr int STR = 256 + 16;
    using T = typename AR::T;
    auto gld = [&](int rl, int c) {
        if constexpr (RAW_IN) return ar.from_raw(ld(rl, c));
        else return ar.in(ld(rl, c));
    };
    auto sld = [&](int rl, int c) { return ar.unbits(sm[rl * STR + rowpad(c)]); };
    auto sst = [&](int rl, int c, T v) { sm[rl * STR + rowpad(c)] = ar.bits(v); };
    if constexpr (J0 == 0) row_round<A, RB, NT, J0, K, true>(ar, tw, R0, gld, sst);
    else row_round<A, RB, NT, J0, K, true>(ar, tw, R0, sld, sst);
    __syncthreads();
    if constexpr (!LAST) fwd_row_rounds<A, RB, NT, KMAX, J0 + K, RAW_IN>(sm, tw, R0, ar, ld);
}

// Inverse row pass: GS stages A+7..A. Input is staged into shared memory
// (row-contiguous, coalesced) by the caller through ar.stage_in; the last
// round stores via `st`, which receives the policy's output.
// RAW_OUT: `st` receives the policy's own words (ar.to_raw) for a following
// column pass that reads them with RAW_IN.
template <int A, int RB, int NT, int KMAX, int JE, bool RAW_OUT = false, class AR, class TW, class ST>
__device__ __forceinline__ void inv_row_rounds(u64* sm, const TW& tw, u32 R0, const AR& ar, ST&& st) {
    constexpr int J0 = ((JE - 1) / KMAX) * KMAX;
    constexpr int K = JE - J0;
    constexpr bool LAST = (J0 == 0);
    constexpr int STR = 256 + 16;
    using T = typename AR::T;
    auto gst = [&](int rl, int c, T v) {
        if constexpr (RAW_OUT) st(rl, c, ar.to_raw(v));
        else st(rl, c, ar.out(v));
    };
    auto sld = [&](int rl, int c) { return ar.unbits(sm[rl * STR + rowpad(c)]); };
    auto sst = [&](int rl, int c, T v) { sm[rl * STR + rowpad(c)] = ar.bits(v); };
    if constexpr (LAST) row_round<A, RB, NT, J0, K, false>(ar, tw, R0, sld, gst);
    else {
        row_round<A, RB, NT, J0, K, false>(ar, tw, R0, sld, sst);
        __syncthreads();
        inv_row_rounds<A, RB, NT, KMAX, J0, RAW_OUT>(sm, tw, R0, ar, st);
    }
}

// Coalesced walks over a row tile (RB rows x 256), 2 words per step so that a
// warp touches 512 contiguous bytes.
template <int RB, int NT, class F>
__device__ __forceinline__ void row_tile_walk(F&& f) {
#pragma unroll 4
    for (int e = threadIdx.x; e < RB * 256; e += NT) f(e >> 8, e & 255);
}

// Same walk for staging a tile: every load of the thread (RB*256/NT words)
// is issued before the first conversion and shared-memory store.
template <int RB, int NT, class LD, class ST>
__device__ __forceinline__ void row_tile_stage(LD&& ld, ST&& st) {
    constexpr int PER = RB * 256 / NT;
    static_assert(PER * NT == RB * 256 && PER <= 16, "stage geometry");
    u64 v[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = threadIdx.x + k * NT;
        v[k] = ld(e >> 8, e & 255);
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = threadIdx.x + k * NT;
        st(e >> 8, e & 255, v[k]);
    }
}

// Two-operand staging in batches of 8 words per thread: both operands of a
// batch are loaded before st(rl, c, a, b) combines them.
template <int RB, int NT, class LDA, class LDB, class ST>
__device__ __forceinline__ void row_tile_stage2(LDA&& lda, LDB&& ldb, ST&& st) {
    constexpr int PER = RB * 256 / NT;
    constexpr int BT = PER < 8 ? PER : 8;
    static_assert(PER * NT == RB * 256 && PER % BT == 0, "stage geometry");
#pragma unroll
    for (int k0 = 0; k0 < PER; k0 += BT) {
        u64 a[BT], b[BT];
#pragma unroll
        for (int k = 0; k < BT; ++k) {
            const int e = threadIdx.x + (k0 + k) * NT;
            a[k] = lda(e >> 8, e & 255);
            b[k] = ldb(e >> 8, e & 255);
        }
#pragma unroll
        for (int k = 0; k < BT; ++k) {
            const int e = threadIdx.x + (k0 + k) * NT;
            st(e >> 8, e & 255, a[k], b[k]);
        }
    }
}

}  // namespace ntt
