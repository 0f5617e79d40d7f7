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
// and writes global memory once. Butterflies are Harvey's lazy forms
// (forward values in [0,4q), inverse in [0,2q)).
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
template <int A, int C, int NT, int J0, int K, bool FWD, class TW, class LD, class ST>
__device__ __forceinline__ void col_round(const TW& tw, u64 q, u64 two_q, LD&& ld, ST&& st) {
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
        u64 v[1 << K];
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) v[u] = ld(hi + (u << SH) + lo, cl);
        const u32 B = (1u << J0) + (u32)hidx;
        if (FWD) ct_reg<K>(v, tw, B, q, two_q);
        else gs_reg<K>(v, tw, B, q, two_q);
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) st(hi + (u << SH) + lo, cl, v[u]);
    }
}

// Forward column pass: stages 0..A-1. First round loads via `ld`, last round
// stores via `st`; intermediate rounds go through shared memory `sm`.
template <int A, int C, int NT, int J0, class TW, class LD, class ST>
__device__ __forceinline__ void fwd_col_rounds(u64* sm, const TW& tw, u64 q, u64 two_q, LD&& ld, ST&& st) {
    constexpr int K = cmin(4, A - J0);
    constexpr bool FIRST = (J0 == 0);
    constexpr bool LAST = (J0 + K == A);
    auto sld = [&](int r, int cl) { return sm[r * C + cl]; };
    auto sst = [&](int r, int cl, u64 v) { sm[r * C + cl] = v; };
    if constexpr (FIRST && LAST) col_round<A, C, NT, J0, K, true>(tw, q, two_q, ld, st);
    else if constexpr (FIRST) col_round<A, C, NT, J0, K, true>(tw, q, two_q, ld, sst);
    else if constexpr (LAST) col_round<A, C, NT, J0, K, true>(tw, q, two_q, sld, st);
    else col_round<A, C, NT, J0, K, true>(tw, q, two_q, sld, sst);
    if constexpr (!LAST) {
        __syncthreads();
        fwd_col_rounds<A, C, NT, J0 + K>(sm, tw, q, two_q, ld, st);
    }
}

// Inverse column pass: stages A-1..0 (GS). Rounds run from the top stage
// group down; JE is the exclusive end of the current round's stage range.
template <int A, int C, int NT, int JE, class TW, class LD, class ST>
__device__ __forceinline__ void inv_col_rounds(u64* sm, const TW& tw, u64 q, u64 two_q, LD&& ld, ST&& st) {
    // partition identical to the forward one: rounds [0,4),[4,8),... last ragged
    constexpr int J0 = ((JE - 1) / 4) * 4;
    constexpr int K = JE - J0;
    constexpr bool FIRST = (JE == A);
    constexpr bool LAST = (J0 == 0);
    auto sld = [&](int r, int cl) { return sm[r * C + cl]; };
    auto sst = [&](int r, int cl, u64 v) { sm[r * C + cl] = v; };
    if constexpr (FIRST && LAST) col_round<A, C, NT, J0, K, false>(tw, q, two_q, ld, st);
    else if constexpr (FIRST) col_round<A, C, NT, J0, K, false>(tw, q, two_q, ld, sst);
    else if constexpr (LAST) col_round<A, C, NT, J0, K, false>(tw, q, two_q, sld, st);
    else col_round<A, C, NT, J0, K, false>(tw, q, two_q, sld, sst);
    if constexpr (!LAST) {
        __syncthreads();
        inv_col_rounds<A, C, NT, J0>(sm, tw, q, two_q, ld, st);
    }
}

// ------------------------------------------------------------------ row pass
// Round (J0, K) over a row tile of RB rows; global row of tile row 0 is R0.
// Twiddle base B = 2^(A+J0) + ((R0+rl) << J0) + hidx.
template <int A, int RB, int NT, int J0, int K, bool FWD, class TW, class LD, class ST>
__device__ __forceinline__ void row_round(const TW& tw, u32 R0, u64 q, u64 two_q, LD&& ld, ST&& st) {
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
        u64 v[1 << K];
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) v[u] = ld(rl, cb + (u << SH));
        const u32 B = (1u << (A + J0)) + ((R0 + (u32)rl) << J0) + (u32)hidx;
        if (FWD) ct_reg<K>(v, tw, B, q, two_q);
        else gs_reg<K>(v, tw, B, q, two_q);
#pragma unroll
        for (int u = 0; u < (1 << K); ++u) st(rl, cb + (u << SH), v[u]);
    }
}

template <int KMAX, int J0>
struct RowK { static constexpr int K = cmin(KMAX, 8 - J0); };

// Forward row pass: stages A..A+7, rounds of KMAX. The first round reads with
// `ld` directly; the last round writes shared memory and the tile is then
// stored row-contiguously through `st` (coalesced).
template <int A, int RB, int NT, int KMAX, int J0, class TW, class LD>
__device__ __forceinline__ void fwd_row_rounds(u64* sm, const TW& tw, u32 R0, u64 q, u64 two_q, LD&& ld) {
    constexpr int K = RowK<KMAX, J0>::K;
    constexpr bool LAST = (J0 + K == 8);
    constexpr int STR = 256 + 16;
    auto sld = [&](int rl, int c) { return sm[rl * STR + rowpad(c)]; };
    auto sst = [&](int rl, int c, u64 v) { sm[rl * STR + rowpad(c)] = v; };
    if constexpr (J0 == 0) row_round<A, RB, NT, J0, K, true>(tw, R0, q, two_q, ld, sst);
    else row_round<A, RB, NT, J0, K, true>(tw, R0, q, two_q, sld, sst);
    __syncthreads();
    if constexpr (!LAST) fwd_row_rounds<A, RB, NT, KMAX, J0 + K>(sm, tw, R0, q, two_q, ld);
}

// Inverse row pass: GS stages A+7..A. Input is staged into shared memory
// (row-contiguous, coalesced) by the caller; the last round stores via `st`.
template <int A, int RB, int NT, int KMAX, int JE, class TW, class ST>
__device__ __forceinline__ void inv_row_rounds(u64* sm, const TW& tw, u32 R0, u64 q, u64 two_q, ST&& st) {
    constexpr int J0 = ((JE - 1) / KMAX) * KMAX;
    constexpr int K = JE - J0;
    constexpr bool LAST = (J0 == 0);
    constexpr int STR = 256 + 16;
    auto sld = [&](int rl, int c) { return sm[rl * STR + rowpad(c)]; };
    auto sst = [&](int rl, int c, u64 v) { sm[rl * STR + rowpad(c)] = v; };
    if constexpr (LAST) row_round<A, RB, NT, J0, K, false>(tw, R0, q, two_q, sld, st);
    else {
        row_round<A, RB, NT, J0, K, false>(tw, R0, q, two_q, sld, sst);
        __syncthreads();
        inv_row_rounds<A, RB, NT, KMAX, J0>(sm, tw, R0, q, two_q, st);
    }
}

// Coalesced walks over a row tile (RB rows x 256), 2 words per step so that a
// warp touches 512 contiguous bytes.
template <int RB, int NT, class F>
__device__ __forceinline__ void row_tile_walk(F&& f) {
#pragma unroll 4
    for (int e = threadIdx.x; e < RB * 256; e += NT) f(e >> 8, e & 255);
}

}  // namespace ntt
