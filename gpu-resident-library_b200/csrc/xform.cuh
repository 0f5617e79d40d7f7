// Batched in-place forward / inverse NTT kernels over a list of tower jobs.
// Between its two passes a transform keeps the tower in the arithmetic
// path's own word format (FP64 bits on that path); only the second pass
// writes canonical residues.
// One launch per pass covers every job (ciphertexts x towers): grid =
// jobs x tiles-per-job. Used by the reference ABI (LaunchNTT_CT /
// LaunchINTT_GS, one job) and by the batched transform entry points.
#pragma once
#include "ntt.cuh"

namespace xf {

// One tower to transform in place. Twiddles either packed {w, wp} (library
// tables) or split (two arrays, the reference's table layout). fp != 0 (only
// for q < 2^50) selects the FP64 arithmetic, with the signed double table twd
// (twiddles in (-q/2, q/2)) or, when twd is null, the split w table converted
// on load. Fields after scale_p default to zero (integer path) in brace
// initialisation. `lift` (forward transforms launched by xf_launch_ntt_lift
// only): the column pass reads its words from lift instead of x, each lifted
// into this tower's modulus on load, and x receives the transform.
struct Job {
    u64* x;
    const Tw* tw;        // packed tables, or nullptr when split
    const u64* w;        // split tables
    const u64* wp;
    u64 q;
    u64 scale, scale_p;  // inverse only: n^-1 (and precon) folded in at the end
    const double* twd;   // FP64 twiddles (fp path), or nullptr
    u32 fp;
    u32 reserved;
    const u64* lift;     // words to lift (see xf_launch_ntt_lift), or nullptr
    u64 lift_q0;         // lift source modulus q0 (centred lift), or 0 (signed 64-bit words)
    u64 lift_r64;        // floor(2^64 / q) for the lift's reduction
};

// v (below q0, centred to (-q0/2, q0/2]; or, with q0 = 0, a signed 64-bit
// word) reduced into [0, q): ((c % q) + q) % q of the centred value c, the
// reference's embedding (src/rotate.cpp:108-110, centring src/encdec.cpp:79).
__device__ __forceinline__ u64 lift_word(u64 v, u64 q0, u64 q, u64 r64) {
    const long long c = (q0 && v > (q0 >> 1)) ? (long long)v - (long long)q0 : (long long)v;
    const u64 mag = c < 0 ? 0ull - (u64)c : (u64)c;
    u64 r = mag - __umul64hi(mag, r64) * q;   // [0, 2q)
    r = r >= q ? r - q : r;
    return (c < 0 && r) ? q - r : r;
}

// Calls f(arith policy, twiddle accessor) for the job's path.
template <class F>
__device__ __forceinline__ void with_path(const Job& j, F&& f) {
    if (j.fp) {
        const double qd = ntt::u2d(j.q);
        const double qi = __ddiv_rn(1.0, qd);
        if (j.twd) f(ntt::FpArS{qd, qi}, ntt::TwD{j.twd});
        else f(ntt::FpAr{qd, qi}, ntt::TwDConv{j.w});
        return;
    }
    const ntt::IntAr ar{j.q, 2 * j.q};
    if (j.tw) f(ar, ntt::TwPacked{j.tw});
    else f(ar, ntt::TwSplit{j.w, j.wp});
}

// Jobs come either from a device array (SINGLE = false) or a single by-value
// kernel parameter (SINGLE = true, the reference ABI's one-tower calls).
template <bool SINGLE>
__device__ __forceinline__ Job get_job(const Job* __restrict__ arr, const Job& one, int i) {
    if constexpr (SINGLE) return one;
    else return arr[i];
}

template <int LOGN, bool SINGLE>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
k_fwd_col(const Job* __restrict__ arr, const Job one) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const int job = blockIdx.x / G::COL_TILES;
    const int c0 = (blockIdx.x % G::COL_TILES) * G::C;
    const Job j = get_job<SINGLE>(arr, one, job);
    u64* x = j.x;
    auto ld = [&](int r, int cl) { return x[r * 256 + c0 + cl]; };
    auto st = [&](int r, int cl, u64 v) { x[r * 256 + c0 + cl] = v; };
    with_path(j, [&](const auto& ar, const auto& tw) {
        ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0, true>(sm, tw, ar, ld, st);
    });
}

// Forward column pass whose words come lifted from job.lift (ModRaise: tower 0
// in coefficient form, centred mod q0, into every tower; plaintext embedding:
// signed 64-bit coefficients into every tower), written to job.x: the lift
// and the first transform pass in one read of the source.
template <int LOGN>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
k_fwd_col_lift(const Job* __restrict__ arr) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const int job = blockIdx.x / G::COL_TILES;
    const int c0 = (blockIdx.x % G::COL_TILES) * G::C;
    const Job j = arr[job];
    u64* x = j.x;
    const u64* src = j.lift;
    const u64 q0 = j.lift_q0, q = j.q, r64 = j.lift_r64;
    auto ld = [&](int r, int cl) { return lift_word(__ldg(src + r * 256 + c0 + cl), q0, q, r64); };
    auto st = [&](int r, int cl, u64 v) { x[r * 256 + c0 + cl] = v; };
    with_path(j, [&](const auto& ar, const auto& tw) {
        ntt::fwd_col_rounds<G::A, G::C, G::COL_THREADS, 0, true>(sm, tw, ar, ld, st);
    });
}

template <int LOGN, bool SINGLE>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS, 4)
k_fwd_row(const Job* __restrict__ arr, const Job one) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const int job = blockIdx.x / G::ROW_TILES;
    const u32 R0 = (blockIdx.x % G::ROW_TILES) * G::RB;
    const Job j = get_job<SINGLE>(arr, one, job);
    u64* x = j.x + (size_t)R0 * 256;
    auto ld = [&](int rl, int c) { return x[rl * 256 + c]; };
    with_path(j, [&](const auto& ar, const auto& tw) {
        ntt::fwd_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 0, true>(sm, tw, R0, ar, ld);
        ntt::row_tile_walk<G::RB, G::ROW_THREADS>([&](int rl, int c) {
            x[rl * 256 + c] = ar.final_canon(sm[rl * G::ROW_STRIDE + ntt::rowpad(c)]);
        });
    });
}

template <int LOGN, bool SINGLE>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::ROW_THREADS, 4)
k_inv_row(const Job* __restrict__ arr, const Job one) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const int job = blockIdx.x / G::ROW_TILES;
    const u32 R0 = (blockIdx.x % G::ROW_TILES) * G::RB;
    const Job j = get_job<SINGLE>(arr, one, job);
    u64* x = j.x + (size_t)R0 * 256;
    auto st = [&](int rl, int c, u64 v) { x[rl * 256 + c] = v; };
    with_path(j, [&](const auto& ar, const auto& tw) {
        ntt::row_tile_stage<G::RB, G::ROW_THREADS>(
            [&](int rl, int c) { return x[rl * 256 + c]; },
            [&](int rl, int c, u64 v) { sm[rl * G::ROW_STRIDE + ntt::rowpad(c)] = ar.stage_in(v); });
        __syncthreads();
        ntt::inv_row_rounds<G::A, G::RB, G::ROW_THREADS, 4, 8, true>(sm, tw, R0, ar, st);
    });
}

template <int LOGN, bool SINGLE>
__global__ void __launch_bounds__(ntt::Geo<LOGN>::COL_THREADS, 4)
k_inv_col(const Job* __restrict__ arr, const Job one) {
    using G = ntt::Geo<LOGN>;
    extern __shared__ __align__(16) u64 sm[];
    const int job = blockIdx.x / G::COL_TILES;
    const int c0 = (blockIdx.x % G::COL_TILES) * G::C;
    const Job j = get_job<SINGLE>(arr, one, job);
    const u64 q = j.q;
    u64* x = j.x;
    auto ld = [&](int r, int cl) { return x[r * 256 + c0 + cl]; };
    const u64 sc = j.scale, scp = j.scale_p;
    if (j.fp && sc < q) {   // n^-1 as an exact FP64 product (both operands below q < 2^50)
        const ntt::FpAr ua{ntt::u2d(q), __ddiv_rn(1.0, ntt::u2d(q))};
        const double scd = ntt::u2d(sc);
        auto st = [&](int r, int cl, u64 v) {
            x[r * 256 + c0 + cl] = ua.out(ua.norm(ua.mulq<true>(ntt::u2d(v), scd)));
        };
        with_path(j, [&](const auto& ar, const auto& tw) {
            ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A, true>(sm, tw, ar, ld, st);
        });
        return;
    }
    auto st = [&](int r, int cl, u64 v) { x[r * 256 + c0 + cl] = shoup(v, sc, scp, q); };
    with_path(j, [&](const auto& ar, const auto& tw) {
        ntt::inv_col_rounds<G::A, G::C, G::COL_THREADS, G::A, true>(sm, tw, ar, ld, st);
    });
}

}  // namespace xf

// Host-side dispatch (xform.cu). `jobs` is a device array of njobs jobs, or
// nullptr with `one` used for a single job. Returns cudaErrorInvalidValue for
// an unsupported ring size.
cudaError_t xf_launch_ntt(const xf::Job* jobs, const xf::Job* one, int njobs, int logn,
                          bool inverse, cudaStream_t s);
// Forward transforms of the device job array `jobs`, every job with `lift`
// set: the column pass reads lift-embedded words (k_fwd_col_lift).
cudaError_t xf_launch_ntt_lift(const xf::Job* jobs, int njobs, int logn, cudaStream_t s);
bool xf_supported_logn(int logn);
