// ApproxSwitchCRTBasis on the integer tensor cores, by byte limbs.
//
// The conversion dst_j = (sum_i x_i * M[i][j]) mod p_j, x_i = shoup(a_i,
// QHatInv_i) (reference kernels/basis_convert.cu:14-114) is, over a block of
// coefficients, a product of an (n x sizeQ) matrix by a (sizeQ x sizeP) one
// with 125-bit exact sums. Split every x_i and every M[i][j] into eight
// bytes: with k = 8i + a indexing byte a of x_i, and
//     B_s[k][j] = byte (s - a) of M[i][j]   (0 when s - a lies outside 0..7),
// the exact sum is S_j = sum_{s=0..14} 2^(8s) * C_s[j], C_s = X_bytes * B_s.
// Each C_s is an unsigned 8-bit matrix product with 32-bit accumulation
// (at most 8 * sizeQ * 255^2 < 2^23 per entry), run by mma.sync m16n8k32
// u8.u8.s32 on the tensor pipe; the 15 partial sums of an output are folded
// into four 64-bit words with one wide multiply-add each, combined into 128
// bits and reduced by the same Barrett step as the integer form. The sum is
// the same integer, so the result is bit-identical to LaunchApproxSwitchCRTBasis.
//
// Layout per warp: a tile of 16 coefficients; x of the tile staged in shared
// memory as [16][4C] words (C = k-chunks of 32 bytes = 4 towers each); the
// A fragment of chunk c for lane (g = lane/4, t = lane%4) is word t%2 of
// x[g][4c + t/2] (and of rows g+8, towers 4c+2+t/2), so the staged words are
// the fragment. B fragments depend only on the constants: built once per CTA
// in shared memory for every (shift, chunk, group of 8 targets, lane).
#include <algorithm>
#include <cstdint>
#include <string>

#include "convert.hpp"
#include "devonce.hpp"
#include "gf.cuh"
#include "gpufhe_b200.h"
#include "context.hpp"

namespace {

constexpr int CV_WARPS = 4;
constexpr int CV_SHIFTS = 15;
constexpr int CV_MAX_Q = 12;    // source towers (3 k-chunks)
constexpr int CV_MAX_P = 64;    // target towers (8 groups of 8)

__device__ __forceinline__ void mma_u8(int (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc += a * b with a, b 32-bit (one wide multiply-add): folds a 32-bit
// partial sum into a 64-bit word at a byte shift b = 2^(8k).
__device__ __forceinline__ void mad_wide(u64& acc, uint32_t a, uint32_t b) {
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(acc) : "r"(a), "r"(b));
}

__device__ __forceinline__ u64 bswap64(u64 v) {
    return ((u64)__byte_perm((uint32_t)v, 0, 0x0123) << 32) | __byte_perm((uint32_t)(v >> 32), 0, 0x0123);
}

// Bytes off..off+3 of the 8-byte value r (zero outside 0..7) as one word.
__device__ __forceinline__ uint32_t byte_window(u64 r, int off) {
    if (off >= 8 || off <= -4) return 0u;
    return off >= 0 ? (uint32_t)(r >> (8 * off)) : (uint32_t)(r << (-8 * off));
}

template <int C>
__global__ void __launch_bounds__(CV_WARPS * 32)
k_approx_switch_mma(const u64* __restrict__ src, u64* __restrict__ dst, const u64* __restrict__ qhi,
                    const u64* __restrict__ qhip, const u64* __restrict__ qm, const u64* __restrict__ qmp,
                    const u64* __restrict__ p, const u64* __restrict__ mulo, const u64* __restrict__ muhi,
                    uint32_t sizeQ, uint32_t sizeP, uint32_t n) {
    constexpr int XW = 4 * C;                     // staged towers per coefficient (padded)
    const int groups = (int)(sizeP + 7) / 8;
    extern __shared__ __align__(16) uint2 cv_sm[];
    uint2* bw = cv_sm;                                            // [CV_SHIFTS][C][groups][32]
    u64* xs = reinterpret_cast<u64*>(bw + CV_SHIFTS * C * groups * 32);   // [warps][16][XW]
    u64* os = xs + CV_WARPS * 16 * XW;                            // [warps][8][16]

    // B fragments: lane (g, t), target j = 8*grp + g, towers i0 = 4c + t/2 (b0) and i0 + 2 (b1),
    // bytes a = 4*(t%2) + e of x meet byte s - a of M[i][j]; with r = bswap(M) that byte is
    // byte 7 - s + a of r, so the four bytes are one window of r.
    const int nb = CV_SHIFTS * C * groups * 32;
    for (int e = threadIdx.x; e < nb; e += blockDim.x) {
        const int lane = e % 32, grp = (e / 32) % groups, c = (e / (32 * groups)) % C, s = e / (32 * groups * C);
        const int g = lane >> 2, t = lane & 3;
        const int j = 8 * grp + g;
        const int off = 7 - s + 4 * (t & 1);
        uint32_t w[2] = {0u, 0u};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 4 * c + 2 * h + (t >> 1);
            if (i < (int)sizeQ && j < (int)sizeP) w[h] = byte_window(bswap64(qmp[(size_t)i * sizeP + j]), off);
        }
        bw[e] = make_uint2(w[0], w[1]);
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    u64* x = xs + warp * 16 * XW;
    u64* o = os + warp * 128;
    const uint32_t tiles = n / 16;
    for (uint32_t tile = blockIdx.x * CV_WARPS + warp; tile < tiles; tile += gridDim.x * CV_WARPS) {
        const uint32_t n0 = tile * 16;
        // stage x_i = shoup(a_i, QHatInv_i) for the tile (zero past sizeQ)
        {
            const int row = lane & 15;
            for (int i = lane >> 4; i < XW; i += 2)
                x[row * XW + i] = i < (int)sizeQ ? shoup(src[(size_t)i * n + n0 + row], qhi[i], qhip[i], qm[i]) : 0;
        }
        __syncwarp();
        uint32_t a[C][4];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const uint32_t* x32 = reinterpret_cast<const uint32_t*>(x);
            a[c][0] = x32[2 * (g * XW + 4 * c + (t >> 1)) + (t & 1)];
            a[c][1] = x32[2 * ((g + 8) * XW + 4 * c + (t >> 1)) + (t & 1)];
            a[c][2] = x32[2 * (g * XW + 4 * c + 2 + (t >> 1)) + (t & 1)];
            a[c][3] = x32[2 * ((g + 8) * XW + 4 * c + 2 + (t >> 1)) + (t & 1)];
        }
        for (int grp = 0; grp < groups; ++grp) {
            u64 acc[4][4];
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int h = 0; h < 4; ++h) acc[v][h] = 0;
#pragma unroll
            for (int s = 0; s < CV_SHIFTS; ++s) {
                int cf[4] = {0, 0, 0, 0};
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const uint2 b = bw[((s * C + c) * groups + grp) * 32 + lane];
                    mma_u8(cf, a[c], b.x, b.y);
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[v][s >> 2] += (u64)(uint32_t)cf[v] << (8 * (s & 3));
            }
            // S = acc0 + acc1 2^32 + acc2 2^64 + acc3 2^96 (< 2^125), then Barrett mod p_j
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int jl = 2 * t + (v & 1);
                const int j = 8 * grp + jl;
                u64 lo = acc[v][0], hi = acc[v][2] + (acc[v][3] << 32);
                add_wide(lo, hi, acc[v][1] << 32, acc[v][1] >> 32);
                u64 r = 0;
                if (j < (int)sizeP) {
                    ModC m;
                    m.q = p[j]; m.two_q = 2 * m.q; m.mu_lo = mulo[j]; m.mu_hi = muhi[j];
                    r = barrett(lo, hi, m);
                }
                o[jl * 16 + g + ((v >> 1) << 3)] = r;
            }
            __syncwarp();
            // coalesced store: two targets per pass, 16 consecutive coefficients each
#pragma unroll
            for (int pass = 0; pass < 4; ++pass) {
                const int jl = 2 * pass + (lane >> 4);
                const int j = 8 * grp + jl;
                if (j < (int)sizeP) dst[(size_t)j * n + n0 + (lane & 15)] = o[jl * 16 + (lane & 15)];
            }
            __syncwarp();
        }
    }
}

template <int C>
size_t cv_smem(uint32_t sizeP) {
    const int groups = (int)(sizeP + 7) / 8;
    return (size_t)CV_SHIFTS * C * groups * 32 * sizeof(uint2) + (size_t)CV_WARPS * 16 * 4 * C * 8 +
           (size_t)CV_WARPS * 128 * 8;
}

template <int C>
cudaError_t cv_launch(const u64* src, u64* dst, const u64* qhi, const u64* qhip, const u64* qm, const u64* qmp,
                      const u64* p, const u64* mulo, const u64* muhi, uint32_t sizeQ, uint32_t sizeP, uint32_t n,
                      cudaStream_t s) {
    static gfx::DeviceOnce attrs;
    attrs([] {
        cudaFuncSetAttribute(k_approx_switch_mma<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)cv_smem<C>(CV_MAX_P));
    });
    const uint32_t tiles = n / 16;
    const unsigned grid = (unsigned)std::min<uint32_t>((tiles + CV_WARPS - 1) / CV_WARPS,
                                                        (uint32_t)gfx::current_sm_count() * 8u);
    k_approx_switch_mma<C><<<grid, CV_WARPS * 32, cv_smem<C>(sizeP), s>>>(src, dst, qhi, qhip, qm, qmp, p, mulo,
                                                                         muhi, sizeQ, sizeP, n);
    return cudaGetLastError();
}


// ---------------------------------------------------------------- tcgen05 form
// The same byte-limb products on the 5th-generation tensor cores: per tile of
// 128 coefficients, one elected thread issues tcgen05.mma kind::i8 (M = 128
// coefficients, K = 32 bytes per instruction, N = 16 columns per target: the
// fifteen shifts s and one zero column) with A (the bytes of x) and B (the
// shifted bytes of M) in shared memory in the canonical K-major layout without
// swizzle: byte b of row r at (r % 8) * 16 + (r / 8) * 256 + (b / 16) * 128.
// The 32-bit partial sums land in tensor memory (row r = lane r, column
// 16 * target + s); every thread then reads its row's sixteen columns per
// target (tcgen05.ld 32x32b, two targets per wait), folds them into four
// 64-bit words, combines them into 128 bits and reduces, writing 32
// consecutive coefficients per warp. Targets go in chunks of at most 8 (128
// tensor-memory columns per CTA), up to four CTAs per SM, so one CTA's MMA
// and tile loads overlap the others' reductions; the next tile's inputs are
// loaded into registers before the current tile's MMA is awaited. The wait on
// each MMA batch is bounded (about two seconds of %globaltimer); on expiry the
// CTA records an error in g_cv_err, waits (bounded) once more, frees its
// tensor memory and returns.
constexpr int TC_THREADS = 256;
constexpr int TC_M = 128;
constexpr int TC_CHUNK = 8;          // targets per MMA batch
constexpr int TC_COLS = 128;         // tensor-memory columns per CTA (16 per target)
constexpr int TC_MIN_SMEM = 46 * 1024;   // at most four CTAs (4 x 128 columns) on an SM

__device__ u32 g_cv_err;

__device__ __forceinline__ u32 sm_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ u64 umma_desc(u32 addr) {
    // start address, leading (K) byte offset 128, stride (8-row) byte offset 256,
    // descriptor version 1, no swizzle
    return (u64)((addr >> 4) & 0x3FFFu) | ((u64)(128u >> 4) << 16) | ((u64)(256u >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool cv_mbar_test(u32 bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool cv_mbar_wait(u32 bar, u32 parity) {
    if (cv_mbar_test(bar, parity)) return true;
    u64 t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (u32 k = 1;; ++k) {
        if (cv_mbar_test(bar, parity)) return true;
        if ((k & 63) == 0) {
            u64 t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (t - t0 > 2000000000ull) return false;
        }
    }
}

__device__ __forceinline__ void tc_ld16(u32 taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tc_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// One 16-byte unit of A or B for the canonical layout: row r, K-half h, at
// base + (r % 8) * 16 + (r / 8) * 256 + h * 128.
__device__ __forceinline__ u32 canon_off(int r, int h) { return (u32)((r & 7) * 16 + (r >> 3) * 256 + h * 128); }

// The sixteen partial sums of one output (fifteen shifts) -> the exact sum -> mod p_j.
__device__ __forceinline__ u64 tc_reduce(const uint32_t (&cs)[16], const ModC& m) {
    u64 acc4[4] = {0, 0, 0, 0};
#pragma unroll
    for (int sft = 0; sft < 15; ++sft) mad_wide(acc4[sft >> 2], cs[sft], 1u << (8 * (sft & 3)));
    u64 lo = acc4[0], hi = acc4[2] + (acc4[3] << 32);
    add_wide(lo, hi, acc4[1] << 32, acc4[1] >> 32);
    return barrett(lo, hi, m);
}

template <int KS>
__global__ void __launch_bounds__(TC_THREADS, 4)
k_approx_switch_tc(const u64* __restrict__ src, u64* __restrict__ dst, const u64* __restrict__ qhi,
                   const u64* __restrict__ qhip, const u64* __restrict__ qm, const u64* __restrict__ qmp,
                   const u64* __restrict__ p, const u64* __restrict__ mulo, const u64* __restrict__ muhi,
                   uint32_t sizeQ, uint32_t sizeP, uint32_t n) {
    extern __shared__ __align__(1024) unsigned char tc_sm[];
    const int chunks = (int)(sizeP + TC_CHUNK - 1) / TC_CHUNK;
    unsigned char* A = tc_sm;                                   // [KS][4096]
    unsigned char* B = tc_sm + KS * 4096;                       // [chunk][KS][Nc * 32]
    const u32 b_bytes = (u32)KS * 32u * 16u * sizeP;            // sum over chunks of KS * Nc * 32
    u64* bar = reinterpret_cast<u64*>(B + ((b_bytes + 15) & ~15u));
    u32* tmem_slot = reinterpret_cast<u32*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // B: chunk c, step ks, row nr = 16 * jl + s, K-half h: towers i0 = 4 ks + 2 h and i0 + 1,
    // bytes a = 0..7 of each hold byte (s - a) of M[i][j], a window of bswap(M[i][j]).
    {
        u32 off = 0;
        for (int c = 0; c < chunks; ++c) {
            const int tc = min(TC_CHUNK, (int)sizeP - TC_CHUNK * c);
            const int nc = 16 * tc;
            for (int e = tid; e < KS * nc * 2; e += TC_THREADS) {
                const int h = e & 1, nr = (e >> 1) % nc, ks = (e >> 1) / nc;
                const int jl = nr >> 4, s = nr & 15, j = TC_CHUNK * c + jl;
                u64 w[2] = {0, 0};
#pragma unroll
                for (int d = 0; d < 2; ++d) {
                    const int i = 4 * ks + 2 * h + d;
                    if (s < 15 && i < (int)sizeQ) {
                        const u64 r = bswap64(qmp[(size_t)i * sizeP + j]);
                        const int sh = 7 - s;
                        w[d] = sh >= 0 ? (r >> (8 * sh)) : (r << (-8 * sh));
                    }
                }
                *reinterpret_cast<uint4*>(B + off + ks * nc * 32 + canon_off(nr, h)) =
                    make_uint4((u32)w[0], (u32)(w[0] >> 32), (u32)w[1], (u32)(w[1] >> 32));
            }
            off += (u32)KS * nc * 32;
        }
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sm_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sm_u32(tmem_slot)),
                     "r"(TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const u32 tmem = *tmem_slot;
    const u32 barp = sm_u32(bar);
    u32 phase = 0;
    bool ok = true;

    // A staging: thread -> row (tid % 128) and tower pairs pr = tid / 128, +2, ...; the raw
    // residues of the next tile are loaded one tile ahead
    const int row = tid & (TC_M - 1);
    const int pr0 = tid >> 7;
    const uint32_t tiles = n / TC_M;
    u64 raw[KS][2];
    auto load_raw = [&](uint32_t tile) {
#pragma unroll
        for (int q = 0; q < KS; ++q)
#pragma unroll
            for (int d = 0; d < 2; ++d) {
                const int i = 2 * (pr0 + 2 * q) + d;
                raw[q][d] = (i < (int)sizeQ && tile < tiles) ? src[(size_t)i * n + (size_t)tile * TC_M + row] : 0;
            }
    };
    load_raw(blockIdx.x);
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t n0 = tile * TC_M;
        // A: x_i = shoup(a_i, QHatInv_i) as bytes; pair pr = towers (2 pr, 2 pr + 1)
#pragma unroll
        for (int q = 0; q < KS; ++q) {
            const int pr = pr0 + 2 * q;
            u64 x[2];
#pragma unroll
            for (int d = 0; d < 2; ++d) {
                const int i = 2 * pr + d;
                x[d] = i < (int)sizeQ ? shoup(raw[q][d], qhi[i], qhip[i], qm[i]) : 0;
            }
            *reinterpret_cast<uint4*>(A + (pr >> 1) * 4096 + canon_off(row, pr & 1)) =
                make_uint4((u32)x[0], (u32)(x[0] >> 32), (u32)x[1], (u32)(x[1] >> 32));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        load_raw(tile + gridDim.x);
        u32 boff = 0;
        for (int c = 0; c < chunks && ok; ++c) {
            const int tc = min(TC_CHUNK, (int)sizeP - TC_CHUNK * c);
            const int nc = 16 * tc;
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();   // A written (first chunk), previous chunk's tensor-memory reads done
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (tid == 0) {
                const u32 idesc = (2u << 4) | ((u32)(nc >> 3) << 17) | ((u32)(TC_M >> 4) << 24);
#pragma unroll
                for (int ks = 0; ks < KS; ++ks) {
                    const u64 ad = umma_desc(sm_u32(A + ks * 4096));
                    const u64 bd = umma_desc(sm_u32(B + boff + ks * nc * 32));
                    const u32 acc = ks > 0 ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                        "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                        : "memory");
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(barp)
                             : "memory");
            }
            // every thread must agree before leaving, so the verdict goes through a barrier
            if (!__syncthreads_and(cv_mbar_wait(barp, phase))) {
                if (tid == 0) atomicOr(&g_cv_err, 1u);
                ok = false;
                break;
            }
            phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // epilogue: warp quadrant q reads rows 32q..32q+31; warps q and q+4 split the
            // chunk's targets (jl = half, half + 2, ...), two per tensor-memory wait
            const int q = warp & 3;
            const u32 r_out = (u32)(32 * q + lane);
            const u32 tq = tmem + ((u32)(32 * q) << 16);
            for (int jl = warp >> 2; jl < tc; jl += 4) {
                uint32_t c0[16], c1[16];
                const bool two = jl + 2 < tc;
                tc_ld16(tq + (u32)(16 * jl), c0);
                if (two) tc_ld16(tq + (u32)(16 * (jl + 2)), c1);
                tc_ld_wait();
                const int j = TC_CHUNK * c + jl;
                ModC m;
                m.q = p[j]; m.two_q = 2 * m.q; m.mu_lo = mulo[j]; m.mu_hi = muhi[j];
                dst[(size_t)j * n + n0 + r_out] = tc_reduce(c0, m);
                if (two) {
                    m.q = p[j + 2]; m.two_q = 2 * m.q; m.mu_lo = mulo[j + 2]; m.mu_hi = muhi[j + 2];
                    dst[(size_t)(j + 2) * n + n0 + r_out] = tc_reduce(c1, m);
                }
            }
            boff += (u32)KS * nc * 32;
        }
    }
    if (!ok) {
        // the batch never completed: wait once more (bounded) before freeing its tensor memory
        cv_mbar_wait(barp, phase);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS) : "memory");
    }
}

template <int KS>
size_t tc_smem(uint32_t sizeP) {
    const size_t b = (size_t)KS * 32 * 16 * sizeP;
    const size_t need = (size_t)KS * 4096 + ((b + 15) & ~(size_t)15) + 16 + 1024;   // + base alignment slack
    return std::max<size_t>(need, TC_MIN_SMEM);
}

template <int KS>
cudaError_t tc_launch(const u64* src, u64* dst, const u64* qhi, const u64* qhip, const u64* qm, const u64* qmp,
                      const u64* p, const u64* mulo, const u64* muhi, uint32_t sizeQ, uint32_t sizeP, uint32_t n,
                      cudaStream_t s) {
    static gfx::DeviceOnce attrs;
    attrs([] {
        cudaFuncSetAttribute(k_approx_switch_tc<KS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc_smem<KS>(CV_MAX_P));
    });
    const uint32_t tiles = n / TC_M;
    const uint32_t per_sm = (uint32_t)std::max<size_t>(1, std::min<size_t>(4, (227u * 1024u) / tc_smem<KS>(sizeP)));
    const unsigned grid = (unsigned)std::min<uint32_t>(tiles, per_sm * (uint32_t)gfx::current_sm_count());
    k_approx_switch_tc<KS><<<grid, TC_THREADS, tc_smem<KS>(sizeP), s>>>(src, dst, qhi, qhip, qm, qmp, p, mulo, muhi,
                                                                        sizeQ, sizeP, n);
    return cudaGetLastError();
}

}  // namespace

namespace cv {

bool tcgen05_shape(uint32_t sizeQ, uint32_t sizeP, uint32_t n) {
    return sizeQ >= 1 && sizeQ <= CV_MAX_Q && sizeP >= 1 && sizeP <= CV_MAX_P && n && n % TC_M == 0;
}

cudaError_t approx_switch_tcgen05(const uint64_t* d_src, uint64_t* d_dst, const uint64_t* qhi, const uint64_t* qhip,
                                  const uint64_t* q, const uint64_t* qmp, const uint64_t* p, const uint64_t* mulo,
                                  const uint64_t* muhi, uint32_t sizeQ, uint32_t sizeP, uint32_t n, cudaStream_t s) {
    const int ks = (int)(sizeQ + 3) / 4;
    return ks == 1 ? tc_launch<1>(d_src, d_dst, qhi, qhip, q, qmp, p, mulo, muhi, sizeQ, sizeP, n, s)
         : ks == 2 ? tc_launch<2>(d_src, d_dst, qhi, qhip, q, qmp, p, mulo, muhi, sizeQ, sizeP, n, s)
                   : tc_launch<3>(d_src, d_dst, qhi, qhip, q, qmp, p, mulo, muhi, sizeQ, sizeP, n, s);
}

}  // namespace cv

extern "C" int gpufhe_approx_switch(const uint64_t* d_src, uint64_t* d_dst, const uint64_t* d_QHatInvModq,
                                    const uint64_t* d_QHatInvModqPrecon, const uint64_t* d_q, const uint64_t* d_QHatModp,
                                    const uint64_t* d_p, const uint64_t* d_mu_lo, const uint64_t* d_mu_hi,
                                    uint32_t sizeQ, uint32_t sizeP, uint32_t n, int form, cudaStream_t s) {
    if (!d_src || !d_dst || !d_QHatInvModq || !d_QHatInvModqPrecon || !d_q || !d_QHatModp || !d_p || !d_mu_lo ||
        !d_mu_hi) {
        gfx::set_error("gpufhe_approx_switch: null argument");
        return GPUFHE_EINVAL;
    }
    const bool shape_ok = form == GPUFHE_CONVERT_TCGEN05   ? cv::tcgen05_shape(sizeQ, sizeP, n)
                        : form == GPUFHE_CONVERT_MMA_SYNC ? (sizeQ >= 1 && sizeQ <= CV_MAX_Q && sizeP >= 1 &&
                                                             sizeP <= CV_MAX_P && n && n % 16 == 0)
                        : form == GPUFHE_CONVERT_INTEGER  ? (sizeQ >= 1 && sizeP >= 1 && n)
                                                          : false;
    if (!shape_ok) {
        gfx::set_error("gpufhe_approx_switch: unknown form, or a shape it does not take (tcgen05: sizeQ <= 12, "
                       "sizeP <= 64, n a multiple of 128; mma.sync: the same with n a multiple of 16)");
        return GPUFHE_EINVAL;
    }
    cudaError_t e;
    if (form == GPUFHE_CONVERT_TCGEN05) {
        e = cv::approx_switch_tcgen05(d_src, d_dst, d_QHatInvModq, d_QHatInvModqPrecon, d_q, d_QHatModp, d_p, d_mu_lo,
                                      d_mu_hi, sizeQ, sizeP, n, s);
    } else if (form == GPUFHE_CONVERT_INTEGER) {
        e = cv::approx_switch_integer(d_src, d_dst, d_QHatInvModq, d_QHatInvModqPrecon, d_q, d_QHatModp, d_p, d_mu_lo,
                                      d_mu_hi, sizeQ, sizeP, n, s);
    } else {
        const int ks = (int)(sizeQ + 3) / 4;
        auto go = [&](auto launch) {
            return launch(d_src, d_dst, d_QHatInvModq, d_QHatInvModqPrecon, d_q, d_QHatModp, d_p, d_mu_lo, d_mu_hi,
                          sizeQ, sizeP, n, s);
        };
        e = ks == 1 ? go(cv_launch<1>) : ks == 2 ? go(cv_launch<2>) : go(cv_launch<3>);
    }
    if (e != cudaSuccess) {
        gfx::set_error(std::string("gpufhe_approx_switch: ") + cudaGetErrorString(e));
        return GPUFHE_ECUDA;
    }
    return GPUFHE_OK;
}

extern "C" int gpufhe_approx_switch_status(uint32_t* out) {
    if (!out) return GPUFHE_EINVAL;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpyFromSymbol(out, g_cv_err, sizeof(u32));
    const u32 zero = 0;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_cv_err, &zero, sizeof(u32));
    if (e != cudaSuccess) {
        gfx::set_error(std::string("gpufhe_approx_switch_status: ") + cudaGetErrorString(e));
        return GPUFHE_ECUDA;
    }
    return GPUFHE_OK;
}
