// Batched ciphertext arithmetic without a keyswitch (include/gpufhe_b200.h,
// gpufhe_pointwise_batch): sums and differences of ciphertexts, products with
// an eval-form plaintext, plaintext sums and differences, and products with a
// small integer, over any mix of operations and levels in one launch.
//
// The reference runs each of these as a host loop over towers*n words with
// 128-bit % per product (src/ptops.cpp:13-26, and the add / subtract /
// scale-by-two loops its tests write around them, tests/test_evalmod.cpp:
// 100-113). Here one thread handles a word of one tower of one operation;
// the formulas (and so the bits) are the reference's:
//   add  s = a + b, s - q when s >= q      sub  a >= b ? a - b : a + q - b
//   mul  (a * b) mod q                     small (a * k) mod q
#include <stdexcept>
#include <vector>

#include "context.hpp"
#include "ntt.cuh"
#include "gpufhe_b200.h"

gfx::Context* gpufhe_impl(gpufhe_ctx* h);

namespace {

constexpr unsigned PW_NT = 256;

__device__ __forceinline__ u64 pw_add(u64 a, u64 b, u64 q) {
    const u64 s = a + b;
    return s >= q ? s - q : s;
}
__device__ __forceinline__ u64 pw_sub(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + q - b; }
// (a * b) mod q for any 64-bit a, b: operands reduced first, then one
// product. Canonical operands (the usual case) skip the two reductions, and
// for q < 2^50 their product runs on the FP64 pipe: an exact FP64 modular
// product of unsigned operands below q (|r| <= 2q), normalised to [0, q).
__device__ __forceinline__ u64 pw_mul(u64 a, u64 b, const ModC& m) {
    if (a >= m.q || b >= m.q) return mulmod(reduce64(a, m), reduce64(b, m), m);
    if (fp_tower(m.q)) {
        const ntt::FpAr ar{ntt::u2d(m.q), qinv_of(m)};
        return ar.out(ar.norm(ar.mulq<true>(ntt::u2d(a), ntt::u2d(b))));
    }
    return mulmod(a, b, m);
}

// blockIdx.y = operation, blockIdx.z = tower (towers beyond an operation's
// level do nothing).
__global__ void __launch_bounds__(PW_NT)
k_pointwise_batch(const gpufhe_pw_op* __restrict__ ops, const ModC* __restrict__ mod, uint32_t n) {
    const gpufhe_pw_op op = ops[blockIdx.y];
    const uint32_t t = blockIdx.z;
    if (t >= op.towers) return;
    const ModC m = mod[t];
    const u64 q = m.q;
    const size_t base = (size_t)t * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const size_t x = base + k;
        const u64 a0 = op.a0[x], a1 = op.a1[x];
        u64 r0 = a0, r1 = a1;
        switch (op.kind) {
            case GPUFHE_PW_ADD: r0 = pw_add(a0, op.b0[x], q); r1 = pw_add(a1, op.b1[x], q); break;
            case GPUFHE_PW_SUB: r0 = pw_sub(a0, op.b0[x], q); r1 = pw_sub(a1, op.b1[x], q); break;
            case GPUFHE_PW_MUL_PT: { const u64 p = op.b0[x]; r0 = pw_mul(a0, p, m); r1 = pw_mul(a1, p, m); } break;
            case GPUFHE_PW_ADD_PT: r0 = pw_add(a0, op.b0[x], q); break;
            case GPUFHE_PW_SUB_PT: r0 = pw_sub(a0, op.b0[x], q); break;
            case GPUFHE_PW_MUL_INT: r0 = pw_mul(a0, op.scalar, m); r1 = pw_mul(a1, op.scalar, m); break;
            default: break;
        }
        op.o0[x] = r0;
        op.o1[x] = r1;
    }
}

bool needs_b1(uint32_t kind) { return kind == GPUFHE_PW_ADD || kind == GPUFHE_PW_SUB; }
bool needs_b0(uint32_t kind) { return kind != GPUFHE_PW_MUL_INT; }

}  // namespace

extern "C" int gpufhe_pointwise_batch(gpufhe_ctx* h, uint32_t count, const gpufhe_pw_op* ops, cudaStream_t stream) {
    gfx::Context* c = gpufhe_impl(h);
    if (!c || (count && !ops)) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    if (count > 65535) { gfx::set_error("pointwise: at most 65535 operations per call"); return GPUFHE_EINVAL; }
    uint32_t maxt = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const gpufhe_pw_op& o = ops[i];
        if (o.kind > GPUFHE_PW_MUL_INT || !o.towers || o.towers > c->fullQ() || !o.a0 || !o.a1 || !o.o0 || !o.o1 ||
            (needs_b0(o.kind) && !o.b0) || (needs_b1(o.kind) && !o.b1)) {
            gfx::set_error("pointwise: bad operation (kind, towers or a null buffer)");
            return GPUFHE_EINVAL;
        }
        maxt = std::max(maxt, o.towers);
    }
    gpufhe_pw_op* d = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&d), count * sizeof(gpufhe_pw_op), stream);
    // a copy from pageable memory has read `ops` when it returns
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, ops, count * sizeof(gpufhe_pw_op), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        const uint32_t n = c->n();
        const unsigned gx = (unsigned)std::min<uint32_t>((n + PW_NT - 1) / PW_NT, 64);
        k_pointwise_batch<<<dim3(gx, count, maxt), PW_NT, 0, stream>>>(d, c->dev().mod, n);
        e = cudaGetLastError();
    }
    if (d) cudaFreeAsync(d, stream);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}
