// Baby-step giant-step homomorphic linear transform over the batched
// pipeline: y = sum_g rot_{g*n1}( sum_b diag[g*n1+b] (.) rot_b(x) ), the
// sequence of the reference's tests/test_c2s_bsgs.cpp:129-151 (rotate_ct per
// baby and giant step, ct_mul_pt + ct_add_ct for the inner sums,
// ptops.cpp:13-26). All baby rotations run as one batched plan (optionally
// hoisted: one ModUp shared by all of them), all inner sums as one kernel, all
// giant rotations as one batched plan, and the final sum as one kernel.
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "pipeline.hpp"

gfx::Context* gpufhe_impl(gpufhe_ctx* h);

namespace {

// out[g][c] = sum_b diag[g*n1+b] (.) bab[b][c] mod q_t over L towers of n
// words: grid.z = giant step g, grid.y = component c; null diagonals skipped.
__global__ void k_bsgs_inner(u64* const* __restrict__ outs, const u64* const* __restrict__ bab,
                             const u64* const* __restrict__ diag, const ModC* __restrict__ mod, uint32_t L,
                             uint32_t n, uint32_t n1) {
    const uint32_t g = blockIdx.z, c = blockIdx.y;
    u64* out = outs[2 * g + c];
    const size_t total = (size_t)L * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const ModC m = mod[e / n];
        u64 r = 0;
        for (uint32_t b = 0; b < n1; ++b) {
            const u64* d = diag[(size_t)g * n1 + b];
            if (!d) continue;
            r += mulmod(bab[2 * b + c][e], d[e], m);
            r = csub(r, m.q);
        }
        out[e] = r;
    }
}

// out_c = sum_k parts[k][c] mod q_t
__global__ void k_bsgs_sum(u64* __restrict__ out0, u64* __restrict__ out1, const u64* const* __restrict__ parts,
                           uint32_t nparts, const ModC* __restrict__ mod, uint32_t L, uint32_t n) {
    const uint32_t c = blockIdx.y;
    u64* out = c ? out1 : out0;
    const size_t total = (size_t)L * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const u64 q = mod[e / n].q;
        u64 r = 0;
        for (uint32_t k = 0; k < nparts; ++k) r = csub(r + parts[2 * k + c][e], q);
        out[e] = r;
    }
}

uint64_t galois_of(uint32_t r, uint32_t n) {
    const uint64_t M = 2ull * n;
    uint64_t k = 1;
    for (uint32_t t = 0; t < r; ++t) k = (k * 5) % M;
    return k;
}

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(size_t bytes) {
        if (bytes && cudaMalloc(&p, bytes) != cudaSuccess) {
            p = nullptr;
            throw std::runtime_error("lintrans: device allocation failed");
        }
    }
    ~DevBuf() { if (p) cudaFree(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

}  // namespace

extern "C" int gpufhe_lintrans_bsgs(gpufhe_ctx* h, uint32_t level, const uint64_t* d_c0, const uint64_t* d_c1,
                                    uint32_t n1, uint32_t n2, const uint64_t* const* diag, int hoisted,
                                    uint64_t* d_out0, uint64_t* d_out1, cudaStream_t s) {
    gfx::Context* c = gpufhe_impl(h);
    if (!c || !d_c0 || !d_c1 || !diag || !d_out0 || !d_out1) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (level < 1 || level > c->fullQ() || n1 < 1 || n2 < 1 || (uint64_t)n1 * n2 > 4096) {
        gfx::set_error("gpufhe_lintrans_bsgs: level or step counts out of range");
        return GPUFHE_EINVAL;
    }
    try {
        const uint32_t n = c->n(), L = level;
        const size_t T = (size_t)L * n;
        for (uint32_t b = 1; b < n1; ++b)
            if (!c->key(galois_of(b, n))) throw std::invalid_argument("missing rotation key for a baby step");
        for (uint32_t g = 1; g < n2; ++g)
            if (!c->key(galois_of(g * n1, n))) throw std::invalid_argument("missing rotation key for a giant step");
        // scratch: baby outputs (n1-1), inner sums n2, giant outputs (n2-1), two components each
        const size_t nbuf = 2 * ((size_t)(n1 - 1) + n2 + (n2 - 1));
        DevBuf scratch(nbuf * T * 8);
        u64* base = static_cast<u64*>(scratch.p);
        auto buf = [&](size_t k) { return base + k * T; };
        std::vector<const u64*> bab(2 * n1);
        bab[0] = d_c0;
        bab[1] = d_c1;
        for (uint32_t b = 1; b < n1; ++b) { bab[2 * b] = buf(2 * (b - 1)); bab[2 * b + 1] = buf(2 * (b - 1) + 1); }
        const size_t inner0 = 2 * (size_t)(n1 - 1), giant0 = inner0 + 2 * (size_t)n2;
        std::vector<u64*> inner(2 * n2);
        for (uint32_t g = 0; g < n2; ++g) { inner[2 * g] = buf(inner0 + 2 * g); inner[2 * g + 1] = buf(inner0 + 2 * g + 1); }
        // 1. baby rotations, one batch
        std::unique_ptr<pl::Plan> baby;
        if (n1 > 1) {
            std::vector<pl::Op> ops(n1 - 1);
            for (uint32_t b = 1; b < n1; ++b) {
                pl::Op& op = ops[b - 1];
                op.L = L;
                op.mode = hoisted ? pl::HROT : pl::ROT;
                op.galois = op.key_id = galois_of(b, n);
                op.in[0] = d_c0;
                op.in[1] = d_c1;
                op.out[0] = const_cast<u64*>(bab[2 * b]);
                op.out[1] = const_cast<u64*>(bab[2 * b + 1]);
            }
            baby = pl::build_plan(*c, ops, nullptr, 0);
            pl::tune(*baby, s, false);
            ck(pl::launch(*baby, s), "baby rotations");
        }
        // 2. inner sums, one kernel over every giant step
        DevBuf tables((2 * n1 + (size_t)n1 * n2 + 2 * n2 + 2 * n2) * sizeof(void*));
        void** dt = static_cast<void**>(tables.p);
        std::vector<const void*> host(2 * n1 + (size_t)n1 * n2 + 4 * n2, nullptr);
        for (uint32_t k = 0; k < 2 * n1; ++k) host[k] = bab[k];
        for (size_t k = 0; k < (size_t)n1 * n2; ++k) host[2 * n1 + k] = diag[k];
        for (uint32_t k = 0; k < 2 * n2; ++k) host[2 * n1 + (size_t)n1 * n2 + k] = inner[k];
        // final-sum parts: inner sum 0, then the giant outputs
        const size_t pbase = 2 * n1 + (size_t)n1 * n2 + 2 * n2;
        host[pbase] = inner[0];
        host[pbase + 1] = inner[1];
        for (uint32_t g = 1; g < n2; ++g) {
            host[pbase + 2 * g] = buf(giant0 + 2 * (g - 1));
            host[pbase + 2 * g + 1] = buf(giant0 + 2 * (g - 1) + 1);
        }
        ck(cudaMemcpyAsync(dt, host.data(), host.size() * sizeof(void*), cudaMemcpyHostToDevice, s), "tables");
        const unsigned gx = (unsigned)std::min<size_t>((T + 255) / 256, 1184);
        k_bsgs_inner<<<dim3(gx, 2, n2), 256, 0, s>>>(reinterpret_cast<u64* const*>(dt + 2 * n1 + (size_t)n1 * n2),
                                                    reinterpret_cast<const u64* const*>(dt),
                                                    reinterpret_cast<const u64* const*>(dt + 2 * n1), c->dev().mod, L,
                                                    n, n1);
        ck(cudaGetLastError(), "inner sums");
        // 3. giant rotations, one batch
        std::unique_ptr<pl::Plan> giant;
        if (n2 > 1) {
            std::vector<pl::Op> ops(n2 - 1);
            for (uint32_t g = 1; g < n2; ++g) {
                pl::Op& op = ops[g - 1];
                op.L = L;
                op.mode = pl::ROT;
                op.galois = op.key_id = galois_of(g * n1, n);
                op.in[0] = inner[2 * g];
                op.in[1] = inner[2 * g + 1];
                op.out[0] = buf(giant0 + 2 * (g - 1));
                op.out[1] = buf(giant0 + 2 * (g - 1) + 1);
            }
            giant = pl::build_plan(*c, ops, nullptr, 0);
            pl::tune(*giant, s, false);
            ck(pl::launch(*giant, s), "giant rotations");
        }
        // 4. y = inner_0 + sum of the giant outputs
        k_bsgs_sum<<<dim3(gx, 2), 256, 0, s>>>(d_out0, d_out1, reinterpret_cast<const u64* const*>(dt + pbase), n2,
                                              c->dev().mod, L, n);
        ck(cudaGetLastError(), "final sum");
        ck(cudaStreamSynchronize(s), "lintrans");
        return GPUFHE_OK;
    } catch (const std::invalid_argument& e) {
        gfx::set_error(e.what());
        return GPUFHE_EINVAL;
    } catch (const std::exception& e) {
        gfx::set_error(e.what());
        return GPUFHE_ECUDA;
    }
}
