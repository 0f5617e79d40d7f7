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

// Everything a transform needs, built once: scratch for the baby outputs,
// inner sums and giant outputs, the device pointer tables of the two sum
// kernels, and the batched baby / giant rotation plans (which pin their
// rotation keys while the plan lives). Launching enqueues four steps and
// nothing else, so a launch can be captured in a CUDA graph.
struct gpufhe_lintrans_plan {
    gfx::Context* ctx = nullptr;     // held for the plan's lifetime
    ~gpufhe_lintrans_plan() {
        baby.reset();
        giant.reset();
        tables.reset();
        scratch.reset();
        if (ctx) gfx::Context::drop(ctx);
    }
    uint32_t L = 0, n = 0, n1 = 0, n2 = 0;
    std::unique_ptr<DevBuf> scratch, tables;
    std::unique_ptr<pl::Plan> baby, giant;
    size_t inner_off = 0, diag_off = 0, parts_off = 0;
    u64 *out0 = nullptr, *out1 = nullptr;
    unsigned gx = 0;
};

namespace {

gpufhe_lintrans_plan* build_lintrans(gfx::Context* c, uint32_t level, const uint64_t* d_c0, const uint64_t* d_c1,
                                     uint32_t n1, uint32_t n2, const uint64_t* const* diag, int hoisted,
                                     uint64_t* d_out0, uint64_t* d_out1) {
    const uint32_t n = c->n(), L = level;
    const size_t T = (size_t)L * n;
    for (uint32_t b = 1; b < n1; ++b)
        if (!c->key(galois_of(b, n))) throw std::invalid_argument("missing rotation key for a baby step");
    for (uint32_t g = 1; g < n2; ++g)
        if (!c->key(galois_of(g * n1, n))) throw std::invalid_argument("missing rotation key for a giant step");
    auto pl_ = std::make_unique<gpufhe_lintrans_plan>();
    gpufhe_lintrans_plan& P = *pl_;
    c->hold();
    P.ctx = c;
    P.L = L;
    P.n = n;
    P.n1 = n1;
    P.n2 = n2;
    P.out0 = d_out0;
    P.out1 = d_out1;
    P.gx = (unsigned)std::min<size_t>((T + 255) / 256, 1184);
    // scratch: baby outputs (n1-1), inner sums n2, giant outputs (n2-1), two components each
    const size_t nbuf = 2 * ((size_t)(n1 - 1) + n2 + (n2 - 1));
    P.scratch = std::make_unique<DevBuf>(nbuf * T * 8);
    u64* base = static_cast<u64*>(P.scratch->p);
    auto buf = [&](size_t k) { return base + k * T; };
    std::vector<const u64*> bab(2 * n1);
    bab[0] = d_c0;
    bab[1] = d_c1;
    for (uint32_t b = 1; b < n1; ++b) { bab[2 * b] = buf(2 * (b - 1)); bab[2 * b + 1] = buf(2 * (b - 1) + 1); }
    const size_t inner0 = 2 * (size_t)(n1 - 1), giant0 = inner0 + 2 * (size_t)n2;
    std::vector<u64*> inner(2 * n2);
    for (uint32_t g = 0; g < n2; ++g) { inner[2 * g] = buf(inner0 + 2 * g); inner[2 * g + 1] = buf(inner0 + 2 * g + 1); }
    // baby rotations, one batch (optionally sharing one ModUp)
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
        P.baby = pl::build_plan(*c, ops, nullptr, 0);
    }
    // giant rotations of the inner sums, one batch
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
        P.giant = pl::build_plan(*c, ops, nullptr, 0);
    }
    // pointer tables: baby outputs, diagonals, inner sums, final-sum parts
    // (inner sum 0, then the giant outputs)
    P.diag_off = 2 * (size_t)n1;
    P.inner_off = P.diag_off + (size_t)n1 * n2;
    P.parts_off = P.inner_off + 2 * (size_t)n2;
    std::vector<const void*> host(P.parts_off + 2 * (size_t)n2, nullptr);
    for (uint32_t k = 0; k < 2 * n1; ++k) host[k] = bab[k];
    for (size_t k = 0; k < (size_t)n1 * n2; ++k) host[P.diag_off + k] = diag[k];
    for (uint32_t k = 0; k < 2 * n2; ++k) host[P.inner_off + k] = inner[k];
    host[P.parts_off] = inner[0];
    host[P.parts_off + 1] = inner[1];
    for (uint32_t g = 1; g < n2; ++g) {
        host[P.parts_off + 2 * g] = buf(giant0 + 2 * (g - 1));
        host[P.parts_off + 2 * g + 1] = buf(giant0 + 2 * (g - 1) + 1);
    }
    P.tables = std::make_unique<DevBuf>(host.size() * sizeof(void*));
    ck(cudaMemcpy(P.tables->p, host.data(), host.size() * sizeof(void*), cudaMemcpyHostToDevice), "tables");
    return pl_.release();
}

cudaError_t launch_lintrans(gpufhe_lintrans_plan& P, cudaStream_t s) {
    void** dt = static_cast<void**>(P.tables->p);
    if (P.baby) {
        pl::tune(*P.baby, s, false);   // cached or default schedule; no launch, safe under capture
        const cudaError_t e = pl::launch(*P.baby, s);
        if (e != cudaSuccess) return e;
    }
    k_bsgs_inner<<<dim3(P.gx, 2, P.n2), 256, 0, s>>>(reinterpret_cast<u64* const*>(dt + P.inner_off),
                                                    reinterpret_cast<const u64* const*>(dt),
                                                    reinterpret_cast<const u64* const*>(dt + P.diag_off),
                                                    P.ctx->dev().mod, P.L, P.n, P.n1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (P.giant) {
        pl::tune(*P.giant, s, false);
        e = pl::launch(*P.giant, s);
        if (e != cudaSuccess) return e;
    }
    k_bsgs_sum<<<dim3(P.gx, 2), 256, 0, s>>>(P.out0, P.out1, reinterpret_cast<const u64* const*>(dt + P.parts_off),
                                            P.n2, P.ctx->dev().mod, P.L, P.n);
    return cudaGetLastError();
}

int check_lintrans_args(gfx::Context* c, uint32_t level, const uint64_t* d_c0, const uint64_t* d_c1, uint32_t n1,
                        uint32_t n2, const uint64_t* const* diag, uint64_t* d_out0, uint64_t* d_out1) {
    if (!c || !d_c0 || !d_c1 || !diag || !d_out0 || !d_out1) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (level < 1 || level > c->fullQ() || n1 < 1 || n2 < 1 || (uint64_t)n1 * n2 > 4096) {
        gfx::set_error("gpufhe_lintrans_bsgs: level or step counts out of range");
        return GPUFHE_EINVAL;
    }
    return GPUFHE_OK;
}

}  // namespace

extern "C" {

int gpufhe_lintrans_plan_create(gpufhe_ctx* h, uint32_t level, const uint64_t* d_c0, const uint64_t* d_c1,
                                uint32_t n1, uint32_t n2, const uint64_t* const* diag, int hoisted,
                                uint64_t* d_out0, uint64_t* d_out1, gpufhe_lintrans_plan** out) {
    gfx::Context* c = gpufhe_impl(h);
    if (!out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    *out = nullptr;
    const int rc = check_lintrans_args(c, level, d_c0, d_c1, n1, n2, diag, d_out0, d_out1);
    if (rc) return rc;
    try {
        *out = build_lintrans(c, level, d_c0, d_c1, n1, n2, diag, hoisted, d_out0, d_out1);
        return GPUFHE_OK;
    } catch (const std::invalid_argument& e) {
        gfx::set_error(e.what());
        return GPUFHE_EINVAL;
    } catch (const std::length_error& e) {
        gfx::set_error(e.what());
        return GPUFHE_ENOMEM;
    } catch (const std::exception& e) {
        gfx::set_error(e.what());
        return GPUFHE_ECUDA;
    }
}

int gpufhe_lintrans_plan_launch(gpufhe_lintrans_plan* P, cudaStream_t s) {
    if (!P) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    const cudaError_t e = launch_lintrans(*P, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

void gpufhe_lintrans_plan_destroy(gpufhe_lintrans_plan* P) { delete P; }

int gpufhe_lintrans_bsgs(gpufhe_ctx* h, uint32_t level, const uint64_t* d_c0, const uint64_t* d_c1, uint32_t n1,
                         uint32_t n2, const uint64_t* const* diag, int hoisted, uint64_t* d_out0, uint64_t* d_out1,
                         cudaStream_t s) {
    gpufhe_lintrans_plan* P = nullptr;
    int rc = gpufhe_lintrans_plan_create(h, level, d_c0, d_c1, n1, n2, diag, hoisted, d_out0, d_out1, &P);
    if (rc) return rc;
    rc = gpufhe_lintrans_plan_launch(P, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    gpufhe_lintrans_plan_destroy(P);
    if (!rc && e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return rc;
}

}  // extern "C"
