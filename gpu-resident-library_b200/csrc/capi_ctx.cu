// extern "C" context and batched-transform entry points (include/gpufhe_b200.h).
#include <cstring>
#include <stdexcept>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "xform.cuh"

using gfx::Context;

struct gpufhe_ctx { Context* c; };

#define GPUFHE_TRY(...)                                          \
    try { __VA_ARGS__ } catch (const std::invalid_argument& e) {        \
        gfx::set_error(e.what()); return GPUFHE_EINVAL;          \
    } catch (const std::exception& e) {                          \
        gfx::set_error(e.what()); return GPUFHE_ECUDA;           \
    }

Context* gpufhe_impl(gpufhe_ctx* h) { return h ? h->c : nullptr; }

extern "C" {

const char* gpufhe_last_error(void) {
    static thread_local std::string s;
    s = gfx::last_error();
    return s.c_str();
}

int gpufhe_ctx_create(uint32_t n, const uint64_t* Q, uint32_t fullQ, const uint64_t* P, uint32_t K,
                      uint32_t alpha, const uint64_t* roots_qp, int device, gpufhe_ctx** out) {
    if (!Q || !P || !out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    GPUFHE_TRY({
        std::vector<uint64_t> q(Q, Q + fullQ), p(P, P + K), r;
        if (roots_qp) r.assign(roots_qp, roots_qp + fullQ + K);
        auto* h = new gpufhe_ctx{new Context(n, q, p, alpha, r, device)};
        *out = h;
        return GPUFHE_OK;
    })
}

void gpufhe_ctx_destroy(gpufhe_ctx* h) {
    if (!h) return;
    delete h->c;
    delete h;
}

int gpufhe_ctx_roots(const gpufhe_ctx* h, uint64_t* out) {
    if (!h || !out) return GPUFHE_EINVAL;
    const auto& r = h->c->roots();
    std::memcpy(out, r.data(), r.size() * 8);
    return GPUFHE_OK;
}

int gpufhe_ctx_set_key(gpufhe_ctx* h, uint64_t key_id, const uint64_t* av, const uint64_t* bv) {
    if (!h || !av || !bv) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    GPUFHE_TRY({
        h->c->set_key(key_id, av, bv);
        return GPUFHE_OK;
    })
}

uint64_t gpufhe_ctx_resident_bytes(const gpufhe_ctx* h) { return h ? h->c->resident_bytes() : 0; }

int gpufhe_ntt_batch(gpufhe_ctx* h, uint64_t* d_data, uint32_t npolys, uint32_t towers, uint32_t first_tower,
                     int inverse, uint64_t* d_jobs, cudaStream_t s) {
    if (!h || !d_data || !d_jobs) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    Context* c = h->c;
    if (first_tower + towers > c->fullQ() + c->K()) { gfx::set_error("tower range"); return GPUFHE_EINVAL; }
    const auto& D = c->dev();
    const uint32_t n = c->n();
    std::vector<xf::Job> jobs((size_t)npolys * towers);
    std::vector<ModC> mods(D.QP);
    cudaMemcpy(mods.data(), D.mod, D.QP * sizeof(ModC), cudaMemcpyDeviceToHost);
    std::vector<u64> ninv(D.QP), ninvp(D.QP);
    cudaMemcpy(ninv.data(), D.ninv, D.QP * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(ninvp.data(), D.ninvp, D.QP * 8, cudaMemcpyDeviceToHost);
    for (uint32_t p = 0; p < npolys; ++p)
        for (uint32_t t = 0; t < towers; ++t) {
            const uint32_t qi = first_tower + t;
            xf::Job& j = jobs[(size_t)p * towers + t];
            j.x = d_data + ((size_t)p * towers + t) * n;
            j.tw = (inverse ? D.twi : D.twf) + (size_t)qi * n;
            j.w = j.wp = nullptr;
            j.q = mods[qi].q;
            j.scale = ninv[qi];
            j.scale_p = ninvp[qi];
        }
    cudaError_t e = cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(xf::Job), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    cudaStreamSynchronize(s);
    e = xf_launch_ntt((const xf::Job*)d_jobs, nullptr, (int)jobs.size(), (int)c->logn(), inverse != 0, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

uint64_t gpufhe_ntt_job_bytes(void) { return sizeof(xf::Job); }

int gpufhe_ntt_run_jobs(gpufhe_ctx* h, const uint64_t* d_jobs, uint32_t njobs, int inverse, cudaStream_t s) {
    if (!h || !d_jobs) return GPUFHE_EINVAL;
    cudaError_t e = xf_launch_ntt((const xf::Job*)d_jobs, nullptr, (int)njobs, (int)h->c->logn(), inverse != 0, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

}  // extern "C"
