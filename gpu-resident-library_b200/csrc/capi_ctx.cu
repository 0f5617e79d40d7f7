// extern "C" context and batched-transform entry points (include/gpufhe_b200.h).
#include <cstring>
#include <stdexcept>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "xform.cuh"

using gfx::Context;

struct gpufhe_ctx { Context* c; };

namespace {

// out = a * b mod q_t over [poly][tower][n] (plain residues in and out, the
// result LaunchRNSMultTower gives, rns_arith.cu:13-56). One block covers
// MUL_CHUNK words of one tower; each thread loads all its 16-byte pairs
// before it computes, so every thread has four loads of each operand in flight.
constexpr int MUL_NT = 256, MUL_VEC = 4, MUL_CHUNK = MUL_NT * 2 * MUL_VEC;

__global__ void __launch_bounds__(MUL_NT) k_rns_mult_batch(const u64* __restrict__ a, const u64* __restrict__ b,
                                                           u64* __restrict__ out, const ModC* __restrict__ mod,
                                                           uint32_t towers, uint32_t first, uint32_t n) {
    const size_t base = (size_t)blockIdx.x * MUL_CHUNK;
    const uint32_t t = (uint32_t)((base / n) % towers);
    const ModC m = mod[first + t];
    const ulonglong2* A = reinterpret_cast<const ulonglong2*>(a + base);
    const ulonglong2* B = reinterpret_cast<const ulonglong2*>(b + base);
    ulonglong2* O = reinterpret_cast<ulonglong2*>(out + base);
    ulonglong2 x[MUL_VEC], y[MUL_VEC];
#pragma unroll
    for (int k = 0; k < MUL_VEC; ++k) {
        x[k] = __ldcs(A + threadIdx.x + k * MUL_NT);
        y[k] = __ldcs(B + threadIdx.x + k * MUL_NT);
    }
#pragma unroll
    for (int k = 0; k < MUL_VEC; ++k) {
        ulonglong2 r;
        r.x = mulmod(x[k].x, y[k].x, m);
        r.y = mulmod(x[k].y, y[k].y, m);
        __stcs(O + threadIdx.x + k * MUL_NT, r);
    }
}

}  // namespace

#define GPUFHE_TRY(...)                                          \
    try { __VA_ARGS__ } catch (const std::invalid_argument& e) {        \
        gfx::set_error(e.what()); return GPUFHE_EINVAL;          \
    } catch (const std::length_error& e) {                       \
        gfx::set_error(e.what()); return GPUFHE_ENOMEM;          \
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
    Context::retire(h->c);   // deleted now, or when its last plan or server goes
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

int gpufhe_ctx_set_key_budget(gpufhe_ctx* h, uint64_t bytes) {
    if (!h) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    GPUFHE_TRY({
        h->c->set_key_budget(bytes);
        return GPUFHE_OK;
    })
}

int gpufhe_ctx_key_stats(const gpufhe_ctx* h, uint64_t* out) {
    if (!h || !out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    const auto st = h->c->key_stats();
    out[0] = st.known;
    out[1] = st.resident;
    out[2] = st.resident_bytes;
    out[3] = st.uploads;
    out[4] = st.evictions;
    out[5] = st.budget;
    return GPUFHE_OK;
}

int gpufhe_ctx_device_status(gpufhe_ctx* h, uint32_t* out) {
    if (!h || !out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    GPUFHE_TRY({
        u32* d = h->c->dev().err;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(h->c->device());
        cudaError_t e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(out, d, 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemset(d, 0, 4);
        cudaSetDevice(prev);
        if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
        return GPUFHE_OK;
    })
}

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
            j.fp = fp_tower(j.q) ? 1u : 0u;
            j.twd = j.fp ? (inverse ? D.twid : D.twfd) + (size_t)qi * n : nullptr;
            j.reserved = 0;
        }
    cudaError_t e = cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(xf::Job), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    cudaStreamSynchronize(s);
    e = xf_launch_ntt((const xf::Job*)d_jobs, nullptr, (int)jobs.size(), (int)c->logn(), inverse != 0, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

uint64_t gpufhe_ntt_job_bytes(void) { return sizeof(xf::Job); }

int gpufhe_rns_mult_batch(gpufhe_ctx* h, const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_out, uint32_t npolys,
                          uint32_t towers, uint32_t first_tower, cudaStream_t s) {
    if (!h || !d_a || !d_b || !d_out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    Context* c = h->c;
    if (first_tower + towers > c->fullQ() + c->K() || !towers) { gfx::set_error("tower range"); return GPUFHE_EINVAL; }
    const uint32_t n = c->n();
    if (n % MUL_CHUNK) { gfx::set_error("gpufhe_rns_mult_batch needs n >= 2048"); return GPUFHE_EINVAL; }
    if ((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_b) | reinterpret_cast<uintptr_t>(d_out)) & 15) {
        gfx::set_error("gpufhe_rns_mult_batch needs 16-byte aligned buffers");
        return GPUFHE_EINVAL;
    }
    const size_t words = (size_t)npolys * towers * n;
    if (!words) return GPUFHE_OK;
    k_rns_mult_batch<<<(unsigned)(words / MUL_CHUNK), MUL_NT, 0, s>>>(d_a, d_b, d_out, c->dev().mod, towers,
                                                                     first_tower, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

int gpufhe_ntt_run_jobs(gpufhe_ctx* h, const uint64_t* d_jobs, uint32_t njobs, int inverse, cudaStream_t s) {
    if (!h || !d_jobs) return GPUFHE_EINVAL;
    cudaError_t e = xf_launch_ntt((const xf::Job*)d_jobs, nullptr, (int)njobs, (int)h->c->logn(), inverse != 0, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

}  // extern "C"
