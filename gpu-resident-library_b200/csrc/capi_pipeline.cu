// extern "C" batched-operation entry points (include/gpufhe_b200.h).
#include <cuda.h>

#include <memory>
#include <stdexcept>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "pipeline.hpp"

gfx::Context* gpufhe_impl(gpufhe_ctx* h);

struct gpufhe_plan {
    std::unique_ptr<pl::Plan> p;
};

namespace {
std::vector<pl::Op> to_ops(uint32_t nops, const gpufhe_op* ops) {
    std::vector<pl::Op> v(nops);
    for (uint32_t i = 0; i < nops; ++i) {
        v[i].L = ops[i].level;
        v[i].mode = ops[i].mode;
        v[i].key_id = ops[i].key_id;
        v[i].galois = ops[i].galois;
        for (int k = 0; k < 4; ++k) v[i].in[k] = ops[i].in[k];
        v[i].out[0] = ops[i].out[0];
        v[i].out[1] = ops[i].out[1];
    }
    return v;
}
}  // namespace

#define GPUFHE_TRY(...)                                                  \
    try { __VA_ARGS__ } catch (const std::invalid_argument& e) {         \
        gfx::set_error(e.what()); return GPUFHE_EINVAL;                  \
    } catch (const std::length_error& e) {                               \
        gfx::set_error(e.what()); return GPUFHE_ENOMEM;                  \
    } catch (const std::exception& e) {                                  \
        gfx::set_error(e.what()); return GPUFHE_ECUDA;                   \
    }

extern "C" {

uint64_t gpufhe_op_workspace_bytes(gpufhe_ctx* h, uint32_t level) {
    gfx::Context* c = gpufhe_impl(h);
    if (!c || level < 1 || level > c->fullQ()) return 0;
    return pl::op_workspace_words(*c, level) * 8;
}

int gpufhe_plan_create(gpufhe_ctx* h, uint32_t nops, const gpufhe_op* ops, uint64_t* d_ws, uint64_t ws_bytes,
                       gpufhe_plan** out) {
    gfx::Context* c = gpufhe_impl(h);
    if (!c || !ops || !out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    GPUFHE_TRY({
        auto pp = pl::build_plan(*c, to_ops(nops, ops), d_ws, ws_bytes / 8);
        *out = new gpufhe_plan{std::move(pp)};
        return GPUFHE_OK;
    })
}

int gpufhe_plan_launch(gpufhe_plan* plan, cudaStream_t s) {
    if (!plan) { gfx::set_error("null plan"); return GPUFHE_EINVAL; }
    pl::tune(*plan->p, s);
    cudaError_t e = pl::launch(*plan->p, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

int gpufhe_plan_launch_phase(gpufhe_plan* plan, uint32_t phase, cudaStream_t s) {
    if (!plan || phase >= (uint32_t)pl::NPHASE) { gfx::set_error("bad plan or phase"); return GPUFHE_EINVAL; }
    cudaError_t e = pl::launch(*plan->p, s, 1u << phase);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

uint32_t gpufhe_plan_schedule(const gpufhe_plan* plan) {
    if (!plan) return 0;
    const pl::Plan& p = *plan->p;
    return (uint32_t)p.p5_form | ((p.mix & 0x1ffu) == 0x1ffu ? 4u : 0u) | ((uint32_t)p.p3_form << 3) |
           (p.tuned ? 32u : 0u) | (p.p5_fp ? 64u : 0u) | ((p.p5_fp_form & 1) ? 128u : 0u) | ((p.mix & 0x1ffu) << 8) |
           (p.p5_split ? (1u << 17) : 0u) | (p.p5_fp_form >= 2 ? (1u << 18) : 0u);
}

int gpufhe_plan_set_schedule(gpufhe_plan* plan, uint32_t schedule) {
    if (!plan || ((schedule >> 3) & 3) > 2) {
        gfx::set_error("bad plan or schedule");
        return GPUFHE_EINVAL;
    }
    pl::Plan& p = *plan->p;
    p.p5_form = (int)(schedule & 3);
    if (p.p5_form == pl::P5_ASYNC && !pl::mac_async_ok(p.dc.dnum)) p.p5_form = pl::P5_REG128;
    if (p.p5_form == pl::P5_TMA && !pl::mac_tma_ok(p.dc.dnum)) p.p5_form = pl::P5_REG128;
    p.mix = (schedule & 4) ? 0x1ffu : (schedule >> 8) & 0x1ffu;
    p.p3_form = (int)((schedule >> 3) & 3);
    if (p.p3_form > 2) { gfx::set_error("bad P3 form"); return GPUFHE_EINVAL; }
    p.p5_fp = (schedule >> 6) & 1;
    p.p5_fp_form = ((schedule >> 18) & 1 ? 2 : 0) + (int)((schedule >> 7) & 1);
    if (p.p5_fp_form >= 2 && !pl::mac_tma_ok(p.dc.dnum)) p.p5_fp_form = 0;
    p.p5_split = (schedule >> 17) & 1;
    if (p.p5_split && !pl::ensure_side(p)) {
        gfx::set_error("gpufhe_plan_set_schedule: cannot create the second P5 stream");
        return GPUFHE_ECUDA;
    }
    p.tuned = true;
    return GPUFHE_OK;
}

uint32_t gpufhe_plan_kernel_count(const gpufhe_plan* plan) {
    if (!plan) return 0;
    uint32_t k = 0;
    const pl::Plan& p = *plan->p;
    for (int i = 0; i <= pl::NPHASE; ++i) {
        const int bit = i == pl::NPHASE ? 6 : i;   // the second P7 launch follows phase 7's choice
        if (i == 4) {   // P5: the integer form, and the FP64 form for 50-bit Q rows when chosen
            const uint32_t nfp = p.p5_fp ? p.job_cnt[4][1] : 0u;
            k += (p.job_cnt[4][0] + p.job_cnt[4][1] - nfp ? 1 : 0) + (nfp ? 1 : 0);
            continue;
        }
        if ((p.mix >> bit & 1) && p.job_cnt[i][2]) k += 1;
        else k += (p.job_cnt[i][0] ? 1 : 0) + (p.job_cnt[i][1] ? 1 : 0);
    }
    return k;
}

}  // extern "C"

namespace {
struct Copy {
    char* dst;
    const char* src;
    size_t bytes;
};
// Issues the copies in order. With `merge` (the host side is one buffer,
// walked in order), a copy joins the previous one when both its source and
// its destination continue the previous ranges and the device side stays
// inside one device allocation (cuMemGetAddressRange): a batch laid out
// contiguously on both sides moves in one large copy, which PCIe serves
// faster than many small ones.
// cuMemGetAddressRange through the runtime's driver entry point, so that the
// library carries no link-time dependency on the driver library; null when
// the entry point is unavailable (copies then stay piecewise).
using AddrRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
AddrRangeFn addr_range() {
    static const AddrRangeFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (AddrRangeFn) nullptr;
        return (AddrRangeFn)p;
    }();
    return fn;
}

cudaError_t issue(const std::vector<Copy>& v, cudaMemcpyKind kind, bool merge, cudaStream_t s) {
    const bool dev_dst = kind == cudaMemcpyHostToDevice;
    const AddrRangeFn range = merge ? addr_range() : nullptr;
    size_t i = 0;
    while (i < v.size()) {
        Copy c = v[i++];
        if (range) {
            CUdeviceptr base = 0;
            size_t size = 0;
            const char* d0 = dev_dst ? c.dst : c.src;
            if (range(&base, &size, (CUdeviceptr)d0) == CUDA_SUCCESS) {
                const char* dend = (const char*)base + size;
                while (i < v.size() && v[i].dst == c.dst + c.bytes && v[i].src == c.src + c.bytes &&
                       (dev_dst ? v[i].dst : v[i].src) + v[i].bytes <= dend)
                    c.bytes += v[i++].bytes;
            }
        }
        const cudaError_t e = cudaMemcpyAsync(c.dst, c.src, c.bytes, kind, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int launch_host(gpufhe_plan* plan, const uint64_t* const* h_in, uint64_t* const* h_out, const uint64_t* in_buf,
                uint64_t* out_buf, cudaStream_t s) {
    const pl::Plan& p = *plan->p;
    const size_t n = (size_t)1 << p.logn;
    const bool batch = in_buf != nullptr;
    std::vector<Copy> in, out;
    const char* hin = (const char*)in_buf;
    char* hout = (char*)out_buf;
    for (size_t i = 0; i < p.ops.size(); ++i) {
        const pl::Op& op = p.ops[i];
        for (int k = 0; k < pl::input_count(op.mode); ++k) {
            const size_t b = op.L * n * 8;
            const char* src = batch ? hin : (const char*)h_in[4 * i + k];
            if (batch) hin += b;
            if (src) in.push_back({(char*)op.in[k], src, b});
        }
        const int nout = op.mode == pl::RESCALE ? 1 : 2;
        for (int k = 0; k < nout; ++k) {
            const size_t b = pl::output_towers(op) * n * 8;
            char* dst = batch ? hout : (char*)h_out[2 * i + k];
            if (batch) hout += b;
            if (dst) out.push_back({dst, (const char*)op.out[k], b});
        }
    }
    cudaError_t e = issue(in, cudaMemcpyHostToDevice, batch, s);
    if (e == cudaSuccess) {
        pl::tune(*plan->p, s);
        e = pl::launch(p, s);
    }
    if (e == cudaSuccess) e = issue(out, cudaMemcpyDeviceToHost, batch, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}
}  // namespace

extern "C" {

int gpufhe_plan_launch_host_async(gpufhe_plan* plan, const uint64_t* const* h_in, uint64_t* const* h_out,
                                  cudaStream_t s) {
    if (!plan || !h_in || !h_out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    return launch_host(plan, h_in, h_out, nullptr, nullptr, s);
}

int gpufhe_plan_launch_host_batch_async(gpufhe_plan* plan, const uint64_t* h_in, uint64_t* h_out, cudaStream_t s) {
    if (!plan || !h_in || !h_out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    return launch_host(plan, nullptr, nullptr, h_in, h_out, s);
}

int gpufhe_plan_launch_host(gpufhe_plan* plan, const uint64_t* const* h_in, uint64_t* const* h_out,
                            cudaStream_t s) {
    const int rc = gpufhe_plan_launch_host_async(plan, h_in, h_out, s);
    if (rc) return rc;
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

void gpufhe_plan_destroy(gpufhe_plan* plan) { delete plan; }

int gpufhe_run_ops(gpufhe_ctx* h, uint32_t nops, const gpufhe_op* ops, cudaStream_t s) {
    gpufhe_plan* p = nullptr;
    int rc = gpufhe_plan_create(h, nops, ops, nullptr, 0, &p);
    if (rc) return rc;
    rc = gpufhe_plan_launch(p, s);
    cudaError_t e = cudaStreamSynchronize(s);
    gpufhe_plan_destroy(p);
    if (!rc && e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return rc;
}

}  // extern "C"
