// Rescale that allocates nothing: gpufhe_rescale_noalloc.
//
// Some callers cannot let a library call cudaMalloc / cudaFree: hosts that
// own the whole device-memory budget through their own pool allocator and
// forbid plugins from allocating (cudaMalloc can fail under a fixed budget,
// and cudaFree synchronizes the device), and latency-bound serving threads
// that must not block on an allocation between requests. For them this file
// provides a rescale whose scratch lives in a file-scope device array instead
// of a caller- or library-allocated workspace.
//
// Scratch: g_noalloc_scratch holds NOALLOC_MAX_WORDS uint64 words (8 MiB) on
// every GPU that loads the library, for as long as the process lives. A call
// at level L on ring dimension n uses L*n words: one tower for the dropped
// tower in coefficient form and L-1 towers for its switched, transformed
// copies. Levels with L*n above the maximum are rejected. Every word the
// call reads is written earlier in the same call, so nothing has to start at
// zero; the array keeps the last call's contents. All calls on a device share
// the one array, so calls that overlap on the GPU (different streams, or
// different host threads without ordering) race and corrupt each other.
//
// The host cannot use the array's name as a device address: in host code the
// symbol is a host-side stand-in. On its first call on a device (with that
// device current) the entry point asks the runtime for the array's device
// address with cudaGetSymbolAddress and keeps it per device; that first call
// should therefore come before any stream capture.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "hostmath.hpp"
#include "rescale.h"
#include "xform.cuh"

gfx::Context* gpufhe_impl(gpufhe_ctx* h);

namespace {

constexpr size_t NOALLOC_MAX_WORDS = (size_t)16 << 16;   // 16 towers at n = 2^16
constexpr int MAX_DEVICES = 64;

__device__ __align__(256) uint64_t g_noalloc_scratch[NOALLOC_MAX_WORDS];

std::mutex g_mu;
uint64_t* g_scratch_addr[MAX_DEVICES] = {};

// dst[t] = SwitchModulus(src, q_last -> q_t) for every surviving tower t
// (blockIdx.y), the reference's switch_modulus.cu:11-27 semantics.
struct SwitchParams {
    u64 half[gfx::MAXQ];
    u64 diff[gfx::MAXQ];
    int larger[gfx::MAXQ];
    ModC m[gfx::MAXQ];
};

__global__ void k_switch_fan(u64* __restrict__ dst, const u64* __restrict__ src, const SwitchParams sp, uint32_t n) {
    const uint32_t t = blockIdx.y;
    const ModC m = sp.m[t];
    const u64 half = sp.half[t], diff = sp.diff[t];
    const int larger = sp.larger[t];
    u64* d = dst + (size_t)t * n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const u64 x = src[i];
        const u64 dd = x > half ? diff : 0;
        if (larger) { d[i] = x + dd; continue; }
        const u64 xm = reduce64(x, m);
        d[i] = xm >= dd ? xm - dd : xm + m.q - dd;
    }
}

uint64_t* scratch_for_current_device(std::string& err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        err = "gpufhe_rescale_noalloc: no usable current device";
        return nullptr;
    }
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            err = std::string("gpufhe_rescale_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_scratch_addr[dev] = static_cast<uint64_t*>(p);
    }
    return g_scratch_addr[dev];
}

}  // namespace

extern "C" {

uint64_t gpufhe_rescale_noalloc_max_words(void) { return NOALLOC_MAX_WORDS; }

int gpufhe_rescale_noalloc(gpufhe_ctx* h, uint32_t level, uint64_t* d_comp, cudaStream_t s) {
    gfx::Context* c = gpufhe_impl(h);
    if (!c || !d_comp) { gfx::set_error("gpufhe_rescale_noalloc: null context or buffer"); return GPUFHE_EINVAL; }
    const uint32_t n = c->n();
    if (level < 2 || level > c->fullQ()) {
        gfx::set_error("gpufhe_rescale_noalloc: level must be in [2, fullQ]");
        return GPUFHE_EINVAL;
    }
    if ((size_t)level * n > NOALLOC_MAX_WORDS) {
        gfx::set_error("gpufhe_rescale_noalloc: level * n = " + std::to_string((size_t)level * n) +
                       " words exceeds the static scratch of " + std::to_string(NOALLOC_MAX_WORDS) + " words");
        return GPUFHE_ENOMEM;
    }
    std::string err;
    uint64_t* scratch = scratch_for_current_device(err);
    if (!scratch) { gfx::set_error(err); return GPUFHE_ECUDA; }

    const auto& D = c->dev();
    const std::vector<u64>& q = c->Q();
    const uint32_t last = level - 1;
    const int logn = (int)c->logn();
    const gfx::Level& lv = c->level_host(level);
    const u64 ninv[2] = {hm::invmod(n, q[last]), hm::precon(hm::invmod(n, q[last]), q[last])};

    // 1. dropped tower -> scratch tower 0, inverse NTT (times n^-1)
    u64* drop = scratch;
    cudaError_t e = cudaMemcpyAsync(drop, d_comp + (size_t)last * n, (size_t)n * 8, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    xf::Job ji{drop, D.twi + (size_t)last * n, nullptr, nullptr, q[last], ninv[0], ninv[1]};
    e = xf_launch_ntt(nullptr, &ji, 1, logn, true, s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }

    // 2. switched copies into scratch towers 1..last
    SwitchParams sp;
    std::memset(&sp, 0, sizeof(sp));
    for (uint32_t t = 0; t < last; ++t) {
        sp.half[t] = q[last] >> 1;
        sp.larger[t] = q[t] > q[last];
        sp.diff[t] = sp.larger[t] ? q[t] - q[last] : (q[last] - q[t]) % q[t];
        sp.m[t] = hm::modc(q[t]);
    }
    u64* sw = scratch + n;
    dim3 g((unsigned)std::min<uint32_t>((n + 255) / 256, 64), last);
    k_switch_fan<<<g, 256, 0, s>>>(sw, drop, sp, n);

    // 3. forward NTT of each switched tower, then a*s1 + b*s2 into the survivor
    for (uint32_t t = 0; t < last; ++t) {
        xf::Job jf{sw + (size_t)t * n, D.twf + (size_t)t * n, nullptr, nullptr, q[t], 0, 0};
        e = xf_launch_ntt(nullptr, &jf, 1, logn, false, s);
        if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
        LaunchRescaleFuse(d_comp + (size_t)t * n, sw + (size_t)t * n, lv.s1[t], lv.s2[t], q[t], n, s);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

}  // extern "C"
