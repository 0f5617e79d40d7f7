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
// Scratch: g_noalloc_scratch holds NOALLOC_MAX_WORDS uint64 words (8 MiB) of
// tower data plus a small table of transform jobs, on every GPU that loads
// the library, for as long as the process lives. A call at level L on ring
// dimension n uses L*n words: one tower for the dropped tower in coefficient
// form and L-1 towers for its switched, transformed copies. Levels with L*n
// above the maximum are rejected. Every word the call reads is written
// earlier in the same call, so nothing has to start at zero; the array keeps
// the last call's contents. All calls on a device share the one array, so
// calls that overlap on the GPU (different streams, or different host threads
// without ordering) race and corrupt each other.
//
// The host cannot use the array's name as a device address: in host code the
// symbol is a host-side stand-in. On its first call on a device (with that
// device current) the entry point asks the runtime for the array's device
// address with cudaGetSymbolAddress and keeps it per device; that first call
// should therefore come before any stream capture. The call runs on the
// context's device (made current for the call and restored on return).
//
// Work per call, whatever the level: one device copy and seven launches (the
// dropped tower's inverse transform, one switch kernel for every surviving
// tower, one kernel writing the job table, one batched forward transform and
// one fused multiply-add over every surviving tower).
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "hostmath.hpp"
#include "xform.cuh"

gfx::Context* gpufhe_impl(gpufhe_ctx* h);

namespace {

constexpr size_t NOALLOC_MAX_WORDS = (size_t)16 << 16;   // 16 towers at n = 2^16
constexpr size_t JOB_WORDS = (gfx::MAXQ * sizeof(xf::Job) + 255) / 256 * 32;   // job table, 256-byte granules
constexpr int MAX_DEVICES = 64;

// tower data [0, NOALLOC_MAX_WORDS), then the forward-transform job table
__device__ __align__(256) uint64_t g_noalloc_scratch[NOALLOC_MAX_WORDS + JOB_WORDS];

std::mutex g_mu;
uint64_t* g_scratch_addr[MAX_DEVICES] = {};

// Per surviving tower t (blockIdx.y): SwitchModulus constants (the reference's
// switch_modulus.cu:11-27 semantics), rescale constants and modulus.
struct TowerParams {
    u64 half[gfx::MAXQ];
    u64 diff[gfx::MAXQ];
    int larger[gfx::MAXQ];
    u64 s1[gfx::MAXQ], s1p[gfx::MAXQ], s2[gfx::MAXQ], s2p[gfx::MAXQ];
    ModC m[gfx::MAXQ];
};

// dst[t] = SwitchModulus(src, q_last -> q_t) for every surviving tower t
__global__ void k_switch_fan(u64* __restrict__ dst, const u64* __restrict__ src, const TowerParams tp, uint32_t n) {
    const uint32_t t = blockIdx.y;
    const ModC m = tp.m[t];
    const u64 half = tp.half[t], diff = tp.diff[t];
    const int larger = tp.larger[t];
    u64* d = dst + (size_t)t * n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const u64 x = src[i];
        const u64 dd = x > half ? diff : 0;
        if (larger) { d[i] = x + dd; continue; }
        const u64 xm = reduce64(x, m);
        d[i] = xm >= dd ? xm - dd : xm + m.q - dd;
    }
}

// job t: forward transform of switched tower t in place, integer path with
// the context's packed tables of modulus t
__global__ void k_fill_jobs(xf::Job* __restrict__ jobs, u64* sw, const Tw* twf, const TowerParams tp, uint32_t n,
                            uint32_t count) {
    const uint32_t t = threadIdx.x;
    if (t >= count) return;
    xf::Job j{};
    j.x = sw + (size_t)t * n;
    j.tw = twf + (size_t)t * n;
    j.q = tp.m[t].q;
    jobs[t] = j;
}

// c_t = (c_t * s1 + sw_t * s2) mod q_t for every surviving tower t (blockIdx.y),
// the reference's rescale.cu:10-21 fuse
__global__ void k_fuse_all(u64* __restrict__ c, const u64* __restrict__ sw, const TowerParams tp, uint32_t n) {
    const uint32_t t = blockIdx.y;
    const u64 q = tp.m[t].q, s1 = tp.s1[t], s1p = tp.s1p[t], s2 = tp.s2[t], s2p = tp.s2p[t];
    u64* a = c + (size_t)t * n;
    const u64* b = sw + (size_t)t * n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] = csub(shoup(a[i], s1, s1p, q) + shoup(b[i], s2, s2p, q), q);
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

// Makes the context's device current for the call; puts the caller's back.
struct DeviceScope {
    int prev = -1;
    bool ok = true;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; prev = -1; return; }
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceScope() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int fail(const std::string& step, cudaError_t e) {
    gfx::set_error("gpufhe_rescale_noalloc: " + step + ": " + cudaGetErrorString(e));
    return GPUFHE_ECUDA;
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
    DeviceScope scope(c->device());
    if (!scope.ok) {
        gfx::set_error("gpufhe_rescale_noalloc: cannot make the context's device current");
        return GPUFHE_ECUDA;
    }
    // an error left by an earlier launch is reported as such, not as this call's
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return fail("a CUDA error from an earlier call is pending", e);
    std::string err;
    uint64_t* scratch = scratch_for_current_device(err);
    if (!scratch) { gfx::set_error(err); return GPUFHE_ECUDA; }

    const auto& D = c->dev();
    const std::vector<u64>& q = c->Q();
    const uint32_t last = level - 1;
    const int logn = (int)c->logn();
    const gfx::Level& lv = c->level_host(level);
    const u64 ninv = hm::invmod(n, q[last]);

    TowerParams tp;
    std::memset(&tp, 0, sizeof(tp));
    for (uint32_t t = 0; t < last; ++t) {
        tp.half[t] = q[last] >> 1;
        tp.larger[t] = q[t] > q[last];
        tp.diff[t] = tp.larger[t] ? q[t] - q[last] : (q[last] - q[t]) % q[t];
        tp.m[t] = hm::modc(q[t]);
        tp.s1[t] = lv.s1[t];
        tp.s1p[t] = hm::precon(lv.s1[t], q[t]);
        tp.s2[t] = lv.s2[t];
        tp.s2p[t] = hm::precon(lv.s2[t], q[t]);
    }
    u64* drop = scratch;
    u64* sw = scratch + n;
    auto* jobs = reinterpret_cast<xf::Job*>(scratch + NOALLOC_MAX_WORDS);
    const dim3 grid((unsigned)std::min<uint32_t>((n + 255) / 256, 64), last);

    // 1. dropped tower -> scratch tower 0, inverse transform (times n^-1)
    e = cudaMemcpyAsync(drop, d_comp + (size_t)last * n, (size_t)n * 8, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return fail("copy of the dropped tower", e);
    const xf::Job ji{drop, D.twi + (size_t)last * n, nullptr, nullptr, q[last], ninv, hm::precon(ninv, q[last])};
    e = xf_launch_ntt(nullptr, &ji, 1, logn, true, s);
    if (e != cudaSuccess) return fail("inverse transform of the dropped tower", e);
    // 2. switched copies into scratch towers 1..last, and their job table
    k_switch_fan<<<grid, 256, 0, s>>>(sw, drop, tp, n);
    k_fill_jobs<<<1, gfx::MAXQ, 0, s>>>(jobs, sw, D.twf, tp, n, last);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail("modulus switch of the dropped tower", e);
    // 3. one forward transform over every switched tower, then one fused
    //    c * s1 + sw * s2 over every surviving tower
    e = xf_launch_ntt(jobs, nullptr, (int)last, logn, false, s);
    if (e != cudaSuccess) return fail("forward transforms of the switched towers", e);
    k_fuse_all<<<grid, 256, 0, s>>>(d_comp, sw, tp, n);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail("rescale multiply-add", e);
    return GPUFHE_OK;
}

}  // extern "C"
