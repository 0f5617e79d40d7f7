// The reference's C++ API (namespace gpufhe) on this library's kernels:
// DeviceCiphertext, DeviceTables / mul_resident / rescale_resident,
// KeySwitchConstants / compute_keyswitch_constants / keyswitch_core_resident,
// DeviceKSContext / DeviceKSWork / keyswitch_resident / rescale_resident_raw,
// rotation, the host keygen / evalkeygen / encrypt / decrypt harness, and the
// headerless host-vector helpers (automorphism, plaintext embedding,
// pointwise ciphertext ops).
// Same names, arguments, results and error behaviour (std::runtime_error on
// CUDA failures and unknown moduli) as the reference headers they replace.
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "ckks_ops.h"
#include "context.hpp"
#include "device_ciphertext.h"
#include "host_ops.h"
#include "hostmath.hpp"
#include "keygen.h"
#include "keyswitch.h"
#include "keyswitch_resident.h"
#include "params.h"
#include "pipeline.hpp"
#include "rescale.h"
#include "rns_arith.h"
#include "xform.cuh"

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("gpufhe: ") + what + ": " + cudaGetErrorString(e));
}

template <class T>
T* dup_to_device(const std::vector<T>& h) {
    T* d = nullptr;
    ck(cudaMalloc(&d, std::max<size_t>(h.size(), 1) * sizeof(T)), "cudaMalloc");
    ck(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
    return d;
}

constexpr int MAXT = gfx::MAXQ;
struct TowerMods { ModC m[MAXT]; };

__global__ void k_mul_towers(u64* __restrict__ a0, u64* __restrict__ a1, const u64* __restrict__ b0,
                             const u64* __restrict__ b1, TowerMods tm, uint32_t n) {
    const uint32_t t = blockIdx.y;
    const ModC m = tm.m[t];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const size_t x = (size_t)t * n + k;
        a0[x] = mulmod(a0[x], b0[x], m);
        a1[x] = mulmod(a1[x], b1[x], m);
    }
}

// dst = SwitchModulus(src, q_old -> q_new) (switch_modulus.cu:11-42 semantics)
__global__ void k_switch_copy(u64* __restrict__ dst, const u64* __restrict__ src, u64 half, u64 diff, int larger,
                              ModC mnew, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const u64 x = src[i];
        const u64 d = x > half ? diff : 0;
        if (larger) { dst[i] = x + d; continue; }
        const u64 xm = reduce64(x, mnew);
        dst[i] = xm >= d ? xm - d : xm + mnew.q - d;
    }
}

// out[j] = in[sigma slot] for eval-form towers (blockIdx.y = tower)
__global__ void k_galois_gather(u64* __restrict__ out, const u64* __restrict__ in, uint32_t logn, u64 k) {
    const uint32_t n = 1u << logn;
    out += (size_t)blockIdx.y << logn;
    in += (size_t)blockIdx.y << logn;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t e = 2 * (__brev(j) >> (32 - logn)) + 1;
        const uint32_t t = (uint32_t)(((u64)e * k) & (2ull * n - 1));
        out[j] = in[__brev((t - 1) >> 1) >> (32 - logn)];
    }
}

// c = c (+) d per tower (blockIdx.y = tower) for both components: the
// reference's add, s = a + b then s - q when s >= q (ptops.cpp:11, 13-18), or
// its exact product (a * b) mod q (ptops.cpp:10, 20-26); operands are reduced
// first so the product is exact for any 64-bit words.
__global__ void k_pointwise(u64* __restrict__ c0, u64* __restrict__ c1, const u64* __restrict__ d0,
                            const u64* __restrict__ d1, const ModC* __restrict__ mods, uint32_t n, int mul) {
    const ModC m = mods[blockIdx.y];
    const size_t base = (size_t)blockIdx.y * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const size_t x = base + k;
        if (mul) {
            c0[x] = mulmod(reduce64(c0[x], m), reduce64(d0[x], m), m);
            c1[x] = mulmod(reduce64(c1[x], m), reduce64(d1[x], m), m);
        } else {
            const u64 s0 = c0[x] + d0[x], s1 = c1[x] + d1[x];
            c0[x] = s0 >= m.q ? s0 - m.q : s0;
            c1[x] = s1 >= m.q ? s1 - m.q : s1;
        }
    }
}

// out[t][k] = ((m[k] % q_t) + q_t) % q_t in signed 64-bit arithmetic, the
// reference's embedding of an integer-coefficient plaintext (rotate.cpp:108-110).
__global__ void k_embed_towers(u64* __restrict__ out, const int64_t* __restrict__ m, const ModC* __restrict__ mods,
                               uint32_t n) {
    const long long q = (long long)mods[blockIdx.y].q;
    u64* o = out + (size_t)blockIdx.y * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const long long v = (long long)m[k];
        o[k] = (u64)((v % q + q) % q);
    }
}

unsigned grid_for(uint32_t n) { return (unsigned)std::min<uint64_t>((n + 255) / 256, 4096); }

// Switch-modulus values of one component's dropped tower into a survivor.
void switch_params(u64 q_old, u64 q_new, u64& half, u64& diff, int& larger) {
    half = q_old >> 1;
    larger = q_new > q_old;
    diff = larger ? q_new - q_old : (q_old - q_new) % q_new;
}

// Drops the last of `towers` towers of one eval-form component, tower by
// tower through n-word scratch buffers (the reference's rescale contract).
// fwd(t)/inv(t) give the transform job for modulus t.
template <class FJ, class IJ>
void rescale_component(u64* base, uint32_t towers, uint32_t n, const std::vector<u64>& q,
                       const std::vector<u64>& s1, const std::vector<u64>& s2, u64* scratch, u64* drop,
                       cudaStream_t s, FJ fwd, IJ inv) {
    if (towers < 2) return;
    const uint32_t last = towers - 1;
    const int logn = hm::ilog2(n);
    ck(cudaMemcpyAsync(drop, base + (size_t)last * n, (size_t)n * 8, cudaMemcpyDeviceToDevice, s), "copy");
    xf::Job ji = inv(last);
    ji.x = drop;
    ck(xf_launch_ntt(nullptr, &ji, 1, logn, true, s), "intt");
    for (uint32_t t = 0; t < last; ++t) {
        u64 half, diff;
        int larger;
        switch_params(q[last], q[t], half, diff, larger);
        k_switch_copy<<<grid_for(n), 256, 0, s>>>(scratch, drop, half, diff, larger, hm::modc(q[t]), n);
        xf::Job jf = fwd(t);
        jf.x = scratch;
        ck(xf_launch_ntt(nullptr, &jf, 1, logn, false, s), "ntt");
        LaunchRescaleFuse(base + (size_t)t * n, scratch, s1[t], s2[t], q[t], n, s);
    }
}

// Process-wide cache of packed twiddle tables for host-orchestrated helpers.
struct TabEntry { Tw* f; Tw* i; u64 ninv, ninvp; };
std::mutex g_tab_mu;
std::map<std::tuple<int, uint32_t, u64, u64>, TabEntry> g_tabs;

TabEntry tables_for(uint32_t n, u64 q, u64 root) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(g_tab_mu);
    auto key = std::make_tuple(dev, n, q, root);
    auto it = g_tabs.find(key);
    if (it != g_tabs.end()) return it->second;
    std::vector<Tw> f, iv;
    hm::twiddles(n, q, root, f, iv);
    TabEntry e{dup_to_device(f), dup_to_device(iv), hm::invmod(n, q), 0};
    e.ninvp = hm::precon(e.ninv, q);
    g_tabs.emplace(key, e);
    return e;
}

// Per-device staging for the host-vector helpers, grown on demand and kept
// for the process: the reference calls them once per diagonal of a linear
// transform, where a cudaMalloc / cudaFree pair per call would dominate.
// A helper holds the device's lock from upload to download.
struct Staging {
    std::mutex mu;
    char* p = nullptr;
    size_t cap = 0;
};
std::mutex g_stage_map_mu;
std::map<int, std::unique_ptr<Staging>> g_stage;

struct StageLease {
    std::unique_lock<std::mutex> lk;
    char* base;
    size_t off = 0;
    // Next 256-byte aligned region of `bytes`.
    template <class T>
    T* take(size_t count) {
        T* r = reinterpret_cast<T*>(base + off);
        off += (count * sizeof(T) + 255) & ~(size_t)255;
        return r;
    }
};

// Total bytes of regions of the given sizes as StageLease::take lays them out.
size_t stage_bytes(std::initializer_list<size_t> sizes) {
    size_t t = 0;
    for (size_t b : sizes) t += (b + 255) & ~(size_t)255;
    return t;
}

StageLease stage(size_t bytes) {
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    Staging* st;
    {
        std::lock_guard<std::mutex> g(g_stage_map_mu);
        auto& slot = g_stage[dev];
        if (!slot) slot.reset(new Staging);
        st = slot.get();
    }
    std::unique_lock<std::mutex> lk(st->mu);
    if (bytes > st->cap) {
        if (st->p) ck(cudaFree(st->p), "cudaFree");
        st->p = nullptr;
        st->cap = 0;
        ck(cudaMalloc(&st->p, bytes), "cudaMalloc");
        st->cap = bytes;
    }
    return StageLease{std::move(lk), st->p};
}

// Fills `jobs` with the transform of every tower of d ([towers][n], tower t
// mod[t]) and launches it in one batched launch per pass on stream 0.
void launch_xform(u64* d, xf::Job* d_jobs, uint32_t towers, uint32_t n, const std::vector<u64>& mod,
                  const std::vector<u64>& root, bool inverse) {
    std::vector<xf::Job> jobs(towers);
    for (uint32_t t = 0; t < towers; ++t) {
        TabEntry e = tables_for(n, mod[t], root[t]);
        jobs[t] = xf::Job{d + (size_t)t * n, inverse ? e.i : e.f, nullptr, nullptr, mod[t], e.ninv, e.ninvp};
    }
    ck(cudaMemcpy(d_jobs, jobs.data(), towers * sizeof(xf::Job), cudaMemcpyHostToDevice), "upload");
    ck(xf_launch_ntt(d_jobs, nullptr, (int)towers, hm::ilog2(n), inverse, 0), "transform");
}

std::vector<ModC> modcs(const std::vector<u64>& mod, uint32_t towers) {
    std::vector<ModC> m(towers);
    for (uint32_t t = 0; t < towers; ++t) m[t] = hm::modc(mod[t]);
    return m;
}

void need(bool ok, const char* what) {
    if (!ok) throw std::invalid_argument(std::string("gpufhe: ") + what);
}

// Transforms every tower of a host [towers][n] array (tower t mod[t]).
void host_xform(std::vector<u64>& h, uint32_t towers, uint32_t n, const std::vector<u64>& mod,
                const std::vector<u64>& root, bool inverse) {
    const size_t T = (size_t)towers * n;
    StageLease L = stage(stage_bytes({towers * sizeof(xf::Job), T * 8}));
    xf::Job* dj = L.take<xf::Job>(towers);
    u64* d = L.take<u64>(T);
    ck(cudaMemcpy(d, h.data(), T * 8, cudaMemcpyHostToDevice), "upload");
    launch_xform(d, dj, towers, n, mod, root, inverse);
    ck(cudaMemcpy(h.data(), d, T * 8, cudaMemcpyDeviceToHost), "download");
}

inline u64 emb(long v, u64 q) { return (u64)((v % (long)q + (long)q) % (long)q); }
uint32_t g_hw = 0;

struct WorkImpl {
    std::unique_ptr<pl::Plan> plan;
    gfx::Context* ctx = nullptr;
};

}  // namespace

namespace gpufhe {

// The reference's A/B switch between its batched and per-digit inner-product
// launches. Here every keyswitch is one fused plan whatever the value; both of
// the reference's settings give the same bits, so the flag is accepted and
// read by nothing.
bool g_ks_batched = true;

// ---------------------------------------------------------------- DeviceCiphertext
// Both components live in one device allocation: c0 at the start, c1 right
// after the n x towers words of c0 (one cudaMalloc, one cudaFree). The
// object owns that allocation through d_c0_; d_c1_ points into it.
namespace {
void release_components(uint64_t*& c0, uint64_t*& c1) {
    if (c0) cudaFree(c0);
    c0 = c1 = nullptr;
}
void check_words(const char* what, size_t have, size_t want) {
    if (have != want)
        throw std::runtime_error(std::string("gpufhe::DeviceCiphertext: ") + what + " has " + std::to_string(have) +
                                 " words, the ciphertext holds " + std::to_string(want) + " per component");
}
}  // namespace

DeviceCiphertext::DeviceCiphertext(Scheme scheme, uint32_t n, uint32_t num_towers)
    : scheme_(scheme), n_(n), towers_(num_towers) {
    const size_t words = (size_t)n_ * towers_;
    ck(cudaMalloc(&d_c0_, std::max<size_t>(2 * words, 1) * sizeof(uint64_t)), "DeviceCiphertext: device allocation");
    d_c1_ = d_c0_ + words;
}
DeviceCiphertext::~DeviceCiphertext() { release_components(d_c0_, d_c1_); }
DeviceCiphertext::DeviceCiphertext(DeviceCiphertext&& o) noexcept
    : scheme_(o.scheme_), format_(o.format_), n_(o.n_), towers_(o.towers_), d_c0_(o.d_c0_), d_c1_(o.d_c1_) {
    o.d_c0_ = o.d_c1_ = nullptr;
}
DeviceCiphertext& DeviceCiphertext::operator=(DeviceCiphertext&& o) noexcept {
    if (this == &o) return *this;
    release_components(d_c0_, d_c1_);
    std::swap(scheme_, o.scheme_);
    std::swap(format_, o.format_);
    std::swap(n_, o.n_);
    std::swap(towers_, o.towers_);
    std::swap(d_c0_, o.d_c0_);
    std::swap(d_c1_, o.d_c1_);
    return *this;
}
void DeviceCiphertext::upload(const std::vector<uint64_t>& c0, const std::vector<uint64_t>& c1) {
    const size_t words = (size_t)n_ * towers_;
    check_words("upload: c0", c0.size(), words);
    check_words("upload: c1", c1.size(), words);
    ck(cudaMemcpy(d_c0_, c0.data(), words * sizeof(uint64_t), cudaMemcpyHostToDevice), "DeviceCiphertext: c0 to device");
    ck(cudaMemcpy(d_c1_, c1.data(), words * sizeof(uint64_t), cudaMemcpyHostToDevice), "DeviceCiphertext: c1 to device");
}
void DeviceCiphertext::to_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1) const {
    const size_t words = (size_t)n_ * towers_;
    c0.assign(words, 0);
    c1.assign(words, 0);
    ck(cudaMemcpy(c0.data(), d_c0_, words * sizeof(uint64_t), cudaMemcpyDeviceToHost), "DeviceCiphertext: c0 to host");
    ck(cudaMemcpy(c1.data(), d_c1_, words * sizeof(uint64_t), cudaMemcpyDeviceToHost), "DeviceCiphertext: c1 to host");
}

// ---------------------------------------------------------------- DeviceTables
void build_device_tables(DeviceTables& T, uint32_t n, const std::vector<uint64_t>& moduli) {
    T.n = n;
    T.q = moduli;
    const uint32_t towers = (uint32_t)moduli.size();
    T.d_froots.assign(towers, nullptr); T.d_fprecon.assign(towers, nullptr);
    T.d_iroots.assign(towers, nullptr); T.d_iprecon.assign(towers, nullptr);
    T.ninv.resize(towers); T.ninv_precon.resize(towers);
    for (uint32_t t = 0; t < towers; ++t) {
        const u64 q = moduli[t];
        const u64 root = native_root(n, q);   // smallest-generator root, as ckks_ops.cpp:25-38
        std::vector<Tw> f, iv;
        hm::twiddles(n, q, root, f, iv);
        std::vector<u64> fr(n), fp(n), ir(n), ip(n);
        for (uint32_t i = 0; i < n; ++i) { fr[i] = f[i].w; fp[i] = f[i].wp; ir[i] = iv[i].w; ip[i] = iv[i].wp; }
        T.d_froots[t] = dup_to_device(fr); T.d_fprecon[t] = dup_to_device(fp);
        T.d_iroots[t] = dup_to_device(ir); T.d_iprecon[t] = dup_to_device(ip);
        T.ninv[t] = hm::invmod(n, q);
        T.ninv_precon[t] = hm::precon(T.ninv[t], q);
    }
}

DeviceTables::~DeviceTables() {
    for (auto* v : {&d_froots, &d_fprecon, &d_iroots, &d_iprecon})
        for (auto p : *v) if (p) cudaFree(p);
}

void mul_resident(DeviceCiphertext& a, const DeviceCiphertext& b, const DeviceTables& T, cudaStream_t stream) {
    const uint32_t n = a.n(), towers = a.num_towers();
    if (!towers) return;
    for (uint32_t t0 = 0; t0 < towers; t0 += MAXT) {
        const uint32_t cnt = std::min<uint32_t>(MAXT, towers - t0);
        TowerMods tm;
        for (uint32_t t = 0; t < cnt; ++t) tm.m[t] = hm::modc(T.q[t0 + t]);
        dim3 g(std::max(1u, std::min(grid_for(n), 64u)), cnt);
        DeviceCiphertext& bb = const_cast<DeviceCiphertext&>(b);
        k_mul_towers<<<g, 256, 0, stream>>>(a.c0() + (size_t)t0 * n, a.c1() + (size_t)t0 * n,
                                            bb.c0() + (size_t)t0 * n, bb.c1() + (size_t)t0 * n, tm, n);
    }
}

void rescale_resident(DeviceCiphertext& ct, const DeviceTables& T, const std::vector<uint64_t>& s1,
                      const std::vector<uint64_t>& s2, cudaStream_t stream, uint64_t* scratch, uint64_t* dropCoeff) {
    const uint32_t n = ct.n(), towers = ct.num_towers();
    if (towers < 2) return;
    auto fwd = [&](uint32_t t) { return xf::Job{nullptr, nullptr, T.d_froots[t], T.d_fprecon[t], T.q[t], 0, 0}; };
    auto inv = [&](uint32_t t) {
        return xf::Job{nullptr, nullptr, T.d_iroots[t], T.d_iprecon[t], T.q[t], T.ninv[t], T.ninv_precon[t]};
    };
    rescale_component(ct.c0(), towers, n, T.q, s1, s2, scratch, dropCoeff, stream, fwd, inv);
    rescale_component(ct.c1(), towers, n, T.q, s1, s2, scratch, dropCoeff, stream, fwd, inv);
    ct.drop_tower();
}

// ---------------------------------------------------------------- constants
void compute_keyswitch_constants(KeySwitchConstants& K, const std::vector<uint64_t>& moduliQ,
                                 const std::vector<uint64_t>& moduliP, uint32_t numPart) {
    const uint32_t sizeQ = (uint32_t)moduliQ.size(), sizeP = (uint32_t)moduliP.size();
    if (!numPart) throw std::invalid_argument("numPart must be >= 1");
    const uint32_t alpha = (uint32_t)std::ceil((double)sizeQ / numPart);
    K.sizeQl = sizeQ; K.sizeP = sizeP; K.numPart = numPart; K.alpha = alpha; K.fullQ = sizeQ;
    K.qMod = moduliQ; K.pMod = moduliP;
    K.pInvModq.resize(sizeQ);
    for (uint32_t i = 0; i < sizeQ; ++i)
        K.pInvModq[i] = hm::invmod(hm::prod_mod(moduliP.data(), sizeP, moduliQ[i]), moduliQ[i]);
    K.pHatInv.resize(sizeP); K.pHatInvPrec.resize(sizeP); K.pHatModq.resize((size_t)sizeP * sizeQ);
    for (uint32_t j = 0; j < sizeP; ++j) {
        const u64 pj = moduliP[j];
        K.pHatInv[j] = hm::invmod(hm::prod_mod(moduliP.data(), sizeP, pj, (int)j), pj);
        K.pHatInvPrec[j] = hm::precon(K.pHatInv[j], pj);
        for (uint32_t i = 0; i < sizeQ; ++i)
            K.pHatModq[(size_t)j * sizeQ + i] = hm::prod_mod(moduliP.data(), sizeP, moduliQ[i], (int)j);
    }
    K.mdBMuLo.resize(sizeQ); K.mdBMuHi.resize(sizeQ);
    for (uint32_t i = 0; i < sizeQ; ++i) {
        const ModC m = hm::modc(moduliQ[i]);
        K.mdBMuLo[i] = m.mu_lo; K.mdBMuHi[i] = m.mu_hi;
    }
    for (auto* v : {&K.partQHatInv, &K.partQHatInvPrec, &K.partSrcMod, &K.partQHatModp, &K.partComplMod,
                    &K.partBMuLo, &K.partBMuHi}) v->assign(numPart, {});
    K.sizePart.resize(numPart); K.sizeCompl.resize(numPart); K.startIdx.resize(numPart);
    for (uint32_t part = 0; part < numPart; ++part) {
        const uint32_t st = alpha * part;
        const uint32_t sp = (sizeQ > st + alpha) ? alpha : (sizeQ > st ? sizeQ - st : 0);
        K.startIdx[part] = st; K.sizePart[part] = sp;
        std::vector<u64> src(moduliQ.begin() + st, moduliQ.begin() + st + sp);
        K.partSrcMod[part] = src;
        K.partQHatInv[part].resize(sp); K.partQHatInvPrec[part].resize(sp);
        for (uint32_t i = 0; i < sp; ++i) {
            K.partQHatInv[part][i] = hm::invmod(hm::prod_mod(src.data(), sp, src[i], (int)i), src[i]);
            K.partQHatInvPrec[part][i] = hm::precon(K.partQHatInv[part][i], src[i]);
        }
        std::vector<u64> compl_;
        for (uint32_t i = 0; i < sizeQ; ++i) if (i < st || i >= st + sp) compl_.push_back(moduliQ[i]);
        for (uint32_t j = 0; j < sizeP; ++j) compl_.push_back(moduliP[j]);
        const uint32_t sc = (uint32_t)compl_.size();
        K.sizeCompl[part] = sc; K.partComplMod[part] = compl_;
        K.partQHatModp[part].resize((size_t)sp * sc);
        for (uint32_t i = 0; i < sp; ++i)
            for (uint32_t j = 0; j < sc; ++j)
                K.partQHatModp[part][(size_t)i * sc + j] = hm::prod_mod(src.data(), sp, compl_[j], (int)i);
        K.partBMuLo[part].resize(sc); K.partBMuHi[part].resize(sc);
        for (uint32_t j = 0; j < sc; ++j) {
            const ModC m = hm::modc(compl_[j]);
            K.partBMuLo[part][j] = m.mu_lo; K.partBMuHi[part][j] = m.mu_hi;
        }
    }
}

// ---------------------------------------------------------------- resident keyswitch
namespace {
// Root tables in the reference's split layout (psi^bitrev(i), its Shoup
// precomputation, and the same from psi^-1), shared by every context of a
// device for the process: DeviceKSContext publishes them and never frees them.
struct SplitTab { u64 *fr, *fp, *ir, *ip; u64 ninv, ninvp; };
std::mutex g_split_mu;
std::map<std::tuple<int, uint32_t, u64, u64>, SplitTab> g_split;

u64* upload_words(const std::vector<u64>& h) {
    u64* d = nullptr;
    ck(cudaMalloc(&d, std::max<size_t>(h.size(), 1) * 8), "ks_context_create: table");
    if (!h.empty()) ck(cudaMemcpy(d, h.data(), h.size() * 8, cudaMemcpyHostToDevice), "ks_context_create: upload");
    return d;
}

SplitTab split_tables_for(uint32_t n, u64 q, u64 root) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(g_split_mu);
    const auto key = std::make_tuple(dev, n, q, root);
    auto it = g_split.find(key);
    if (it != g_split.end()) return it->second;
    std::vector<Tw> f, iv;
    hm::twiddles(n, q, root, f, iv);
    std::vector<u64> a(n), b(n), c(n), d(n);
    for (uint32_t i = 0; i < n; ++i) { a[i] = f[i].w; b[i] = f[i].wp; c[i] = iv[i].w; d[i] = iv[i].wp; }
    const u64 ni = hm::invmod(n, q);
    const SplitTab t{upload_words(a), upload_words(b), upload_words(c), upload_words(d), ni, hm::precon(ni, q)};
    g_split.emplace(key, t);
    return t;
}

// The reference's public tables of a context (its ks_context_create,
// src/keyswitch_resident.cpp:32-107): the same values under the same names.
void publish_tables(DeviceKSContext& C, const KeySwitchConstants& K) {
    auto root_of = [&](u64 q) {
        for (size_t r = 0; r < K.rootModList.size(); ++r) if (K.rootModList[r] == q) return K.rootValList[r];
        throw std::runtime_error("no root table for modulus");
    };
    for (u64 q : C.modList) {
        const SplitTab t = split_tables_for(C.n, q, root_of(q));
        C.d_fr.push_back(t.fr); C.d_fp.push_back(t.fp); C.d_ir.push_back(t.ir); C.d_ip.push_back(t.ip);
        C.ninv.push_back(t.ninv); C.ninv_p.push_back(t.ninvp);
    }
    for (uint32_t p = 0; p < K.numPart; ++p) {
        C.complModHost.push_back(K.partComplMod[p]);
        C.d_qhi.push_back(upload_words(K.partQHatInv[p]));
        C.d_qhip.push_back(upload_words(K.partQHatInvPrec[p]));
        C.d_srcMod.push_back(upload_words(K.partSrcMod[p]));
        C.d_qmp.push_back(upload_words(K.partQHatModp[p]));
        C.d_complMod.push_back(upload_words(K.partComplMod[p]));
        C.d_mlo.push_back(upload_words(K.partBMuLo[p]));
        C.d_mhi.push_back(upload_words(K.partBMuHi[p]));
        if (p < K.av.size() && p < K.bv.size()) {
            C.d_av.push_back(upload_words(K.av[p]));
            C.d_bv.push_back(upload_words(K.bv[p]));
        }
    }
    C.d_pHatInv = upload_words(K.pHatInv);
    C.d_pHatInvPrec = upload_words(K.pHatInvPrec);
    C.d_pMod = upload_words(K.pMod);
    C.d_pHatModq = upload_words(K.pHatModq);
    C.d_qMod = upload_words(K.qMod);
    C.d_mdMuLo = upload_words(K.mdBMuLo);
    C.d_mdMuHi = upload_words(K.mdBMuHi);
    // per QlP tower: modulus, and the eval-key row (P rows sit after all fullQ rows)
    std::vector<u64> mq(C.sizeQlP);
    std::vector<uint32_t> kr(C.sizeQlP);
    for (uint32_t i = 0; i < C.sizeQlP; ++i) {
        mq[i] = i < C.sizeQl ? K.qMod[i] : K.pMod[i - C.sizeQl];
        kr[i] = i < C.sizeQl ? i : i + (C.fullQ - C.sizeQl);
    }
    C.d_modsQlP = upload_words(mq);
    ck(cudaMalloc(&C.d_keyRow, std::max<size_t>(kr.size(), 1) * 4), "ks_context_create: key rows");
    ck(cudaMemcpy(C.d_keyRow, kr.data(), kr.size() * 4, cudaMemcpyHostToDevice), "ks_context_create: key rows");
}

void free_published(DeviceKSContext& C) {
    for (auto* v : {&C.d_qhi, &C.d_qhip, &C.d_srcMod, &C.d_qmp, &C.d_complMod, &C.d_mlo, &C.d_mhi, &C.d_av, &C.d_bv}) {
        for (u64* p : *v) cudaFree(p);
        v->clear();
    }
    for (u64** p : {&C.d_pHatInv, &C.d_pHatInvPrec, &C.d_pMod, &C.d_pHatModq, &C.d_qMod, &C.d_mdMuLo, &C.d_mdMuHi,
                    &C.d_modsQlP}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (C.d_keyRow) cudaFree(C.d_keyRow);
    C.d_keyRow = nullptr;
    C.d_fr.clear(); C.d_fp.clear(); C.d_ir.clear(); C.d_ip.clear();   // shared root tables stay
}
}  // namespace

DeviceKSContext ks_context_create(const KeySwitchConstants& K) {
    DeviceKSContext C;
    C.n = K.n; C.sizeQl = K.sizeQl; C.sizeP = K.sizeP; C.sizeQlP = K.sizeQl + K.sizeP;
    C.numPart = K.numPart; C.fullQ = K.fullQ ? K.fullQ : K.sizeQl;
    C.sizePart = K.sizePart; C.sizeCompl = K.sizeCompl; C.startIdx = K.startIdx;
    C.qModHost = K.qMod; C.pModHost = K.pMod; C.pInvModqHost = K.pInvModq;
    std::vector<u64> roots;
    auto root_of = [&](u64 q) {
        for (size_t r = 0; r < K.rootModList.size(); ++r) if (K.rootModList[r] == q) return K.rootValList[r];
        throw std::runtime_error("no root table for modulus");
    };
    for (u64 q : K.qMod) { roots.push_back(root_of(q)); C.modList.push_back(q); }
    for (u64 p : K.pMod) { roots.push_back(root_of(p)); C.modList.push_back(p); }
    // a digit wider than the level covers all of it: the same partition as alpha = sizeQl
    const uint32_t alpha = std::min(K.alpha ? K.alpha : (K.sizeQl + K.numPart - 1) / K.numPart, K.sizeQl);
    int dev = 0;
    cudaGetDevice(&dev);
    auto* ctx = new gfx::Context(K.n, K.qMod, K.pMod, alpha, roots, dev);
    C.impl = ctx;
    if (!K.av.empty()) {
        // repack the full-QP key rows for this level into [dnum][sizeQl+sizeP][n]
        const uint32_t dnum = ctx->dnum(), QlP = C.sizeQlP, n = K.n;
        if (K.av.size() < dnum || K.bv.size() < dnum) {
            delete ctx;
            throw std::runtime_error("eval key has fewer digits than the partition");
        }
        const uint32_t delta = C.fullQ - K.sizeQl;
        std::vector<u64> av((size_t)dnum * QlP * n), bv(av.size());
        for (uint32_t p = 0; p < dnum; ++p)
            for (uint32_t i = 0; i < QlP; ++i) {
                const uint32_t row = i >= K.sizeQl ? i + delta : i;
                std::memcpy(&av[((size_t)p * QlP + i) * n], &K.av[p][(size_t)row * n], (size_t)n * 8);
                std::memcpy(&bv[((size_t)p * QlP + i) * n], &K.bv[p][(size_t)row * n], (size_t)n * 8);
            }
        ctx->set_key(0, av.data(), bv.data());
    }
    try {
        publish_tables(C, K);
    } catch (...) {
        free_published(C);
        gfx::Context::retire(ctx);
        throw;
    }
    return C;
}

void ks_context_destroy(DeviceKSContext& C) {
    free_published(C);
    gfx::Context::retire(static_cast<gfx::Context*>(C.impl));
    C.impl = nullptr;
}

DeviceKSWork ks_work_create(const DeviceKSContext& C) {
    auto* ctx = static_cast<gfx::Context*>(C.impl);
    if (!ctx) throw std::runtime_error("ks_work_create: empty context");
    DeviceKSWork W;
    const uint32_t L = C.sizeQl;
    const size_t words = pl::op_workspace_words(*ctx, L);
    ck(cudaMalloc(&W.d_ws, words * 8), "ks_work_create: workspace");
    // the reference's scratch buffers, at its sizes (keyswitch_resident.cpp:109-120)
    const size_t n = C.n;
    uint32_t max_part = 0;
    for (uint32_t sp : C.sizePart) max_part = std::max(max_part, sp);
    ck(cudaMalloc(&W.d_part, std::max<size_t>(max_part, 1) * n * 8), "ks_work_create: scratch");
    ck(cudaMalloc(&W.d_compl, (size_t)C.sizeQlP * n * 8), "ks_work_create: scratch");
    ck(cudaMalloc(&W.d_res0, (size_t)C.sizeQlP * n * 8), "ks_work_create: scratch");
    ck(cudaMalloc(&W.d_res1, (size_t)C.sizeQlP * n * 8), "ks_work_create: scratch");
    ck(cudaMalloc(&W.d_pwork, std::max<size_t>(C.sizeP, 1) * n * 8), "ks_work_create: scratch");
    ck(cudaMalloc(&W.d_qsw, (size_t)C.sizeQl * n * 8), "ks_work_create: scratch");
    ck(cudaMalloc(reinterpret_cast<void**>(&W.d_digPtrs), std::max<size_t>(C.sizeQlP, 1) * sizeof(uint64_t*)),
       "ks_work_create: scratch");
    auto* wi = new WorkImpl();
    wi->ctx = ctx;
    if (ctx->key(0)) {
        pl::Op op;
        op.L = L;
        op.mode = pl::KS;
        alignas(16) static u64 dummy[2];
        op.in[0] = dummy;   // rebound on every call
        op.out[0] = op.out[1] = dummy;
        wi->plan = pl::build_plan(*ctx, {op}, W.d_ws, words);
    }
    W.impl = wi;
    return W;
}

void ks_work_destroy(DeviceKSWork& W) {
    delete static_cast<WorkImpl*>(W.impl);
    W.impl = nullptr;
    for (uint64_t** p : {&W.d_ws, &W.d_part, &W.d_compl, &W.d_res0, &W.d_res1, &W.d_pwork, &W.d_qsw}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (W.d_digPtrs) cudaFree(const_cast<uint64_t**>(W.d_digPtrs));
    W.d_digPtrs = nullptr;
}

void keyswitch_resident(const uint64_t* d_a, uint64_t* d_ba0, uint64_t* d_ba1, const DeviceKSContext& C,
                        DeviceKSWork& W, cudaStream_t s) {
    auto* wi = static_cast<WorkImpl*>(W.impl);
    if (!wi || !wi->plan) throw std::runtime_error("keyswitch_resident: context has no eval key");
    pl::Op op;
    op.L = C.sizeQl;
    op.mode = pl::KS;
    op.in[0] = d_a;
    op.out[0] = d_ba0;
    op.out[1] = d_ba1;
    pl::rebind(*wi->plan, 0, op, *wi->ctx, s);
    ck(pl::launch(*wi->plan, s), "keyswitch_resident");
}

void rescale_resident_raw(uint64_t* d_c, uint32_t towers, const DeviceKSContext& C, const std::vector<uint64_t>& s1,
                          const std::vector<uint64_t>& s2, uint64_t* d_scratch, uint64_t* d_drop, cudaStream_t s) {
    auto* ctx = static_cast<gfx::Context*>(C.impl);
    if (!ctx) throw std::runtime_error("rescale_resident_raw: empty context");
    if (towers < 2) return;
    if (towers > ctx->fullQ()) throw std::runtime_error("rescale_resident_raw: more towers than the context");
    const auto& D = ctx->dev();
    const uint32_t n = C.n;
    const std::vector<u64>& q = ctx->Q();
    // n^-1 from the host moduli: no device read, so the call stays capturable
    std::vector<u64> ninv(towers), ninvp(towers);
    for (uint32_t t = 0; t < towers; ++t) {
        ninv[t] = hm::invmod(n, q[t]);
        ninvp[t] = hm::precon(ninv[t], q[t]);
    }
    auto fwd = [&](uint32_t t) { return xf::Job{nullptr, D.twf + (size_t)t * n, nullptr, nullptr, q[t], 0, 0}; };
    auto inv = [&](uint32_t t) { return xf::Job{nullptr, D.twi + (size_t)t * n, nullptr, nullptr, q[t], ninv[t], ninvp[t]}; };
    rescale_component(d_c, towers, n, q, s1, s2, d_scratch, d_drop, s, fwd, inv);
}

KeySwitchResult keyswitch_core_resident(const std::vector<uint64_t>& aTowers, const KeySwitchConstants& K) {
    DeviceKSContext C = ks_context_create(K);
    DeviceKSWork W = ks_work_create(C);
    const size_t T = (size_t)K.sizeQl * K.n;
    u64* da = dup_to_device(aTowers);
    u64 *d0 = nullptr, *d1 = nullptr;
    ck(cudaMalloc(&d0, T * 8), "cudaMalloc");
    ck(cudaMalloc(&d1, T * 8), "cudaMalloc");
    keyswitch_resident(da, d0, d1, C, W, 0);
    ck(cudaDeviceSynchronize(), "keyswitch");
    KeySwitchResult R;
    R.ba0.resize(T);
    R.ba1.resize(T);
    ck(cudaMemcpy(R.ba0.data(), d0, T * 8, cudaMemcpyDeviceToHost), "download");
    ck(cudaMemcpy(R.ba1.data(), d1, T * 8, cudaMemcpyDeviceToHost), "download");
    cudaFree(da); cudaFree(d0); cudaFree(d1);
    ks_work_destroy(W);
    ks_context_destroy(C);
    return R;
}

// ---------------------------------------------------------------- rotation
void automorphism_eval_device(uint64_t* d_v, uint32_t towers, uint32_t n, uint32_t k, const std::vector<uint64_t>&,
                              const std::vector<uint64_t>&, uint64_t* d_scratch, cudaStream_t s) {
    const uint32_t logn = (uint32_t)hm::ilog2(n);
    for (uint32_t t = 0; t < towers; ++t) {
        uint64_t* col = d_v + (size_t)t * n;
        k_galois_gather<<<grid_for(n), 256, 0, s>>>(d_scratch, col, logn, k);
        ck(cudaMemcpyAsync(col, d_scratch, (size_t)n * 8, cudaMemcpyDeviceToDevice, s), "automorphism copy");
    }
}

void rotate_ct_device(uint64_t* d_c0, uint64_t* d_c1, uint32_t k, const DeviceKSContext& C, DeviceKSWork& W,
                      uint32_t towers, uint32_t n, const std::vector<uint64_t>&, const std::vector<uint64_t>&,
                      uint64_t*, uint64_t* d_b0, uint64_t* d_b1, cudaStream_t s) {
    auto* wi = static_cast<WorkImpl*>(W.impl);
    if (!wi || !wi->plan) throw std::runtime_error("rotate_ct_device: context has no rotation key");
    if (towers != C.sizeQl) throw std::runtime_error("rotate_ct_device: tower count differs from the context");
    pl::Op op;
    op.L = towers;
    op.mode = pl::ROT;
    op.galois = k;
    op.in[0] = d_c0;
    op.in[1] = d_c1;
    op.out[0] = d_b0;
    op.out[1] = d_b1;
    pl::rebind(*wi->plan, 0, op, *wi->ctx, s);
    ck(pl::launch(*wi->plan, s), "rotate_ct_device");
    const size_t bytes = (size_t)towers * n * 8;
    ck(cudaMemcpyAsync(d_c0, d_b0, bytes, cudaMemcpyDeviceToDevice, s), "rotate copy");
    ck(cudaMemcpyAsync(d_c1, d_b1, bytes, cudaMemcpyDeviceToDevice, s), "rotate copy");
}

void rotate_ct_resident(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, uint32_t k,
                        const KeySwitchConstants& Krot, uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod,
                        const std::vector<uint64_t>& root) {
    const size_t T = (size_t)towers * n;
    need(c0.size() >= T && c1.size() >= T, "rotate_ct_resident: ciphertext shorter than towers*n");
    c1.resize(T);
    DeviceKSContext C = ks_context_create(Krot);
    DeviceKSWork W = ks_work_create(C);
    u64 *d0 = dup_to_device(c0), *d1 = dup_to_device(c1), *b0 = nullptr, *b1 = nullptr;
    ck(cudaMalloc(&b0, T * 8), "cudaMalloc");
    ck(cudaMalloc(&b1, T * 8), "cudaMalloc");
    rotate_ct_device(d0, d1, k, C, W, towers, n, mod, root, nullptr, b0, b1, 0);
    ck(cudaDeviceSynchronize(), "rotate");
    ck(cudaMemcpy(c0.data(), d0, T * 8, cudaMemcpyDeviceToHost), "download");
    ck(cudaMemcpy(c1.data(), d1, T * 8, cudaMemcpyDeviceToHost), "download");
    cudaFree(d0); cudaFree(d1); cudaFree(b0); cudaFree(b1);
    ks_work_destroy(W);
    ks_context_destroy(C);
}

// ---------------------------------------------------------------- host-vector helpers
// Functions the reference defines without a header (rotate.cpp:87-112,
// 176-188, ptops.cpp:13-26) and its tests declare where they call them.
// Each stages its operands through the device's staging buffer, runs one
// batched launch per step over all towers, and copies the result back.

void automorphism_eval_host(std::vector<uint64_t>& v, uint32_t towers, uint32_t n, uint32_t k,
                            const std::vector<uint64_t>&, const std::vector<uint64_t>&) {
    const size_t T = (size_t)towers * n;
    need(hm::is_pow2(n) && n >= 2, "automorphism_eval_host: n must be a power of two");
    need(k & 1, "automorphism_eval_host: Galois element must be odd");
    need(v.size() >= T, "automorphism_eval_host: vector shorter than towers*n");
    v.resize(T);
    if (!T) return;
    StageLease L = stage(stage_bytes({T * 8, T * 8}));
    u64* din = L.take<u64>(T);
    u64* dout = L.take<u64>(T);
    ck(cudaMemcpy(din, v.data(), T * 8, cudaMemcpyHostToDevice), "upload");
    k_galois_gather<<<dim3(grid_for(n), towers), 256>>>(dout, din, (uint32_t)hm::ilog2(n), k);
    ck(cudaGetLastError(), "automorphism");
    ck(cudaMemcpy(v.data(), dout, T * 8, cudaMemcpyDeviceToHost), "download");
}

void pt_to_eval_host(std::vector<uint64_t>& out, const std::vector<int64_t>& m, uint32_t towers, uint32_t n,
                     const std::vector<uint64_t>& mod, const std::vector<uint64_t>& root) {
    const size_t T = (size_t)towers * n;
    need(xf_supported_logn(hm::ilog2(n)) && hm::is_pow2(n), "pt_to_eval_host: unsupported ring size");
    need(m.size() >= n && mod.size() >= towers && root.size() >= towers, "pt_to_eval_host: short input");
    out.resize(T);
    if (!T) return;
    const std::vector<ModC> mc = modcs(mod, towers);
    StageLease L = stage(stage_bytes({towers * sizeof(xf::Job), towers * sizeof(ModC), (size_t)n * 8, T * 8}));
    xf::Job* dj = L.take<xf::Job>(towers);
    ModC* dm = L.take<ModC>(towers);
    int64_t* dmsg = L.take<int64_t>(n);
    u64* d = L.take<u64>(T);
    ck(cudaMemcpy(dm, mc.data(), towers * sizeof(ModC), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(dmsg, m.data(), (size_t)n * 8, cudaMemcpyHostToDevice), "upload");
    k_embed_towers<<<dim3(grid_for(n), towers), 256>>>(d, dmsg, dm, n);
    ck(cudaGetLastError(), "embed");
    launch_xform(d, dj, towers, n, mod, root, false);
    ck(cudaMemcpy(out.data(), d, T * 8, cudaMemcpyDeviceToHost), "download");
}

namespace {
void pointwise_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, const std::vector<uint64_t>& d0,
                    const std::vector<uint64_t>* d1, uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod,
                    int mul) {
    const size_t T = (size_t)towers * n;
    need(c0.size() >= T && c1.size() >= T && d0.size() >= T && (!d1 || d1->size() >= T) && mod.size() >= towers,
         mul ? "ct_mul_pt_host: operand shorter than towers*n" : "ct_add_ct_host: operand shorter than towers*n");
    if (!T) return;
    const std::vector<ModC> mc = modcs(mod, towers);
    StageLease L = stage(stage_bytes({towers * sizeof(ModC), T * 8, T * 8, T * 8, d1 ? T * 8 : 0}));
    ModC* dm = L.take<ModC>(towers);
    u64* a0 = L.take<u64>(T);
    u64* a1 = L.take<u64>(T);
    u64* b0 = L.take<u64>(T);
    u64* b1 = d1 ? L.take<u64>(T) : b0;
    ck(cudaMemcpy(dm, mc.data(), towers * sizeof(ModC), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(a0, c0.data(), T * 8, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(a1, c1.data(), T * 8, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(b0, d0.data(), T * 8, cudaMemcpyHostToDevice), "upload");
    if (d1) ck(cudaMemcpy(b1, d1->data(), T * 8, cudaMemcpyHostToDevice), "upload");
    k_pointwise<<<dim3(grid_for(n), towers), 256>>>(a0, a1, b0, b1, dm, n, mul);
    ck(cudaGetLastError(), "pointwise");
    ck(cudaMemcpy(c0.data(), a0, T * 8, cudaMemcpyDeviceToHost), "download");
    ck(cudaMemcpy(c1.data(), a1, T * 8, cudaMemcpyDeviceToHost), "download");
}
}  // namespace

void ct_add_ct_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, const std::vector<uint64_t>& d0,
                    const std::vector<uint64_t>& d1, uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod) {
    pointwise_host(c0, c1, d0, &d1, towers, n, mod, 0);
}

void ct_mul_pt_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, const std::vector<uint64_t>& ptEval,
                    uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod) {
    pointwise_host(c0, c1, ptEval, nullptr, towers, n, mod, 1);
}

void rotate_ct_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, uint32_t k, const KeySwitchConstants& Krot,
                    uint32_t towers, uint32_t n, const std::vector<uint64_t>& mod,
                    const std::vector<uint64_t>& root) {
    // Same result as the reference's host-orchestrated form (coefficient
    // automorphism, keyswitch_core_resident, host add): the automorphism is
    // a permutation of eval slots and the keyswitch is the resident one.
    const size_t T = (size_t)towers * n;
    need(c0.size() >= T && c1.size() >= T, "rotate_ct_host: ciphertext shorter than towers*n");
    c0.resize(T);
    rotate_ct_resident(c0, c1, k, Krot, towers, n, mod, root);
}

// ---------------------------------------------------------------- host harness
void set_secret_hamming_weight(uint32_t h) { g_hw = h; }

KeyPairHost keygen_host(uint32_t n, const std::vector<uint64_t>& moduli, const std::vector<uint64_t>& roots,
                        uint64_t ns, double sigma, uint64_t seed) {
    const uint32_t sizeQ = (uint32_t)moduli.size();
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, sigma);
    std::vector<int> sc(n), ec(n);
    if (g_hw == 0) {
        for (uint32_t k = 0; k < n; ++k) sc[k] = (int)(rng() % 3) - 1;
    } else {
        std::vector<uint32_t> idx(n);
        for (uint32_t k = 0; k < n; ++k) idx[k] = k;
        for (uint32_t k = n - 1; k > 0; --k) { uint32_t j = (uint32_t)(rng() % (k + 1)); std::swap(idx[k], idx[j]); }
        const uint32_t h = g_hw < n ? g_hw : n;
        for (uint32_t k = 0; k < h; ++k) sc[idx[k]] = (rng() & 1ull) ? 1 : -1;
    }
    for (uint32_t k = 0; k < n; ++k) ec[k] = (int)std::lround(gauss(rng));
    KeyPairHost K;
    const size_t T = (size_t)sizeQ * n;
    K.s.resize(T); K.pkA.resize(T); K.pkB.resize(T);
    std::vector<u64> eT(T);
    for (uint32_t t = 0; t < sizeQ; ++t) {
        const u64 q = moduli[t];
        for (uint32_t k = 0; k < n; ++k) {
            const size_t x = (size_t)t * n + k;
            K.s[x] = emb(sc[k], q);
            eT[x] = emb(ec[k], q);
            K.pkA[x] = rng() % q;
        }
    }
    host_xform(K.s, sizeQ, n, moduli, roots, false);
    host_xform(eT, sizeQ, n, moduli, roots, false);
    for (uint32_t t = 0; t < sizeQ; ++t) {
        const u64 q = moduli[t];
        for (uint32_t k = 0; k < n; ++k) {
            const size_t x = (size_t)t * n + k;
            const u64 as = hm::mulmod(K.pkA[x], K.s[x], q);
            const u64 nse = hm::mulmod(ns % q, eT[x], q);
            K.pkB[x] = nse >= as ? nse - as : nse + q - as;
        }
    }
    return K;
}

void evalkeygen_host_sold(KeySwitchConstants& K, const std::vector<uint64_t>& /*sQP*/,
                          const std::vector<uint64_t>& sOld, const std::vector<uint64_t>& pkA_QP,
                          const std::vector<uint64_t>& pkB_QP, const std::vector<uint64_t>& PModq_QP,
                          const std::vector<uint64_t>& modQP, const std::vector<uint64_t>& rootQP, uint64_t ns,
                          double sigma, uint64_t seed) {
    const uint32_t n = K.n, sizeQlP = (uint32_t)modQP.size();
    const uint32_t sizeQl = K.sizeQl, alpha = K.alpha, numPart = K.numPart;
    K.evalKeyTowers = sizeQlP;
    K.av.assign(numPart, {});
    K.bv.assign(numPart, {});
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, sigma);
    const size_t T = (size_t)sizeQlP * n;
    for (uint32_t part = 0; part < numPart; ++part) {
        const uint32_t st = alpha * part;
        const uint32_t sp = (sizeQl > st + alpha) ? alpha : (sizeQl - st);
        const uint32_t en = st + sp;
        std::vector<int> uc(n), e0c(n), e1c(n);
        for (uint32_t k = 0; k < n; ++k) {
            uc[k] = (int)(rng() % 3) - 1;
            e0c[k] = (int)std::lround(gauss(rng));
            e1c[k] = (int)std::lround(gauss(rng));
        }
        std::vector<u64> uT(T), e0T(T), e1T(T);
        for (uint32_t t = 0; t < sizeQlP; ++t)
            for (uint32_t k = 0; k < n; ++k) {
                const size_t x = (size_t)t * n + k;
                uT[x] = emb(uc[k], modQP[t]); e0T[x] = emb(e0c[k], modQP[t]); e1T[x] = emb(e1c[k], modQP[t]);
            }
        host_xform(uT, sizeQlP, n, modQP, rootQP, false);
        host_xform(e0T, sizeQlP, n, modQP, rootQP, false);
        host_xform(e1T, sizeQlP, n, modQP, rootQP, false);
        K.av[part].resize(T);
        K.bv[part].resize(T);
        for (uint32_t t = 0; t < sizeQlP; ++t) {
            const u64 q = modQP[t];
            for (uint32_t k = 0; k < n; ++k) {
                const size_t x = (size_t)t * n + k;
                u64 a = hm::mulmod(pkA_QP[x], uT[x], q) + hm::mulmod(ns % q, e1T[x], q);
                u64 b = hm::mulmod(pkB_QP[x], uT[x], q) + hm::mulmod(ns % q, e0T[x], q);
                a = a >= q ? a - q : a;
                b = b >= q ? b - q : b;
                if (t >= st && t < en) {
                    b += hm::mulmod(PModq_QP[t] % q, sOld[x], q);
                    b = b >= q ? b - q : b;
                }
                K.av[part][x] = a;
                K.bv[part][x] = b;
            }
        }
    }
}

void evalkeygen_host(KeySwitchConstants& K, const std::vector<uint64_t>& sQP, const std::vector<uint64_t>& pkA_QP,
                     const std::vector<uint64_t>& pkB_QP, const std::vector<uint64_t>& PModq_QP,
                     const std::vector<uint64_t>& modQP, const std::vector<uint64_t>& rootQP, uint64_t ns,
                     double sigma, uint64_t seed) {
    const uint32_t n = K.n, sizeQlP = (uint32_t)modQP.size();
    std::vector<u64> s2(sQP.size());
    for (uint32_t t = 0; t < sizeQlP; ++t)
        for (uint32_t k = 0; k < n; ++k) {
            const size_t x = (size_t)t * n + k;
            s2[x] = hm::mulmod(sQP[x], sQP[x], modQP[t]);
        }
    evalkeygen_host_sold(K, sQP, s2, pkA_QP, pkB_QP, PModq_QP, modQP, rootQP, ns, sigma, seed);
}

void encrypt_host(std::vector<uint64_t>& c0, std::vector<uint64_t>& c1, const std::vector<int64_t>& m,
                  const std::vector<uint64_t>& pkA, const std::vector<uint64_t>& pkB, uint32_t n,
                  const std::vector<uint64_t>& mod, const std::vector<uint64_t>& root, uint64_t ns, double sigma,
                  uint64_t seed) {
    const uint32_t sizeQ = (uint32_t)mod.size();
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> g(0.0, sigma);
    std::vector<int> vc(n), e0c(n), e1c(n);
    for (uint32_t k = 0; k < n; ++k) {
        vc[k] = (int)(rng() % 3) - 1;
        e0c[k] = (int)std::lround(g(rng));
        e1c[k] = (int)std::lround(g(rng));
    }
    const size_t T = (size_t)sizeQ * n;
    std::vector<u64> vT(T), e0T(T), e1T(T), mT(T);
    for (uint32_t t = 0; t < sizeQ; ++t)
        for (uint32_t k = 0; k < n; ++k) {
            const size_t x = (size_t)t * n + k;
            const u64 q = mod[t];
            vT[x] = emb(vc[k], q); e0T[x] = emb(e0c[k], q); e1T[x] = emb(e1c[k], q); mT[x] = emb((long)m[k], q);
        }
    for (auto* v : {&vT, &e0T, &e1T, &mT}) host_xform(*v, sizeQ, n, mod, root, false);
    c0.resize(T);
    c1.resize(T);
    for (uint32_t t = 0; t < sizeQ; ++t) {
        const u64 q = mod[t];
        for (uint32_t k = 0; k < n; ++k) {
            const size_t x = (size_t)t * n + k;
            u64 b = hm::mulmod(pkB[x], vT[x], q) + hm::mulmod(ns % q, e0T[x], q);
            b = b >= q ? b - q : b;
            u64 a = hm::mulmod(pkA[x], vT[x], q) + hm::mulmod(ns % q, e1T[x], q);
            a = a >= q ? a - q : a;
            b += mT[x];
            c0[x] = b >= q ? b - q : b;
            c1[x] = a;
        }
    }
}

void decrypt_host(std::vector<int64_t>& mout, const std::vector<uint64_t>& c0, const std::vector<uint64_t>& c1,
                  const std::vector<uint64_t>& s, uint32_t n, const std::vector<uint64_t>& mod,
                  const std::vector<uint64_t>& root) {
    const u64 q = mod[0];
    std::vector<u64> ph(n);
    for (uint32_t k = 0; k < n; ++k) {
        u64 v = c0[k] + hm::mulmod(c1[k], s[k], q);
        ph[k] = v >= q ? v - q : v;
    }
    host_xform(ph, 1, n, {q}, {root[0]}, true);
    mout.resize(n);
    for (uint32_t k = 0; k < n; ++k) mout[k] = ph[k] > q / 2 ? (int64_t)ph[k] - (int64_t)q : (int64_t)ph[k];
}

}  // namespace gpufhe
