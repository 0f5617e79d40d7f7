// Key generation, encryption, decryption and ModRaise on the device
// (include/gpufhe_b200.h).
//
// The reference builds every key and ciphertext with host loops: per tower it
// embeds the sampled small polynomials, uploads them to a fresh cudaMalloc,
// runs one NTT launch, copies back and multiplies on the host
// (src/keygen.cpp:55-112, src/evalkeygen.cpp:42-113, src/encdec.cpp:41-81).
// Here only the random draws stay on the host, because they must reproduce the
// reference's sequential std::mt19937_64 / std::normal_distribution stream
// exactly (same seed, same keys); independent keys and messages draw in
// parallel host threads. Everything else runs as a few launches over the whole
// batch: embedding of the small polynomials into every tower, one batched
// NTT (or INTT) launch over every tower of every polynomial, and one
// elementwise kernel for the products. Eval keys go straight into the
// context's resident key storage.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>
#include <thread>
#include <vector>

#include "context.hpp"
#include "gpufhe_b200.h"
#include "hostmath.hpp"
#include "xform.cuh"

gfx::Context* gpufhe_impl(gpufhe_ctx* h);

namespace {

using gfx::Context;
constexpr unsigned KNT = 256;

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

unsigned blocks_for(size_t words) { return (unsigned)std::min<size_t>((words + KNT - 1) / KNT, 148u * 64u); }

// ---------------------------------------------------------------- host draws
// Same draw order as the reference (keygen.cpp:60-87 secret and error, then
// the uniform a tower by tower inside the tower loop).
void draw_keygen(uint32_t n, const std::vector<u64>& mods, uint32_t towers, uint32_t hw, double sigma, u64 seed,
                 int32_t* s, int32_t* e, u64* a) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, sigma);
    if (hw == 0) {
        for (uint32_t k = 0; k < n; ++k) s[k] = (int32_t)(rng() % 3) - 1;
    } else {
        std::vector<uint32_t> idx(n);
        for (uint32_t k = 0; k < n; ++k) idx[k] = k;
        for (uint32_t k = n - 1; k > 0; --k) std::swap(idx[k], idx[(uint32_t)(rng() % (k + 1))]);
        std::fill(s, s + n, 0);
        const uint32_t h = hw < n ? hw : n;
        for (uint32_t k = 0; k < h; ++k) s[idx[k]] = (rng() & 1ull) ? 1 : -1;
    }
    for (uint32_t k = 0; k < n; ++k) e[k] = (int32_t)std::lround(gauss(rng));
    for (uint32_t t = 0; t < towers; ++t)
        for (uint32_t k = 0; k < n; ++k) a[(size_t)t * n + k] = rng() % mods[t];
}

// Per digit p: ternary u, Gaussian e0, e1, drawn per coefficient in that
// order (evalkeygen.cpp:75-77); out[p][3][n]. The same order serves
// encryption (v, e0, e1 per coefficient, encdec.cpp:51-52) with parts = 1.
void draw_tern_gauss2(uint32_t n, uint32_t parts, double sigma, u64 seed, int32_t* out) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, sigma);
    for (uint32_t p = 0; p < parts; ++p) {
        int32_t* u = out + (size_t)p * 3 * n;
        for (uint32_t k = 0; k < n; ++k) {
            u[k] = (int32_t)(rng() % 3) - 1;
            u[n + k] = (int32_t)std::lround(gauss(rng));
            u[2 * n + k] = (int32_t)std::lround(gauss(rng));
        }
    }
}

// Runs f(i) for i < count on up to hardware_concurrency threads.
template <class F>
void parallel_for(uint32_t count, F&& f) {
    const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint32_t nt = std::min(count, hw);
    if (nt <= 1) {
        for (uint32_t i = 0; i < count; ++i) f(i);
        return;
    }
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < nt; ++w)
        th.emplace_back([&, w] {
            for (uint32_t i = w; i < count; i += nt) f(i);
        });
    for (auto& t : th) t.join();
}

// ---------------------------------------------------------------- kernels
// x mod q for a signed value (the reference's ((v % q) + q) % q).
template <class S>
__device__ __forceinline__ u64 emb(S v, const ModC& m) {
    const long long x = (long long)v;
    const u64 mag = x < 0 ? 0ull - (u64)x : (u64)x;
    const u64 r = reduce64(mag, m);
    return (x < 0 && r) ? m.q - r : r;
}

// out[p][t][k] = src[p][k] mod QP[first + t], p < polys.
template <class S>
__global__ void k_embed(const S* __restrict__ src, u64* __restrict__ out, const ModC* __restrict__ mod,
                        uint32_t polys, uint32_t towers, uint32_t n) {
    const size_t total = (size_t)polys * towers * n;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i / ((size_t)towers * n);
        const uint32_t t = (uint32_t)((i / n) % towers);
        out[i] = emb(src[p * n + i % n], mod[t]);
    }
}

// Public key: b = ns*e - a*s over towers x n (keygen.cpp:100-105).
__global__ void k_keygen_b(const u64* __restrict__ s, const u64* __restrict__ e, const u64* __restrict__ a,
                           u64* __restrict__ b, const ModC* __restrict__ mod, uint32_t towers, uint32_t n, u64 ns) {
    const size_t total = (size_t)towers * n;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const ModC m = mod[i / n];
        const u64 as = mulmod(a[i], s[i], m);
        const u64 nse = mulmod(reduce64(ns, m), e[i], m);
        b[i] = nse >= as ? nse - as : nse + m.q - as;
    }
}

// Eval-slot index of the Galois automorphism X -> X^k in the bit-reversed
// NTT order: sigma_k(a)[j] = a[slot(j)].
__device__ __forceinline__ uint32_t galois_slot_rt(uint32_t j, u64 k, uint32_t logn) {
    const uint32_t e = 2 * (__brev(j) >> (32 - logn)) + 1;
    const uint32_t t = (uint32_t)(((u64)e * k) & ((2ull << logn) - 1));
    return __brev((t - 1) >> 1) >> (32 - logn);
}

struct EvkJob {
    const u64* uee;   // [dnum][3][QP][n] NTT'd u, e0, e1
    u64* av;          // [dnum][QP][n]
    u64* bv;
    u64 galois;       // 0: sOld = s^2, else sigma_galois(s)
};

// Per (key, digit p, QP tower t): av = pkA*u + ns*e1, bv = pkB*u + ns*e0,
// plus (P mod q_t) * sOld on the digit's own Q towers [alpha p, alpha p + sp)
// (evalkeygen.cpp:80-93).
__global__ void k_evalkey(const EvkJob* __restrict__ jobs, const u64* __restrict__ s, const u64* __restrict__ pkA,
                          const u64* __restrict__ pkB, const u64* __restrict__ pmodq, const ModC* __restrict__ mod,
                          uint32_t dnum, uint32_t QP, uint32_t fullQ, uint32_t alpha, uint32_t n, uint32_t logn,
                          u64 ns) {
    const EvkJob J = jobs[blockIdx.z];
    const uint32_t p = blockIdx.y / QP, t = blockIdx.y % QP;
    const ModC m = mod[t];
    const uint32_t st = alpha * p, en = min(st + alpha, fullQ);
    const bool own = t >= st && t < en;
    const u64 nsq = reduce64(ns, m);
    const u64* u = J.uee + ((size_t)p * 3 * QP + t) * n;
    const u64* e0 = u + (size_t)QP * n;
    const u64* e1 = e0 + (size_t)QP * n;
    const size_t row = (size_t)t * n;
    u64* av = J.av + ((size_t)p * QP + t) * n;
    u64* bv = J.bv + ((size_t)p * QP + t) * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        u64 a = mulmod(pkA[row + k], u[k], m) + mulmod(nsq, e1[k], m);
        u64 b = mulmod(pkB[row + k], u[k], m) + mulmod(nsq, e0[k], m);
        a = csub(a, m.q);
        b = csub(b, m.q);
        if (own) {
            const u64 so = J.galois ? s[row + galois_slot_rt(k, J.galois, logn)] : mulmod(s[row + k], s[row + k], m);
            b = csub(b + mulmod(pmodq[t], so, m), m.q);
        }
        av[k] = a;
        bv[k] = b;
    }
}

// c0 = pkB*v + ns*e0 + m, c1 = pkA*v + ns*e1 (encdec.cpp:55-61); vem[msg] holds
// the NTT'd [v, e0, e1, m][towers][n].
__global__ void k_encrypt(const u64* __restrict__ vem, const u64* __restrict__ pkA, const u64* __restrict__ pkB,
                          u64* const* __restrict__ c0s, u64* const* __restrict__ c1s, const ModC* __restrict__ mod,
                          uint32_t towers, uint32_t n, u64 ns) {
    const uint32_t msg = blockIdx.z, t = blockIdx.y;
    const ModC m = mod[t];
    const size_t T = (size_t)towers * n, row = (size_t)t * n;
    const u64* v = vem + (size_t)msg * 4 * T + row;
    const u64 nsq = reduce64(ns, m);
    u64* c0 = c0s[msg] + row;
    u64* c1 = c1s[msg] + row;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const u64 b = csub(mulmod(pkB[row + k], v[k], m) + mulmod(nsq, v[T + k], m), m.q);
        const u64 a = csub(mulmod(pkA[row + k], v[k], m) + mulmod(nsq, v[2 * T + k], m), m.q);
        c0[k] = csub(b + v[3 * T + k], m.q);
        c1[k] = a;
    }
}

// ph[ct][t] = c0 + c1 * s over the first `towers` Q towers.
__global__ void k_phase(const u64* const* __restrict__ c0s, const u64* const* __restrict__ c1s,
                        const u64* __restrict__ s, u64* __restrict__ ph, const ModC* __restrict__ mod,
                        uint32_t towers, uint32_t n) {
    const uint32_t ct = blockIdx.z, t = blockIdx.y;
    const ModC m = mod[t];
    const size_t row = (size_t)t * n;
    const u64* c0 = c0s[ct] + row;
    const u64* c1 = c1s[ct] + row;
    u64* out = ph + ((size_t)ct * towers + t) * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        out[k] = csub(c0[k] + mulmod(c1[k], s[row + k], m), m.q);
}

// Tower-0 decryption (encdec.cpp:73-80): centred residue mod q0.
__global__ void k_center0(const u64* __restrict__ ph, int64_t* __restrict__ out, u64 q, size_t words) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x) {
        const u64 v = ph[i];
        out[i] = v > q / 2 ? (int64_t)v - (int64_t)q : (int64_t)v;
    }
}

struct CrtConst {
    uint32_t L;
    const ModC* mod;       // [L]
    const u64* inv;        // [L][L]: inv[j * L + i] = q_j^-1 mod q_i (j < i)
    const u64* prefix;     // [L][2]: prod_{j<i} q_j mod 2^128 (lo, hi)
    const u64* half;       // [L]: mixed-radix digits of (Q - 1) / 2
    u64 qlo, qhi;          // Q mod 2^128
};

// Exact centred CRT reconstruction of every coefficient (Garner's mixed-radix
// digits v_i, value = sum v_i prod_{j<i} q_j), as a two's-complement 128-bit
// integer; exact whenever |value| < 2^127. out[ct][k] = {lo, hi}.
__global__ void k_garner(const u64* __restrict__ ph, u64* __restrict__ out, CrtConst C, uint32_t n, size_t words) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x) {
        const size_t ct = i / n, k = i % n;
        const u64* p = ph + ct * C.L * n + k;
        u64 v[gfx::MAXQ];
        u64 lo = 0, hi = 0;
        for (uint32_t t = 0; t < C.L; ++t) {
            const ModC m = C.mod[t];
            u64 x = p[(size_t)t * n];
            for (uint32_t j = 0; j < t; ++j) {
                const u64 vj = reduce64(v[j], m);
                x = mulmod(x >= vj ? x - vj : x + m.q - vj, C.inv[j * C.L + t], m);
            }
            v[t] = x;
            // (lo, hi) += x * prefix_t mod 2^128
            u64 a_lo, a_hi;
            mul_wide(x, C.prefix[2 * t], a_lo, a_hi);
            a_hi += x * C.prefix[2 * t + 1];
            add_wide(lo, hi, a_lo, a_hi);
        }
        int cmp = 0;   // value vs (Q - 1) / 2, most significant digit first
        for (int t = (int)C.L - 1; t >= 0 && !cmp; --t) cmp = v[t] > C.half[t] ? 1 : (v[t] < C.half[t] ? -1 : 0);
        if (cmp > 0) {   // value - Q
            const u64 nlo = lo - C.qlo;
            hi = hi - C.qhi - (lo < C.qlo ? 1 : 0);
            lo = nlo;
        }
        out[2 * i] = lo;
        out[2 * i + 1] = hi;
    }
}

// ---------------------------------------------------------------- host helpers
// ModRaise, first step: x[p][k] = in[p][k] for the 2*count components
// (p even: c0 of ciphertext p/2, odd: c1), tower 0 only.
__global__ void k_gather_tower0(const u64* const* __restrict__ in, u64* __restrict__ x, uint32_t n) {
    const u64* src = in[blockIdx.y];
    u64* dst = x + (size_t)blockIdx.y * n;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) dst[k] = src[k];
}

struct Scratch {
    cudaStream_t s;
    std::vector<void*> ptrs;
    explicit Scratch(cudaStream_t st) : s(st) {}
    template <class T>
    T* get(size_t count) {
        void* p = nullptr;
        ck(cudaMallocAsync(&p, std::max<size_t>(count * sizeof(T), 16), s), "cudaMallocAsync");
        ptrs.push_back(p);
        return (T*)p;
    }
    ~Scratch() {
        for (void* p : ptrs) cudaFreeAsync(p, s);
    }
};

std::vector<u64> qp_moduli(const Context& c) {
    std::vector<u64> m(c.Q());
    m.insert(m.end(), c.P().begin(), c.P().end());
    return m;
}

// One transform job for QP tower qi of the context on x.
xf::Job xjob(const Context& c, const std::vector<u64>& qp, u64* x, uint32_t qi, bool inverse) {
    const gfx::DevCtx& D = c.dev();
    const uint32_t n = c.n();
    xf::Job j{};
    j.x = x;
    j.tw = (inverse ? D.twi : D.twf) + (size_t)qi * n;
    j.q = qp[qi];
    j.scale = c.ninv_host()[qi];   // n^-1 (inverse transforms), kept by the context
    j.scale_p = c.ninvp_host()[qi];
    j.fp = fp_tower(j.q) ? 1u : 0u;
    j.twd = j.fp ? (inverse ? D.twid : D.twfd) + (size_t)qi * n : nullptr;
    return j;
}

template <class T>
T* upload(Scratch& S, const std::vector<T>& h) {
    T* d = S.get<T>(h.size());
    ck(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, S.s), "upload");
    // (a copy from pageable memory has read `h` when it returns)
    return d;
}

// Job p * towers + t of a batch: the template of tower t on x = xs[p] + t n
// (xs given) or base + (p * towers + t) n, lifting from lift + p n when lift
// is set. Built on the device, so a batch of thousands of tower transforms
// costs the host one template per tower.
__global__ void k_tower_jobs(xf::Job* __restrict__ jobs, const xf::Job* __restrict__ tmpl, u64* const* __restrict__ xs,
                             u64* base, const u64* lift, uint32_t polys, uint32_t towers, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= polys * towers) return;
    const uint32_t p = i / towers, t = i % towers;
    xf::Job j = tmpl[t];
    j.x = xs ? xs[p] + (size_t)t * n : base + (size_t)i * n;
    if (lift) j.lift = lift + (size_t)p * n;
    jobs[i] = j;
}

// Device job table for polys x towers transforms (see k_tower_jobs); with
// `lift`, every job's column pass lifts from it (lift_q0 as in xf::Job).
xf::Job* tower_jobs(const Context& c, const std::vector<u64>& qp, Scratch& S, uint32_t polys, uint32_t towers,
                    bool inverse, u64* const* xs, u64* base, const u64* lift = nullptr, u64 lift_q0 = 0) {
    std::vector<xf::Job> tmpl(towers);
    for (uint32_t t = 0; t < towers; ++t) {
        tmpl[t] = xjob(c, qp, nullptr, t, inverse);
        if (lift) {
            tmpl[t].lift_q0 = lift_q0;
            tmpl[t].lift_r64 = ~0ull / qp[t];
        }
    }
    const xf::Job* dt = upload(S, tmpl);
    xf::Job* dj = S.get<xf::Job>((size_t)polys * towers);
    const uint32_t total = polys * towers;
    k_tower_jobs<<<(total + 255) / 256, 256, 0, S.s>>>(dj, dt, xs, base, lift, polys, towers, c.n());
    ck(cudaGetLastError(), "job table");
    return dj;
}

// Transforms polys x towers tower-polys at base ([poly][tower][n], tower t
// uses QP modulus t) in one launch pair.
void transform(const Context& c, const std::vector<u64>& qp, Scratch& S, u64* base, uint32_t polys,
               uint32_t towers, bool inverse) {
    xf::Job* dj = tower_jobs(c, qp, S, polys, towers, inverse, nullptr, base);
    ck(xf_launch_ntt(dj, nullptr, (int)(polys * towers), (int)c.logn(), inverse, S.s), "transform");
}

#define KEYS_TRY(...)                                                          \
    try { __VA_ARGS__ } catch (const std::invalid_argument& e) {               \
        gfx::set_error(e.what()); return GPUFHE_EINVAL;                        \
    } catch (const std::length_error& e) {                                     \
        gfx::set_error(e.what()); return GPUFHE_ENOMEM;                        \
    } catch (const std::exception& e) {                                        \
        gfx::set_error(e.what()); return GPUFHE_ECUDA;                         \
    }

}  // namespace

extern "C" {

int gpufhe_keygen(gpufhe_ctx* h, uint32_t towers, uint32_t hw, uint64_t ns, double sigma, uint64_t seed,
                  uint64_t* d_s, uint64_t* d_pkA, uint64_t* d_pkB, cudaStream_t stream) {
    Context* c = gpufhe_impl(h);
    if (!c || !d_s || !d_pkA || !d_pkB) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!towers || towers > c->fullQ() + c->K()) { gfx::set_error("keygen: towers out of range"); return GPUFHE_EINVAL; }
    KEYS_TRY({
        const uint32_t n = c->n();
        const std::vector<u64> qp = qp_moduli(*c);
        std::vector<int32_t> se(2 * (size_t)n);
        std::vector<u64> a((size_t)towers * n);
        draw_keygen(n, qp, towers, hw, sigma, seed, se.data(), se.data() + n, a.data());
        Scratch S(stream);
        const int32_t* dse = upload(S, se);
        ck(cudaMemcpyAsync(d_pkA, a.data(), a.size() * 8, cudaMemcpyHostToDevice, stream), "upload a");
        u64* de = S.get<u64>((size_t)towers * n);
        const size_t T = (size_t)towers * n;
        const ModC* mod = c->dev().mod;
        k_embed<<<blocks_for(T), KNT, 0, stream>>>(dse, d_s, mod, 1, towers, n);
        k_embed<<<blocks_for(T), KNT, 0, stream>>>(dse + n, de, mod, 1, towers, n);
        ck(cudaGetLastError(), "embed");
        // s and e are two polys of `towers` towers but not adjacent: two job sets
        std::vector<xf::Job> jobs(2 * (size_t)towers);
        for (uint32_t t = 0; t < towers; ++t) {
            jobs[t] = xjob(*c, qp, d_s + (size_t)t * n, t, false);
            jobs[towers + t] = xjob(*c, qp, de + (size_t)t * n, t, false);
        }
        xf::Job* dj = upload(S, jobs);
        ck(xf_launch_ntt(dj, nullptr, (int)jobs.size(), (int)c->logn(), false, stream), "transform");
        k_keygen_b<<<blocks_for(T), KNT, 0, stream>>>(d_s, de, d_pkA, d_pkB, mod, towers, n, ns);
        ck(cudaGetLastError(), "keygen");
        ck(cudaStreamSynchronize(stream), "keygen sync");
        return GPUFHE_OK;
    })
}

int gpufhe_ctx_set_key_device(gpufhe_ctx* h, uint64_t key_id, const uint64_t* d_av, const uint64_t* d_bv) {
    Context* c = gpufhe_impl(h);
    if (!c || !d_av || !d_bv) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    KEYS_TRY({
        c->set_key(key_id, d_av, d_bv, true);
        return GPUFHE_OK;
    })
}

int gpufhe_evalkeygen(gpufhe_ctx* h, uint32_t count, const uint64_t* key_ids, const uint64_t* galois,
                      const uint64_t* seeds, const uint64_t* d_sQP, const uint64_t* d_pkA, const uint64_t* d_pkB,
                      uint64_t ns, double sigma, uint64_t* const* d_av_out, uint64_t* const* d_bv_out,
                      cudaStream_t stream) {
    Context* c = gpufhe_impl(h);
    if (!c || !key_ids || !galois || !seeds || !d_sQP || !d_pkA || !d_pkB) {
        gfx::set_error("null argument");
        return GPUFHE_EINVAL;
    }
    const uint32_t n = c->n();
    for (uint32_t i = 0; i < count; ++i)
        if (galois[i] && (!(galois[i] & 1) || galois[i] >= 2ull * n)) {
            gfx::set_error("evalkeygen: Galois element must be odd and below 2n (0 = relinearisation)");
            return GPUFHE_EINVAL;
        }
    KEYS_TRY({
        const std::vector<u64> qp = qp_moduli(*c);
        const uint32_t QP = (uint32_t)qp.size(), dnum = c->dnum(), fullQ = c->fullQ();
        const size_t T = (size_t)QP * n, keyw = (size_t)dnum * T;
        std::vector<u64> pmodq(QP);
        for (uint32_t t = 0; t < QP; ++t) pmodq[t] = hm::prod_mod(c->P().data(), c->K(), qp[t]);
        Scratch S(stream);
        const u64* dpm = upload(S, pmodq);
        // keys in chunks so that the temporaries stay near 1.5 GB at n = 2^16
        const uint32_t chunk = (uint32_t)std::max<size_t>(1, ((size_t)1536 << 20) / (keyw * 8 * 5));
        for (uint32_t k0 = 0; k0 < count; k0 += chunk) {
            const uint32_t kc = std::min(chunk, count - k0);
            std::vector<int32_t> small((size_t)kc * dnum * 3 * n);
            parallel_for(kc, [&](uint32_t i) {
                draw_tern_gauss2(n, dnum, sigma, seeds[k0 + i], small.data() + (size_t)i * dnum * 3 * n);
            });
            Scratch C(stream);
            const int32_t* dsmall = upload(C, small);
            u64* uee = C.get<u64>((size_t)kc * 3 * keyw);
            u64* keys = C.get<u64>((size_t)kc * 2 * keyw);
            const uint32_t polys = kc * dnum * 3;
            k_embed<<<blocks_for((size_t)polys * T), KNT, 0, stream>>>(dsmall, uee, c->dev().mod, polys, QP, n);
            ck(cudaGetLastError(), "embed");
            transform(*c, qp, C, uee, polys, QP, false);
            std::vector<EvkJob> jobs(kc);
            for (uint32_t i = 0; i < kc; ++i)
                jobs[i] = EvkJob{uee + (size_t)i * 3 * keyw, keys + (size_t)i * 2 * keyw,
                                 keys + (size_t)i * 2 * keyw + keyw, galois[k0 + i]};
            const EvkJob* dj = upload(C, jobs);
            const dim3 grid((n + KNT - 1) / KNT, dnum * QP, kc);
            k_evalkey<<<grid, KNT, 0, stream>>>(dj, d_sQP, d_pkA, d_pkB, dpm, c->dev().mod, dnum, QP, fullQ,
                                                c->alpha(), n, c->logn(), ns);
            ck(cudaGetLastError(), "evalkey");
            for (uint32_t i = 0; i < kc; ++i) {
                const u64* av = keys + (size_t)i * 2 * keyw;
                const u64* bv = av + keyw;
                if (d_av_out && d_av_out[k0 + i])
                    ck(cudaMemcpyAsync(d_av_out[k0 + i], av, keyw * 8, cudaMemcpyDeviceToDevice, stream), "copy av");
                if (d_bv_out && d_bv_out[k0 + i])
                    ck(cudaMemcpyAsync(d_bv_out[k0 + i], bv, keyw * 8, cudaMemcpyDeviceToDevice, stream), "copy bv");
                ck(cudaStreamSynchronize(stream), "evalkey sync");
                c->set_key(key_ids[k0 + i], av, bv, true);
            }
        }
        ck(cudaStreamSynchronize(stream), "evalkeygen sync");
        return GPUFHE_OK;
    })
}

int gpufhe_encrypt_batch(gpufhe_ctx* h, uint32_t count, uint32_t towers, const int64_t* m, const uint64_t* seeds,
                         const uint64_t* d_pkA, const uint64_t* d_pkB, uint64_t ns, double sigma,
                         uint64_t* const* d_c0, uint64_t* const* d_c1, cudaStream_t stream) {
    Context* c = gpufhe_impl(h);
    if (!c || !m || !seeds || !d_pkA || !d_pkB || !d_c0 || !d_c1) {
        gfx::set_error("null argument");
        return GPUFHE_EINVAL;
    }
    if (!towers || towers > c->fullQ() + c->K()) { gfx::set_error("encrypt: towers out of range"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    KEYS_TRY({
        const uint32_t n = c->n();
        const std::vector<u64> qp = qp_moduli(*c);
        const size_t T = (size_t)towers * n;
        // at most ~1 GB of temporaries per round of messages
        const uint32_t chunk = (uint32_t)std::max<size_t>(1, ((size_t)1 << 30) / (4 * T * 8));
        for (uint32_t m0 = 0; m0 < count; m0 += chunk) {
            const uint32_t mc = std::min(chunk, count - m0);
            std::vector<int32_t> small((size_t)mc * 3 * n);
            parallel_for(mc, [&](uint32_t i) { draw_tern_gauss2(n, 1, sigma, seeds[m0 + i], small.data() + (size_t)i * 3 * n); });
            Scratch C(stream);
            const int32_t* dsmall = upload(C, small);
            int64_t* dm = C.get<int64_t>((size_t)mc * n);
            ck(cudaMemcpyAsync(dm, m + (size_t)m0 * n, (size_t)mc * n * 8, cudaMemcpyHostToDevice, stream), "upload m");
            u64* vem = C.get<u64>((size_t)mc * 4 * T);
            // [msg][v, e0, e1, m][towers][n]: the small triple of each message
            // lands in slots 0..2, the message in slot 3
            for (uint32_t i = 0; i < mc; ++i) {
                k_embed<<<blocks_for(3 * T), KNT, 0, stream>>>(dsmall + (size_t)i * 3 * n, vem + (size_t)i * 4 * T,
                                                               c->dev().mod, 3, towers, n);
                k_embed<<<blocks_for(T), KNT, 0, stream>>>(dm + (size_t)i * n, vem + (size_t)i * 4 * T + 3 * T,
                                                           c->dev().mod, 1, towers, n);
            }
            ck(cudaGetLastError(), "embed");
            transform(*c, qp, C, vem, mc * 4, towers, false);
            std::vector<u64*> p0(d_c0 + m0, d_c0 + m0 + mc), p1(d_c1 + m0, d_c1 + m0 + mc);
            u64* const* dp0 = upload(C, p0);
            u64* const* dp1 = upload(C, p1);
            k_encrypt<<<dim3((n + KNT - 1) / KNT, towers, mc), KNT, 0, stream>>>(vem, d_pkA, d_pkB, dp0, dp1,
                                                                                c->dev().mod, towers, n, ns);
            ck(cudaGetLastError(), "encrypt");
            ck(cudaStreamSynchronize(stream), "encrypt sync");
        }
        return GPUFHE_OK;
    })
}

int gpufhe_decrypt_batch(gpufhe_ctx* h, uint32_t count, const uint64_t* const* d_c0, const uint64_t* const* d_c1,
                         const uint64_t* d_s, int64_t* m_out, cudaStream_t stream) {
    Context* c = gpufhe_impl(h);
    if (!c || !d_c0 || !d_c1 || !d_s || !m_out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    KEYS_TRY({
        const uint32_t n = c->n();
        const std::vector<u64> qp = qp_moduli(*c);
        Scratch S(stream);
        u64* ph = S.get<u64>((size_t)count * n);
        const u64* const* dp0 = upload(S, std::vector<const u64*>(d_c0, d_c0 + count));
        const u64* const* dp1 = upload(S, std::vector<const u64*>(d_c1, d_c1 + count));
        k_phase<<<dim3((n + KNT - 1) / KNT, 1, count), KNT, 0, stream>>>(dp0, dp1, d_s, ph, c->dev().mod, 1, n);
        ck(cudaGetLastError(), "phase");
        transform(*c, qp, S, ph, count, 1, true);
        int64_t* dout = S.get<int64_t>((size_t)count * n);
        k_center0<<<blocks_for((size_t)count * n), KNT, 0, stream>>>(ph, dout, qp[0], (size_t)count * n);
        ck(cudaGetLastError(), "center");
        ck(cudaMemcpyAsync(m_out, dout, (size_t)count * n * 8, cudaMemcpyDeviceToHost, stream), "download");
        ck(cudaStreamSynchronize(stream), "decrypt sync");
        return GPUFHE_OK;
    })
}

int gpufhe_decrypt_crt_batch(gpufhe_ctx* h, uint32_t count, uint32_t towers, const uint64_t* const* d_c0,
                             const uint64_t* const* d_c1, const uint64_t* d_s, uint64_t* out128,
                             cudaStream_t stream) {
    Context* c = gpufhe_impl(h);
    if (!c || !d_c0 || !d_c1 || !d_s || !out128) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!towers || towers > c->fullQ()) { gfx::set_error("decrypt: towers out of range"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    KEYS_TRY({
        const uint32_t n = c->n(), L = towers;
        const std::vector<u64> qp = qp_moduli(*c);
        Scratch S(stream);
        const size_t words = (size_t)count * n;
        u64* ph = S.get<u64>(words * L);
        const u64* const* dp0 = upload(S, std::vector<const u64*>(d_c0, d_c0 + count));
        const u64* const* dp1 = upload(S, std::vector<const u64*>(d_c1, d_c1 + count));
        k_phase<<<dim3((n + KNT - 1) / KNT, L, count), KNT, 0, stream>>>(dp0, dp1, d_s, ph, c->dev().mod, L, n);
        ck(cudaGetLastError(), "phase");
        transform(*c, qp, S, ph, count, L, true);
        // Garner constants
        std::vector<u64> inv((size_t)L * L, 0), prefix(2 * (size_t)L), half(L);
        unsigned __int128 pre = 1;
        for (uint32_t t = 0; t < L; ++t) {
            prefix[2 * t] = (u64)pre;
            prefix[2 * t + 1] = (u64)(pre >> 64);
            pre *= qp[t];
            for (uint32_t j = 0; j < t; ++j) inv[j * L + t] = hm::invmod(qp[j] % qp[t], qp[t]);
        }
        u64 carry = 0;   // (Q - 1) / 2 from the digits q_t - 1 of Q - 1, top digit first
        for (int t = (int)L - 1; t >= 0; --t) {
            const unsigned __int128 cur = (unsigned __int128)carry * qp[t] + (qp[t] - 1);
            half[t] = (u64)(cur >> 1);
            carry = (u64)(cur & 1);
        }
        CrtConst C{L, c->dev().mod, upload(S, inv), upload(S, prefix), upload(S, half), (u64)pre, (u64)(pre >> 64)};
        u64* dout = S.get<u64>(2 * words);
        k_garner<<<blocks_for(words), KNT, 0, stream>>>(ph, dout, C, n, words);
        ck(cudaGetLastError(), "crt");
        ck(cudaMemcpyAsync(out128, dout, 2 * words * 8, cudaMemcpyDeviceToHost, stream), "download");
        ck(cudaStreamSynchronize(stream), "decrypt sync");
        return GPUFHE_OK;
    })
}

int gpufhe_pt_to_eval_batch(gpufhe_ctx* h, uint32_t count, uint32_t towers, const int64_t* d_m,
                            uint64_t* const* d_out, cudaStream_t stream) {
    Context* c = gpufhe_impl(h);
    if (!c || !d_m || !d_out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!towers || towers > c->fullQ()) { gfx::set_error("pt_to_eval: towers out of range"); return GPUFHE_EINVAL; }
    if (count > 65535) { gfx::set_error("pt_to_eval: at most 65535 plaintexts per call"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    KEYS_TRY({
        const uint32_t n = c->n();
        const std::vector<u64> qp = qp_moduli(*c);
        std::vector<u64*> out(d_out, d_out + count);
        for (u64* o : out)
            if (!o) throw std::invalid_argument("pt_to_eval: null output pointer");
        Scratch S(stream);
        // each tower's forward transform reads the message and embeds it on
        // load (lift_q0 = 0: signed 64-bit coefficients)
        u64* const* dout = upload(S, out);
        xf::Job* dj = tower_jobs(*c, qp, S, count, towers, false, dout, nullptr, reinterpret_cast<const u64*>(d_m), 0);
        ck(xf_launch_ntt_lift(dj, (int)(count * towers), (int)c->logn(), stream), "pt_to_eval transform");
        return GPUFHE_OK;
    })
}

int gpufhe_modraise_batch(gpufhe_ctx* h, uint32_t count, uint32_t towers, const uint64_t* const* d_c0_in,
                          const uint64_t* const* d_c1_in, uint64_t* const* d_c0_out, uint64_t* const* d_c1_out,
                          cudaStream_t stream) {
    Context* c = gpufhe_impl(h);
    if (!c || !d_c0_in || !d_c1_in || !d_c0_out || !d_c1_out) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!towers || towers > c->fullQ()) { gfx::set_error("modraise: towers out of range"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    if (2 * (size_t)count > 65535) { gfx::set_error("modraise: at most 32767 ciphertexts per call"); return GPUFHE_EINVAL; }
    KEYS_TRY({
        const uint32_t n = c->n(), comps = 2 * count;
        const std::vector<u64> qp = qp_moduli(*c);
        std::vector<const u64*> in(comps);
        std::vector<u64*> out(comps);
        for (uint32_t i = 0; i < count; ++i) {
            if (!d_c0_in[i] || !d_c1_in[i] || !d_c0_out[i] || !d_c1_out[i])
                throw std::invalid_argument("modraise: null ciphertext pointer");
            in[2 * i] = d_c0_in[i];
            in[2 * i + 1] = d_c1_in[i];
            out[2 * i] = d_c0_out[i];
            out[2 * i + 1] = d_c1_out[i];
        }
        Scratch S(stream);
        u64* x = S.get<u64>((size_t)comps * n);
        const u64* const* din = upload(S, in);
        const unsigned gx = (n + KNT - 1) / KNT;
        k_gather_tower0<<<dim3(gx, comps), KNT, 0, stream>>>(din, x, n);
        ck(cudaGetLastError(), "modraise gather");
        transform(*c, qp, S, x, comps, 1, true);                        // tower 0 -> coefficients
        // every tower -> eval form, its column pass lifting tower 0 (centred
        // mod q0) into the tower's modulus on load
        u64* const* dout = upload(S, out);
        xf::Job* dj = tower_jobs(*c, qp, S, comps, towers, false, dout, nullptr, x, qp[0]);
        ck(xf_launch_ntt_lift(dj, (int)(comps * towers), (int)c->logn(), stream), "modraise transform");
        return GPUFHE_OK;
    })
}

}  // extern "C"
