#include "context.hpp"

#include <cstring>
#include <stdexcept>

#include "devonce.hpp"
#include "hostmath.hpp"
#include "params.h"

namespace gfx {

namespace {
thread_local std::string g_err;

// the reference's root choice (params.cpp:42-48), from this library's params.cu
u64 native_root(uint32_t n, u64 q) { return gpufhe::native_root(n, q); }
}  // namespace

std::string last_error() { return g_err; }
void set_error(const std::string& s) { g_err = s; }

void* Context::dalloc(size_t bytes) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs_.push_back(p);
    table_bytes_ += bytes;
    return p;
}

template <class T>
T* Context::upload(const std::vector<T>& h) {
    T* d = (T*)dalloc(h.size() * sizeof(T));
    cudaError_t e = cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMemcpy: ") + cudaGetErrorString(e));
    return d;
}

namespace {
// The batched key, encryption, ModRaise and embedding entry points take their
// scratch (up to a few hundred MB per call) from the device's default
// stream-ordered pool. With the pool's default release threshold of zero,
// every synchronisation hands that memory back, and the next call maps and
// clears it again; keeping up to 4 GiB in the pool makes repeated calls
// reuse it. Raised only, once per device, never lowered.
void keep_scratch_pool(int device) {
    static gfx::DeviceOnce once;
    once([device] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return;
        uint64_t cur = 0, want = 4ull << 30;
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && cur < want)
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &want);
    });
}
}  // namespace

Context::Context(uint32_t n, const std::vector<u64>& Q, const std::vector<u64>& P, uint32_t alpha,
                 const std::vector<u64>& roots, int device)
    : n_(n), alpha_(alpha), device_(device), Q_(Q), P_(P) {
    if (!hm::is_pow2(n) || n < 512 || n > 65536) throw std::invalid_argument("ring dimension must be 2^9..2^16");
    if (Q.empty() || Q.size() > (size_t)MAXQ) throw std::invalid_argument("Q tower count out of range");
    if (P.empty() || P.size() > (size_t)MAXP) throw std::invalid_argument("P tower count out of range");
    if (alpha == 0 || alpha > Q.size()) throw std::invalid_argument("alpha out of range");
    logn_ = (uint32_t)hm::ilog2(n);
    const uint32_t fullQ = (uint32_t)Q.size(), K = (uint32_t)P.size(), QP = fullQ + K;
    dnum_ = (fullQ + alpha - 1) / alpha;
    if (dnum_ > (uint32_t)MAXD) throw std::invalid_argument("too many digits");
    std::vector<u64> QPm(Q);
    QPm.insert(QPm.end(), P.begin(), P.end());
    for (u64 q : QPm) {
        if (q >= (1ull << 61) || (q & 1) == 0 || (q % (2ull * n)) != 1)
            throw std::invalid_argument("moduli must be odd primes < 2^61 with q = 1 mod 2n");
    }
    if (!roots.empty() && roots.size() != QP) throw std::invalid_argument("roots must list Q then P");
    roots_.resize(QP);
    for (uint32_t i = 0; i < QP; ++i) roots_[i] = roots.empty() ? native_root(n, QPm[i]) : roots[i];
    cudaSetDevice(device);
    keep_scratch_pool(device);

    // per-modulus constants and twiddles
    std::vector<ModC> mc(QP);
    std::vector<Tw> twf((size_t)QP * n), twi((size_t)QP * n), f, iv;
    std::vector<u64> ninv(QP), ninvp(QP);
    for (uint32_t i = 0; i < QP; ++i) {
        const u64 q = QPm[i];
        mc[i] = hm::modc(q);
        hm::twiddles(n, q, roots_[i], f, iv);
        std::memcpy(&twf[(size_t)i * n], f.data(), (size_t)n * sizeof(Tw));
        std::memcpy(&twi[(size_t)i * n], iv.data(), (size_t)n * sizeof(Tw));
        ninv[i] = hm::invmod(n, q);
        ninvp[i] = hm::precon(ninv[i], q);
    }
    ninv_h_ = ninv;
    ninvp_h_ = ninvp;

    // Montgomery form of the keys when the key-switch sums stay below q * 2^64 (Key)
    {
        u64 qmax = 0;
        for (u64 q : QPm) qmax = std::max(qmax, q);
        dc_.mont = ((unsigned __int128)2 * dnum_ * qmax < ((unsigned __int128)1 << 64)) ? 1u : 0u;
    }
    auto rmod = [&](u64 m) { return dc_.mont ? hm::mulmod((1ull << 32) % m, (1ull << 32) % m, m) : (u64)1; };

    // level-independent ModDown constants
    std::vector<u64> pinv(fullQ), pinvp(fullQ), pdn(K), pdnp(K), phatmodq((size_t)K * fullQ);
    for (uint32_t i = 0; i < fullQ; ++i) {
        pinv[i] = hm::invmod(hm::prod_mod(P.data(), K, Q[i]), Q[i]);
        pinvp[i] = hm::precon(pinv[i], Q[i]);
    }
    for (uint32_t j = 0; j < K; ++j) {
        const u64 p = P[j];
        u64 phatinv = hm::invmod(hm::prod_mod(P.data(), K, p, (int)j), p);
        pdn[j] = hm::mulmod(phatinv, hm::invmod(n, p), p);
        pdnp[j] = hm::precon(pdn[j], p);
        for (uint32_t i = 0; i < fullQ; ++i) phatmodq[(size_t)j * fullQ + i] = hm::prod_mod(P.data(), K, Q[i], (int)j);
    }

    // Montgomery conversions when the accumulated sums stay below q * 2^64
    u64 qmaxQ = 0, qmaxP = 0;
    for (u64 q : Q) qmaxQ = std::max(qmaxQ, q);
    for (u64 p : P) qmaxP = std::max(qmaxP, p);
    dc_.mont_up = ((unsigned __int128)alpha * qmaxQ < ((unsigned __int128)1 << 64)) ? 1u : 0u;
    dc_.mont_down = ((unsigned __int128)K * qmaxP < ((unsigned __int128)1 << 64)) ? 1u : 0u;
    auto r64mod = [](u64 m) { return hm::mulmod((1ull << 32) % m, (1ull << 32) % m, m); };

    // per-level constants
    lv_host_.assign(fullQ + 1, Level{});
    std::vector<u64> pool;
    for (uint32_t L = 1; L <= fullQ; ++L) {
        Level& lv = lv_host_[L];
        lv.L = L;
        lv.nparts = (L + alpha - 1) / alpha;
        for (uint32_t p = 0; p < lv.nparts; ++p) {
            lv.part_st[p] = alpha * p;
            lv.part_sp[p] = (L > alpha * p + alpha) ? alpha : L - alpha * p;
        }
        lv.qmp_off = (u32)pool.size();
        const uint32_t QlP = L + K;
        for (uint32_t i = 0; i < L; ++i) {
            const uint32_t p = i / alpha, st = lv.part_st[p], sp = lv.part_sp[p];
            const u64 q = Q[i];
            // (partQ / q_i)^-1 mod q_i  (ks_constants.cpp:79-84), times n^-1
            u64 qhat = hm::prod_mod(Q.data() + st, sp, q, (int)(i - st));
            lv.up_scale[i] = hm::mulmod(hm::invmod(qhat, q), ninv[i], q);
            lv.up_scale_p[i] = hm::precon(lv.up_scale[i], q);
            for (uint32_t j = 0; j < QlP; ++j) {
                const u64 m = j < L ? Q[j] : P[j - L];
                const u64 v = hm::prod_mod(Q.data() + st, sp, m, (int)(i - st));
                pool.push_back(dc_.mont_up ? hm::mulmod(v, r64mod(m), m) : v);
            }
        }
        lv.qmpp_off = lv.qmp_off;
        if (dc_.mont_up) {   // plain copies for the FP64 conversion of P3
            lv.qmpp_off = (u32)pool.size();
            for (uint32_t i = 0; i < L; ++i) {
                const uint32_t p = i / alpha, st = lv.part_st[p], sp = lv.part_sp[p];
                for (uint32_t j = 0; j < QlP; ++j) {
                    const u64 m = j < L ? Q[j] : P[j - L];
                    pool.push_back(hm::prod_mod(Q.data() + st, sp, m, (int)(i - st)));
                }
            }
        }
        if (L >= 2) {
            // s1 = ql^-1 mod q_i and s2 = floor(Ql*u/ql) mod q_i (params.cpp:54-75),
            // which equals q_i - s1 (the derivation is at native_rescale_consts)
            const uint32_t last = L - 1;
            std::vector<u64> s1, s2;
            gpufhe::native_rescale_consts(s1, s2, Q, last);
            for (uint32_t i = 0; i < last; ++i) {
                const u64 qi = Q[i];
                lv.s1[i] = s1[i];
                lv.s2[i] = s2[i];
                lv.s1p[i] = hm::precon(lv.s1[i], qi);
                lv.s1r[i] = hm::mulmod(lv.s1[i], rmod(qi), qi);
                lv.s1rp[i] = hm::precon(lv.s1r[i], qi);
                lv.s2p[i] = hm::precon(lv.s2[i], qi);
                lv.ps1[i] = hm::mulmod(pinv[i], lv.s1[i], qi);
                lv.ps1p[i] = hm::precon(lv.ps1[i], qi);
            }
        }
    }

    dc_.n = n; dc_.logn = logn_; dc_.fullQ = fullQ; dc_.K = K; dc_.alpha = alpha; dc_.dnum = dnum_; dc_.QP = QP;
    dc_.mod = upload(mc);
    dc_.twf = upload(twf);
    dc_.twi = upload(twi);
    {
        std::vector<double> fd((size_t)QP * n, 0.0), id((size_t)QP * n, 0.0);
        for (uint32_t i = 0; i < QP; ++i) {
            if (!fp_tower(mc[i].q)) continue;
            // signed representatives in (-q/2, q/2): the FP64 butterflies'
            // bounds (one normalisation per round) rely on |w| <= (q-1)/2
            const u64 q = mc[i].q;
            auto sgn = [q](u64 w) { return w > q / 2 ? -(double)(q - w) : (double)w; };
            for (uint32_t k = 0; k < n; ++k) {
                fd[(size_t)i * n + k] = sgn(twf[(size_t)i * n + k].w);
                id[(size_t)i * n + k] = sgn(twi[(size_t)i * n + k].w);
            }
        }
        dc_.twfd = upload(fd);
        dc_.twid = upload(id);
    }
    dc_.ninv = upload(ninv);
    dc_.ninvp = upload(ninvp);
    dc_.lvl = upload(lv_host_);
    dc_.pool = upload(pool);
    dc_.pinv = upload(pinv);
    // key storage scale per (digit, row), see Key; n^-1 for U in P7
    {
        const size_t rows = (size_t)dnum_ * QP;
        std::vector<u64> ks(2 * rows);
        for (uint32_t p = 0; p < dnum_; ++p)
            for (uint32_t i = 0; i < QP; ++i) {
                const u64 q = QPm[i];
                u64 v = rmod(q);
                if (i < fullQ) v = hm::mulmod(pinv[i], i / alpha == p ? v : 1, q);
                ks[(size_t)p * QP + i] = v;
                ks[rows + (size_t)p * QP + i] = hm::precon(v, q);
            }
        d_key_scale_ = upload(ks);
        std::vector<u64> nu(fullQ), nup(fullQ);
        for (uint32_t i = 0; i < fullQ; ++i) {
            nu[i] = hm::mulmod(ninv[i], rmod(Q[i]), Q[i]);
            nup[i] = hm::precon(nu[i], Q[i]);
        }
        dc_.ninvu = upload(nu);
        dc_.ninvup = upload(nup);
    }
    dc_.pinvp = upload(pinvp);
    dc_.pdn = upload(pdn);
    dc_.pdnp = upload(pdnp);
    dc_.phatmodq = upload(phatmodq);
    dc_.err = const_cast<u32*>(upload(std::vector<u32>(4, 0u)));
}

Context::~Context() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device_);
    for (auto& kv : keys_) {
        if (kv.second.dev.av) { cudaFree(kv.second.dev.av); cudaFree(kv.second.dev.bv); }
        if (kv.second.host_av) { cudaFreeHost(kv.second.host_av); cudaFreeHost(kv.second.host_bv); }
    }
    for (void* p : allocs_) cudaFree(p);
    cudaSetDevice(prev);
}

namespace {
// key[p][r][*] = key * scale[r] mod q_r (Shoup, canonical), every digit p.
__global__ void k_scale_key_rows(u64* __restrict__ key, const ModC* __restrict__ mod, const u64* __restrict__ sc,
                                 uint32_t QP, uint32_t rows, uint32_t n) {
    const uint32_t row = blockIdx.y;               // p * QP + r
    const uint32_t r = row % QP;
    const u64 q = mod[r].q, c = sc[row], cp = sc[rows + row];
    u64* x = key + (size_t)row * n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = shoup(x[i], c, cp, q);
}
}  // namespace

cudaError_t scale_key_rows(u64* key, const ModC* mod, const u64* scale, uint32_t dnum, uint32_t QP, uint32_t n) {
    const dim3 g((n + 255) / 256 < 64 ? (n + 255) / 256 : 64, dnum * QP);
    k_scale_key_rows<<<g, 256>>>(key, mod, scale, QP, dnum * QP, n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e;
}

void Context::set_key(uint64_t id, const u64* av, const u64* bv, bool device_src) {
    std::lock_guard<std::mutex> g(mu_);
    const size_t words = (size_t)dnum_ * (fullQ() + K()) * n_;
    auto it0 = keys_.find(id);
    if (it0 != keys_.end() && it0->second.pins) throw std::invalid_argument("set_key: key is in use by a plan");
    if (key_budget_) evict_for(one_key_bytes(), id);
    Key k;
    auto up = [&](const u64* h) {
        u64* d = nullptr;
        cudaError_t e = cudaMalloc(&d, words * 8);
        if (e != cudaSuccess) throw std::runtime_error(std::string("key cudaMalloc: ") + cudaGetErrorString(e));
        e = cudaMemcpy(d, h, words * 8, device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { cudaFree(d); throw std::runtime_error("key upload failed"); }
        return d;
    };
    k.av = up(av);
    k.bv = up(bv);
    for (u64* d : {k.av, k.bv}) {
        const cudaError_t e = scale_key_rows(d, dc_.mod, d_key_scale_, dnum_, fullQ() + K(), n_);
        if (e != cudaSuccess) {
            cudaFree(k.av);
            cudaFree(k.bv);
            throw std::runtime_error(std::string("key scaling: ") + cudaGetErrorString(e));
        }
    }
    auto it = keys_.find(id);
    if (it != keys_.end()) {
        KeySlot& old = it->second;
        if (old.dev.av) { cudaFree(old.dev.av); cudaFree(old.dev.bv); key_dev_bytes_ -= one_key_bytes(); }
        if (old.host_av) { cudaFreeHost(old.host_av); cudaFreeHost(old.host_bv); }
        keys_.erase(it);
    }
    KeySlot& slot = keys_[id];
    slot.dev = k;
    slot.last_use = ++key_tick_;
    key_dev_bytes_ += one_key_bytes();
    if (key_budget_) host_copy(slot);
}

void Context::host_copy(KeySlot& k) const {
    if (k.host_av || !k.dev.av) return;
    const size_t bytes = one_key_bytes() / 2;
    if (cudaMallocHost(&k.host_av, bytes) != cudaSuccess || cudaMallocHost(&k.host_bv, bytes) != cudaSuccess) {
        if (k.host_av) cudaFreeHost(k.host_av);
        k.host_av = k.host_bv = nullptr;
        throw std::runtime_error("key host copy: pinned allocation failed");
    }
    if (cudaMemcpy(k.host_av, k.dev.av, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(k.host_bv, k.dev.bv, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("key host copy failed");
}

void Context::evict_for(size_t need, uint64_t keep) const {
    if (!key_budget_) return;
    while (key_dev_bytes_ + need > key_budget_) {
        KeySlot* victim = nullptr;
        for (auto& kv : keys_) {
            KeySlot& k = kv.second;
            if (kv.first == keep || !k.dev.av || k.pins) continue;
            if (!victim || k.last_use < victim->last_use) victim = &k;
        }
        if (!victim) return;                       // everything resident is pinned
        host_copy(*victim);
        cudaFree(victim->dev.av);
        cudaFree(victim->dev.bv);
        victim->dev = Key{};
        key_dev_bytes_ -= one_key_bytes();
        ++key_evictions_;
    }
}

void Context::set_key_budget(size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    if (bytes && bytes < one_key_bytes()) throw std::invalid_argument("key budget below one key");
    key_budget_ = bytes;
    if (!bytes) return;
    for (auto& kv : keys_) host_copy(kv.second);
    evict_for(0, ~0ull);
}

const Key* Context::acquire(uint64_t id) const {
    std::lock_guard<std::mutex> g(mu_);
    auto it = keys_.find(id);
    if (it == keys_.end()) return nullptr;
    KeySlot& k = it->second;
    if (!k.dev.av) {
        evict_for(one_key_bytes(), id);
        if (key_budget_ && key_dev_bytes_ + one_key_bytes() > key_budget_)
            throw std::length_error("key budget too small for the keys one batch needs at once");
        const size_t bytes = one_key_bytes() / 2;
        Key d;
        if (cudaMalloc(&d.av, bytes) != cudaSuccess || cudaMalloc(&d.bv, bytes) != cudaSuccess) {
            if (d.av) cudaFree(d.av);
            throw std::length_error("key upload: cudaMalloc failed");
        }
        if (cudaMemcpy(d.av, k.host_av, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d.bv, k.host_bv, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(d.av);
            cudaFree(d.bv);
            throw std::runtime_error("key upload failed");
        }
        k.dev = d;
        key_dev_bytes_ += one_key_bytes();
        ++key_uploads_;
    }
    ++k.pins;
    k.last_use = ++key_tick_;
    return &k.dev;
}

void Context::release(uint64_t id) const {
    std::lock_guard<std::mutex> g(mu_);
    auto it = keys_.find(id);
    if (it != keys_.end() && it->second.pins) --it->second.pins;
}

Context::KeyStats Context::key_stats() const {
    std::lock_guard<std::mutex> g(mu_);
    KeyStats s{};
    s.known = keys_.size();
    for (auto& kv : keys_) s.resident += kv.second.dev.av != nullptr;
    s.resident_bytes = key_dev_bytes_;
    s.uploads = key_uploads_;
    s.evictions = key_evictions_;
    s.budget = key_budget_;
    return s;
}

bool Context::tuned_choice(uint64_t key, int& choice) const {
    std::lock_guard<std::mutex> g(mu_);
    auto it = tune_.find(key);
    if (it == tune_.end()) return false;
    choice = it->second;
    return true;
}

void Context::set_tuned_choice(uint64_t key, int choice) const {
    std::lock_guard<std::mutex> g(mu_);
    tune_[key] = choice;
}

const Key* Context::key(uint64_t id) const {
    std::lock_guard<std::mutex> g(mu_);
    auto it = keys_.find(id);
    return it == keys_.end() ? nullptr : &it->second.dev;
}

size_t Context::key_bytes() const {
    std::lock_guard<std::mutex> g(mu_);
    return key_dev_bytes_;
}

}  // namespace gfx
