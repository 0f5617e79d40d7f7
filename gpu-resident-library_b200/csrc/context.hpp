// Resident CKKS context: the modulus chain Q (fullQ towers) and special
// primes P (K towers) with digit width alpha, their twiddle tables, every
// per-level keyswitch / ModDown / rescale constant, and the resident eval keys.
// Everything a kernel needs is reachable from the POD `DevCtx`, passed by
// value to each launch.
#pragma once
#include <atomic>
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "gf.cuh"

namespace gfx {

constexpr int MAXQ = 48;     // Q towers
constexpr int MAXP = 16;     // special primes
constexpr int MAXQP = MAXQ + MAXP;
constexpr int MAXD = 48;     // digits

// Constants for one level L (L Q towers, dropping tower L-1 on rescale).
struct Level {
    u32 L, nparts;
    u32 part_st[MAXD], part_sp[MAXD];
    u32 qmp_off;                       // pool offset of qhatmodp [L][L+K] (times 2^64 with mont_up)
    u32 qmpp_off;                      // the same entries without the 2^64 factor (FP64 conversions)
    u64 up_scale[MAXQ], up_scale_p[MAXQ];    // n^-1 * QHatInv_i (i's digit) mod q_i
    // rescale of tower L-1 onto i < L-1
    u64 s1[MAXQ], s1p[MAXQ];           // q_l^-1 mod q_i
    u64 s1r[MAXQ], s1rp[MAXQ];         // s1 * 2^64 mod q_i with DevCtx mont, else s1 (P5 EvalMult epilogue)
    u64 s2[MAXQ], s2p[MAXQ];           // floor(Ql*(Ql^-1 mod q_l)/q_l) mod q_i
    u64 ps1[MAXQ], ps1p[MAXQ];         // P^-1 * s1 mod q_i
};

struct DevCtx {
    u32 n, logn, fullQ, K, alpha, dnum, QP;
    u32 mont;                 // keys are stored times 2^64 (Montgomery form), see Context::set_key
    u32 mont_up;              // ModUp pool entries carry 2^64: P3 reduces with Montgomery (alpha * max q < 2^64)
    u32 mont_down;            // P7 / P8 conversions reduce with Montgomery (K * max p < 2^64)
    const ModC* mod;          // [QP]: Q towers then P towers
    const Tw* twf;            // [QP][n]
    const Tw* twi;            // [QP][n]
    const double* twfd;       // [QP][n] forward twiddles as signed doubles in (-q/2, q/2) (towers with q < 2^50; else 0)
    const double* twid;       // [QP][n] inverse twiddles, same form
    const u64* ninv;          // [QP] n^-1 mod q
    const u64* ninvp;
    const u64* ninvu;         // [fullQ] n^-1 * 2^64 mod q with mont, else n^-1 (P7 scaling of U)
    const u64* ninvup;
    const Level* lvl;         // [fullQ + 1]
    const u64* pool;          // qhatmodp pools
    const u64* pinv;          // [fullQ] P^-1 mod q_i
    const u64* pinvp;
    const u64* pdn;           // [K] n^-1 * (P/p_j)^-1 mod p_j
    const u64* pdnp;
    const u64* phatmodq;      // [K][fullQ] (P/p_j) mod q_i
    u32* err;                 // device status word: kernels with bounded waits OR in a code when one expires
};

// A resident eval key: av/bv over full QP for every digit, eval form, layout
// [dnum][fullQ+K][n]. Stored scaled, canonical, with R = 2^64 when the
// key-switch accumulator bound 2*dnum*max(q) < 2^64 allows Montgomery
// reduction (DevCtx mont = 1), else R = 1:
//   P row j (every digit):                 key * R mod p_j
//   Q row i, digit i / alpha (own digit):  key * P^-1 * R mod q_i
//   Q row i, other digits:                 key * P^-1 mod q_i
// With mont, the own-digit source enters the inner product as src * R^-1
// (the EvalMult tensor products are Montgomery products), so every Q-row sum
// is res * P^-1 exactly and every P-row sum is res * R.
struct Key {
    u64* av = nullptr;
    u64* bv = nullptr;
};

class Context {
public:
    Context(uint32_t n, const std::vector<u64>& Q, const std::vector<u64>& P, uint32_t alpha,
            const std::vector<u64>& roots /* empty: native roots */, int device);
    ~Context();
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;

    const DevCtx& dev() const { return dc_; }
    uint32_t n() const { return n_; }
    uint32_t logn() const { return logn_; }
    uint32_t fullQ() const { return (uint32_t)Q_.size(); }
    uint32_t K() const { return (uint32_t)P_.size(); }
    uint32_t alpha() const { return alpha_; }
    uint32_t dnum() const { return dnum_; }
    const std::vector<u64>& Q() const { return Q_; }
    const std::vector<u64>& P() const { return P_; }
    const std::vector<u64>& roots() const { return roots_; }
    // n^-1 mod each QP modulus and its Shoup precomputation (host copies)
    const std::vector<u64>& ninv_host() const { return ninv_h_; }
    const std::vector<u64>& ninvp_host() const { return ninvp_h_; }
    const Level& level_host(uint32_t L) const { return lv_host_[L]; }
    int device() const { return device_; }

    // Upload a key ([dnum][fullQ+K][n] canonical; host arrays, or device
    // arrays with device_src). id 0 = relinearisation; rotation keys are
    // stored under their Galois element.
    void set_key(uint64_t id, const u64* av, const u64* bv, bool device_src = false);
    // The key stored under `id` (its device pointers are null while it is
    // evicted), or nullptr for an unknown id.
    const Key* key(uint64_t id) const;
    size_t key_bytes() const;              // device bytes of the resident keys
    size_t resident_bytes() const { return table_bytes_ + key_bytes(); }

    // Key residency. With a budget (bytes, 0 = unlimited) every key keeps a
    // pinned host copy of its stored form and at most `budget` bytes of keys
    // stay on the device; acquire() makes a key resident (uploading it and
    // evicting least recently used unpinned keys) and pins it until release().
    // A batch that needs more pinned keys than the budget holds throws
    // std::length_error.
    void set_key_budget(size_t bytes);
    const Key* acquire(uint64_t id) const;
    void release(uint64_t id) const;
    struct KeyStats { uint64_t known, resident, resident_bytes, uploads, evictions, budget; };
    KeyStats key_stats() const;

    // Autotuner cache: launch-schedule choice per batch shape key.
    bool tuned_choice(uint64_t key, int& choice) const;
    void set_tuned_choice(uint64_t key, int choice) const;

    // Lifetime. Plans (and through them linear-transform plans) and servers
    // hold the context they use; retire() deletes it at once when nothing
    // holds it, else the last holder's drop() does, so a context destroyed
    // before its plans stays valid until they are gone. Owners end a context
    // with retire(), never with delete.
    void hold() const { life_.fetch_add(2); }
    static void drop(const Context* c) {
        if (c->life_.fetch_sub(2) - 2 == 1) delete const_cast<Context*>(c);
    }
    static void retire(Context* c) {
        if (c && c->life_.fetch_or(1) == 0) delete c;
    }

private:
    mutable std::atomic<uint32_t> life_{0};   // 2 * holders + retired bit
    uint32_t n_, logn_, alpha_, dnum_;
    int device_;
    std::vector<u64> Q_, P_, roots_;
    std::vector<u64> ninv_h_, ninvp_h_;
    std::vector<Level> lv_host_;
    u64* d_key_scale_ = nullptr;                 // [2][dnum * QP] row scale and Shoup precon (Key)
    DevCtx dc_{};
    std::vector<void*> allocs_;
    size_t table_bytes_ = 0;
    struct KeySlot {
        Key dev;                       // device copy (null while evicted)
        u64* host_av = nullptr;        // pinned host copy of the stored form (with a budget)
        u64* host_bv = nullptr;
        uint64_t last_use = 0;
        uint32_t pins = 0;
    };
    mutable std::map<uint64_t, KeySlot> keys_;
    size_t key_budget_ = 0;
    mutable size_t key_dev_bytes_ = 0;
    mutable uint64_t key_tick_ = 0, key_uploads_ = 0, key_evictions_ = 0;
    size_t one_key_bytes() const { return 2 * (size_t)dnum_ * (fullQ() + K()) * n_ * 8; }
    void host_copy(KeySlot& k) const;              // device -> pinned host (caller holds mu_)
    void evict_for(size_t need, uint64_t keep) const;   // caller holds mu_
    mutable std::map<uint64_t, int> tune_;
    mutable std::mutex mu_;
    void* dalloc(size_t bytes);
    template <class T>
    T* upload(const std::vector<T>& h);
};

// Applies the key storage scale of every row (Key) in place on the device.
cudaError_t scale_key_rows(u64* key, const ModC* mod, const u64* scale, uint32_t dnum, uint32_t QP, uint32_t n);

std::string last_error();
void set_error(const std::string& s);

}  // namespace gfx
