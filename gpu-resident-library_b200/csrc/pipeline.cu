// Host side of the batched pipeline: builds per-kernel job tables for a batch
// of operations (uneven levels, mixed modes) and launches the seven phase
// kernels on a stream. A built plan only launches kernels, so it can be
// captured in a CUDA graph and replayed.
#include "pipeline.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <stdexcept>

namespace pl {

namespace {

template <int LOGN>
struct Launcher {
    static void attrs(uint32_t dnum) {
        using G = ntt::Geo<LOGN>;
        static bool done = false;
        static uint32_t mac_dnum = 0;
        if (!done) {
            cudaFuncSetAttribute(p1_inv_row<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
            cudaFuncSetAttribute(p2_inv_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
            cudaFuncSetAttribute(p3_modup_fwd_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
            cudaFuncSetAttribute(p4_modup_fwd_row<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
            cudaFuncSetAttribute(p6_moddown_inv_row<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
            cudaFuncSetAttribute(p7_moddown_inv_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
            cudaFuncSetAttribute(p8_moddown_fwd_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
            cudaFuncSetAttribute(p9_final_fwd_row<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
            done = true;
        }
        if (dnum > mac_dnum) {
            cudaFuncSetAttribute(p5_mac<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, mac_smem(dnum));
            mac_dnum = dnum;
        }
    }
    static void launch(const Plan& p, cudaStream_t s, unsigned mask) {
        using G = ntt::Geo<LOGN>;
        constexpr int MAC_TILES = (1 << LOGN) / MAC_TILE;
        attrs(p.dc.dnum);
        const DevCtx& D = p.dc;
        const PairDesc* pd = p.d_pairs;
        auto J = [&](int k) { return p.d_jobs + p.job_off[k]; };
        auto cnt = [&](int k) { return p.job_cnt[k]; };
        auto on = [&](int k) { return (mask >> k & 1) && cnt(k); };
        if (on(0)) p1_inv_row<LOGN><<<cnt(0) * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(D, pd, J(0));
        if (on(1)) p2_inv_col<LOGN><<<cnt(1) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(1));
        if (on(2)) p3_modup_fwd_col<LOGN><<<cnt(2) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(2));
        if (on(3)) p4_modup_fwd_row<LOGN><<<cnt(3) * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(D, pd, J(3));
        if (on(4)) p5_mac<LOGN><<<cnt(4) * MAC_TILES, MAC_NT, mac_smem(D.dnum), s>>>(D, pd, p.d_mac_jobs, p.d_plist);
        if (on(5)) p6_moddown_inv_row<LOGN><<<cnt(5) * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(D, pd, J(5));
        if (on(6)) p7_moddown_inv_col<LOGN><<<cnt(6) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(6));
        if (on(7)) p8_moddown_fwd_col<LOGN><<<cnt(7) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(7));
        if (on(8)) p9_final_fwd_row<LOGN><<<cnt(8) * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(D, pd, J(8));
    }
};

}  // namespace

bool supported_logn(int logn) { return logn >= 11 && logn <= 16; }

int input_count(uint32_t mode) { return mode == EMR ? 4 : mode == ROT ? 2 : 1; }
uint32_t output_towers(const Op& op) { return (op.mode == EMR || op.mode == RESCALE) ? op.L - 1 : op.L; }

size_t op_workspace_words(const gfx::Context& c, uint32_t L) {
    return (size_t)ws_layout(L, c.K(), c.alpha()).total * c.n();
}

void validate(const gfx::Context& c, const Op& op) {
    if (op.L < 1 || op.L > c.fullQ()) throw std::invalid_argument("level out of range");
    if ((op.mode == EMR || op.mode == RESCALE) && op.L < 2) throw std::invalid_argument("rescale needs L >= 2");
    if (c.alpha() > (uint32_t)MAXA) throw std::invalid_argument("digit width above the fused limit");
    if (c.dnum() > (uint32_t)MAC_MAX_DNUM) throw std::invalid_argument("too many digits for the key-stationary MAC");
    if (op.mode > RESCALE) throw std::invalid_argument("unknown mode");
    const int nin = op.mode == EMR ? 4 : op.mode == ROT ? 2 : 1;
    for (int k = 0; k < nin; ++k) if (!op.in[k]) throw std::invalid_argument("null input");
    if (!op.out[0] || (op.mode != RESCALE && !op.out[1])) throw std::invalid_argument("null output");
    if (op.mode == ROT && (op.galois % 2 == 0 || op.galois >= 2ull * c.n())) throw std::invalid_argument("bad Galois element");
}

Plan::~Plan() {
    if (d_pairs) cudaFree(d_pairs);
    if (d_jobs) cudaFree(d_jobs);
    if (d_mac_jobs) cudaFree(d_mac_jobs);
    if (d_plist) cudaFree(d_plist);
    if (own_ws && ws) cudaFree(ws);
}

std::unique_ptr<Plan> build_plan(const gfx::Context& c, const std::vector<Op>& ops, u64* ws, size_t ws_words) {
    if (!supported_logn((int)c.logn())) throw std::invalid_argument("pipeline supports n = 2^11 .. 2^16");
    auto plan = std::make_unique<Plan>();
    plan->dc = c.dev();
    plan->logn = c.logn();
    const uint32_t K = c.K();
    size_t need = 0;
    for (const Op& op : ops) { validate(c, op); need += op_workspace_words(c, op.L); }
    if (!ws) {
        if (cudaMalloc(&plan->ws, std::max<size_t>(need, 1) * 8) != cudaSuccess)
            throw std::runtime_error("workspace allocation failed");
        plan->own_ws = true;
        ws = plan->ws;
    } else if (ws_words < need) {
        throw std::length_error("workspace too small");
    }
    plan->ws_words = need;
    std::vector<PairDesc> pairs(ops.size());
    std::vector<uint2> jobs[NPHASE];
    // P5: pairs per (key, QP row), streamed in groups of MAC_GROUP
    std::map<std::pair<uint64_t, uint32_t>, std::vector<uint32_t>> rows;
    size_t off = 0;
    for (size_t pi = 0; pi < ops.size(); ++pi) {
        const Op& op = ops[pi];
        PairDesc& P = pairs[pi];
        std::memset(&P, 0, sizeof(P));
        P.L = op.L;
        P.mode = op.mode;
        P.galois = op.galois;
        for (int k = 0; k < 4; ++k) P.in[k] = op.in[k];
        P.out[0] = op.out[0];
        P.out[1] = op.out[1];
        P.ws = ws + off;
        off += op_workspace_words(c, op.L);
        if (op.mode != RESCALE) {
            const gfx::Key* key = c.key(op.key_id);
            if (!key) throw std::invalid_argument("missing eval key");
            P.kav = key->av;
            P.kbv = key->bv;
        }
        const uint32_t L = op.L, QlP = L + K, pu = (uint32_t)pi;
        const uint32_t nparts = (L + c.alpha() - 1) / c.alpha();
        if (op.mode == RESCALE) {
            jobs[0].push_back({pu, L - 1});
            jobs[1].push_back({pu, L - 1});
            for (uint32_t i = 0; i + 1 < L; ++i) { jobs[7].push_back({pu, i}); jobs[8].push_back({pu, i}); }
            continue;
        }
        for (uint32_t i = 0; i < L; ++i) { jobs[0].push_back({pu, i}); jobs[1].push_back({pu, i}); }
        for (uint32_t p = 0; p < nparts; ++p) {
            const uint32_t st = c.alpha() * p, sp = std::min(c.alpha(), L - st);
            for (uint32_t i = 0; i < QlP; ++i)
                if (i < st || i >= st + sp) { jobs[2].push_back({pu, p * QlP + i}); jobs[3].push_back({pu, p * QlP + i}); }
        }
        for (uint32_t i = 0; i < QlP; ++i) rows[{op.key_id, qp_of(i, L, c.fullQ())}].push_back(pu);
        const bool emr = op.mode == EMR;
        for (uint32_t cc = 0; cc < 2; ++cc) {
            for (uint32_t t = emr ? 0 : 1; t <= K; ++t) jobs[5].push_back({pu, cc * (K + 1) + t});
            jobs[6].push_back({pu, cc});
        }
        const uint32_t outL = emr ? L - 1 : L;
        for (uint32_t cc = 0; cc < 2; ++cc)
            for (uint32_t i = 0; i < outL; ++i) { jobs[7].push_back({pu, cc * L + i}); jobs[8].push_back({pu, cc * L + i}); }
    }
    std::vector<uint4> mac_jobs;
    std::vector<uint32_t> plist;
    for (auto& kv : rows) {
        const auto& v = kv.second;
        for (size_t g = 0; g < v.size(); g += MAC_GROUP) {
            const uint32_t cnt = (uint32_t)std::min<size_t>(MAC_GROUP, v.size() - g);
            mac_jobs.push_back({kv.first.second, (uint32_t)plist.size(), cnt, 0});
            plist.insert(plist.end(), v.begin() + g, v.begin() + g + cnt);
        }
    }
    size_t total = 0;
    for (int k = 0; k < NPHASE; ++k) {
        plan->job_off[k] = total;
        plan->job_cnt[k] = (uint32_t)jobs[k].size();
        total += jobs[k].size();
    }
    plan->job_cnt[4] = (uint32_t)mac_jobs.size();
    std::vector<uint2> all;
    all.reserve(total);
    for (int k = 0; k < NPHASE; ++k) all.insert(all.end(), jobs[k].begin(), jobs[k].end());
    if (cudaMalloc(&plan->d_pairs, std::max<size_t>(pairs.size(), 1) * sizeof(PairDesc)) != cudaSuccess ||
        cudaMalloc(&plan->d_jobs, std::max<size_t>(total, 1) * sizeof(uint2)) != cudaSuccess ||
        cudaMalloc(&plan->d_mac_jobs, std::max<size_t>(mac_jobs.size(), 1) * sizeof(uint4)) != cudaSuccess ||
        cudaMalloc(&plan->d_plist, std::max<size_t>(plist.size(), 1) * sizeof(uint32_t)) != cudaSuccess)
        throw std::runtime_error("plan allocation failed");
    cudaMemcpy(plan->d_pairs, pairs.data(), pairs.size() * sizeof(PairDesc), cudaMemcpyHostToDevice);
    cudaMemcpy(plan->d_jobs, all.data(), total * sizeof(uint2), cudaMemcpyHostToDevice);
    cudaMemcpy(plan->d_mac_jobs, mac_jobs.data(), mac_jobs.size() * sizeof(uint4), cudaMemcpyHostToDevice);
    cudaMemcpy(plan->d_plist, plist.data(), plist.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    plan->nops = (uint32_t)ops.size();
    plan->ops = ops;
    plan->pairs_host = pairs;
    return plan;
}

namespace {
__global__ void k_set_pair(PairDesc* dst, PairDesc v) { *dst = v; }
}  // namespace

void rebind(Plan& p, uint32_t idx, const Op& op, const gfx::Context& c, cudaStream_t s) {
    if (idx >= p.pairs_host.size()) throw std::invalid_argument("rebind: index");
    validate(c, op);
    const Op& old = p.ops[idx];
    const bool same_shape = old.L == op.L && (old.mode == op.mode ||
                            ((old.mode == KS || old.mode == ROT) && (op.mode == KS || op.mode == ROT)));
    if (!same_shape) throw std::invalid_argument("rebind: level or job shape differs");
    if (op.key_id != old.key_id && p.ops.size() > 1)
        throw std::invalid_argument("rebind: changing the key of one operation of a shared batch");
    PairDesc P = p.pairs_host[idx];
    P.mode = op.mode;
    P.galois = op.galois;
    for (int k = 0; k < 4; ++k) P.in[k] = op.in[k];
    P.out[0] = op.out[0];
    P.out[1] = op.out[1];
    if (op.mode != RESCALE) {
        const gfx::Key* key = c.key(op.key_id);
        if (!key) throw std::invalid_argument("missing eval key");
        P.kav = key->av;
        P.kbv = key->bv;
    }
    p.pairs_host[idx] = P;
    p.ops[idx] = op;
    k_set_pair<<<1, 1, 0, s>>>(p.d_pairs + idx, P);
}

cudaError_t launch(const Plan& p, cudaStream_t s, unsigned mask) {
    switch (p.logn) {
        case 11: Launcher<11>::launch(p, s, mask); break;
        case 12: Launcher<12>::launch(p, s, mask); break;
        case 13: Launcher<13>::launch(p, s, mask); break;
        case 14: Launcher<14>::launch(p, s, mask); break;
        case 15: Launcher<15>::launch(p, s, mask); break;
        case 16: Launcher<16>::launch(p, s, mask); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace pl
