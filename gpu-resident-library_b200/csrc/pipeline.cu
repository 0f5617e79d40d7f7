// Host side of the batched pipeline: builds per-kernel job tables for a batch
// of operations (uneven levels, mixed modes) and launches the seven phase
// kernels on a stream. A built plan only launches kernels, so it can be
// captured in a CUDA graph and replayed.
#include "pipeline.hpp"

#include <algorithm>
#include <cstring>
#include <stdexcept>

namespace pl {

namespace {

template <int LOGN>
struct Launcher {
    static void attrs() {
        using G = ntt::Geo<LOGN>;
        static bool done = false;
        if (done) return;
        cudaFuncSetAttribute(k1_inv_row<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
        cudaFuncSetAttribute(k2_inv_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
        cudaFuncSetAttribute(k3_modup_fwd_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
        cudaFuncSetAttribute(k4_mac_fwd_row<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, PG<LOGN>::MAC_SMEM);
        cudaFuncSetAttribute(k5_moddown_inv_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
        cudaFuncSetAttribute(k6_moddown_fwd_col<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
        cudaFuncSetAttribute(k7_final_fwd_row<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
        done = true;
    }
    static void launch(const Plan& p, cudaStream_t s, unsigned mask) {
        using G = ntt::Geo<LOGN>;
        using PGL = PG<LOGN>;
        attrs();
        const DevCtx& D = p.dc;
        const PairDesc* pd = p.d_pairs;
        auto J = [&](int k) { return p.d_jobs + p.job_off[k]; };
        auto cnt = [&](int k) { return p.job_cnt[k]; };
        if ((mask >> 0 & 1) && cnt(0)) k1_inv_row<LOGN><<<cnt(0) * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(D, pd, J(0));
        if ((mask >> 1 & 1) && cnt(1)) k2_inv_col<LOGN><<<cnt(1) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(1));
        if ((mask >> 2 & 1) && cnt(2)) k3_modup_fwd_col<LOGN><<<cnt(2) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(2));
        if ((mask >> 3 & 1) && cnt(3)) k4_mac_fwd_row<LOGN><<<cnt(3) * PGL::MAC_TILES, PGL::MAC_THREADS, PGL::MAC_SMEM, s>>>(D, pd, J(3));
        if ((mask >> 4 & 1) && cnt(4)) k5_moddown_inv_col<LOGN><<<cnt(4) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(4));
        if ((mask >> 5 & 1) && cnt(5)) k6_moddown_fwd_col<LOGN><<<cnt(5) * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(D, pd, J(5));
        if ((mask >> 6 & 1) && cnt(6)) k7_final_fwd_row<LOGN><<<cnt(6) * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(D, pd, J(6));
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
    if (op.mode > RESCALE) throw std::invalid_argument("unknown mode");
    const int nin = op.mode == EMR ? 4 : op.mode == ROT ? 2 : 1;
    for (int k = 0; k < nin; ++k) if (!op.in[k]) throw std::invalid_argument("null input");
    if (!op.out[0] || (op.mode != RESCALE && !op.out[1])) throw std::invalid_argument("null output");
    if (op.mode == ROT && (op.galois % 2 == 0 || op.galois >= 2ull * c.n())) throw std::invalid_argument("bad Galois element");
}

Plan::~Plan() {
    if (d_pairs) cudaFree(d_pairs);
    if (d_jobs) cudaFree(d_jobs);
    if (own_ws && ws) cudaFree(ws);
}

std::unique_ptr<Plan> build_plan(const gfx::Context& c, const std::vector<Op>& ops, u64* ws, size_t ws_words) {
    if (!supported_logn((int)c.logn())) throw std::invalid_argument("pipeline supports n = 2^11 .. 2^16");
    auto plan = std::make_unique<Plan>();
    plan->dc = c.dev();
    plan->logn = c.logn();
    const uint32_t n = c.n(), K = c.K();
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
    std::vector<uint2> jobs[7];
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
            for (uint32_t i = 0; i + 1 < L; ++i) { jobs[5].push_back({pu, i}); jobs[6].push_back({pu, i}); }
            continue;
        }
        for (uint32_t i = 0; i < L; ++i) { jobs[0].push_back({pu, i}); jobs[1].push_back({pu, i}); }
        for (uint32_t p = 0; p < nparts; ++p) {
            const uint32_t st = c.alpha() * p, sp = std::min(c.alpha(), L - st);
            for (uint32_t i = 0; i < QlP; ++i)
                if (i < st || i >= st + sp) jobs[2].push_back({pu, p * QlP + i});
        }
        for (uint32_t i = 0; i < QlP; ++i) jobs[3].push_back({pu, i});
        const bool emr = op.mode == EMR;
        for (uint32_t cc = 0; cc < 2; ++cc)
            for (uint32_t t = emr ? 0 : 1; t <= K; ++t) jobs[4].push_back({pu, cc * (K + 1) + t});
        const uint32_t outL = emr ? L - 1 : L;
        for (uint32_t cc = 0; cc < 2; ++cc)
            for (uint32_t i = 0; i < outL; ++i) { jobs[5].push_back({pu, cc * L + i}); jobs[6].push_back({pu, cc * L + i}); }
    }
    (void)n;
    size_t total = 0;
    for (int k = 0; k < 7; ++k) { plan->job_off[k] = total; plan->job_cnt[k] = (uint32_t)jobs[k].size(); total += jobs[k].size(); }
    std::vector<uint2> all;
    all.reserve(total);
    for (int k = 0; k < 7; ++k) all.insert(all.end(), jobs[k].begin(), jobs[k].end());
    if (cudaMalloc(&plan->d_pairs, std::max<size_t>(pairs.size(), 1) * sizeof(PairDesc)) != cudaSuccess ||
        cudaMalloc(&plan->d_jobs, std::max<size_t>(total, 1) * sizeof(uint2)) != cudaSuccess)
        throw std::runtime_error("plan allocation failed");
    cudaMemcpy(plan->d_pairs, pairs.data(), pairs.size() * sizeof(PairDesc), cudaMemcpyHostToDevice);
    cudaMemcpy(plan->d_jobs, all.data(), total * sizeof(uint2), cudaMemcpyHostToDevice);
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
