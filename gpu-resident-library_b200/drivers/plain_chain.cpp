// Plain per-chain resident EvalMult+Rescale: the reference's benchmark driver
// (bench/bench_evalmult_resident.cpp:56-109) with OpenFHE taken out, linked
// against this library's drop-in API. Each chain owns its buffers and one
// CUDA graph of LaunchTensor -> keyswitch_resident -> LaunchCombine ->
// rescale_resident_raw (c0) -> rescale_resident_raw (c1), exactly the
// reference's sequence. Keys come from keygen_host / evalkeygen_host and the
// constants from compute_keyswitch_constants, as in the reference driver;
// chains may sit at different levels, with one DeviceKSContext per level
// sharing the full-QP relinearisation key (the reference's key-row offset,
// keyswitch_resident.cpp:91-96).
//
// usage: plain_chain <n> <fullQ> <K> <alpha> <reps> <dump-file or -> <L_1> ... <L_c>
// Prints one JSON line with the device time of all chains run one after the
// other on one stream, and spread over 16 streams. With a dump file, writes
// for each chain its four inputs and two outputs ([L][n] and [L-1][n] words).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "keygen.h"
#include "keyswitch.h"
#include "keyswitch_resident.h"
#include "params.h"
#include "tensor.h"

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        std::exit(2);
    }
}

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((unsigned __int128)a * b) % q); }

struct Chain {
    uint32_t L;
    uint64_t *c0a, *c1a, *c0b, *c1b, *t0, *t1, *t2, *ba0, *ba1, *r0, *r1, *scr, *drp;
    gpufhe::DeviceKSWork W;
    cudaGraphExec_t exec;
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: plain_chain n fullQ K alpha reps dump L_1 ... L_c\n");
        return 1;
    }
    const uint32_t n = std::atoi(argv[1]), fullQ = std::atoi(argv[2]), K = std::atoi(argv[3]),
                   alpha = std::atoi(argv[4]), reps = std::atoi(argv[5]);
    const std::string dump = argv[6];
    std::vector<uint32_t> levels;
    for (int i = 7; i < argc; ++i) levels.push_back(std::atoi(argv[i]));

    // chain Q = one 60-bit + (fullQ-1) 50-bit primes, P = K 60-bit primes
    std::vector<uint64_t> mod, P, modQP, rootQP;
    gpufhe::native_primes(mod, 1, 60, n, {});
    std::vector<uint64_t> q50;
    gpufhe::native_primes(q50, fullQ - 1, 50, n, mod);
    mod.insert(mod.end(), q50.begin(), q50.end());
    gpufhe::native_primes(P, K, 60, n, mod);
    modQP = mod;
    modQP.insert(modQP.end(), P.begin(), P.end());
    for (uint64_t q : modQP) rootQP.push_back(gpufhe::native_root(n, q));

    // keys and constants (all outside the timed region, as in the reference)
    auto kp = gpufhe::keygen_host(n, modQP, rootQP, 1, 3.19, 101);
    const uint32_t dnum = (fullQ + alpha - 1) / alpha;
    gpufhe::KeySwitchConstants Kf;
    Kf.n = n;
    gpufhe::compute_keyswitch_constants(Kf, mod, P, dnum);
    Kf.alpha = alpha;
    for (size_t i = 0; i < modQP.size(); ++i) {
        Kf.rootModList.push_back(modQP[i]);
        Kf.rootValList.push_back(rootQP[i]);
    }
    std::vector<uint64_t> pmodq(modQP.size());
    for (size_t t = 0; t < modQP.size(); ++t) {
        uint64_t v = 1 % modQP[t];
        for (uint64_t p : P) v = mulmod(v, p % modQP[t], modQP[t]);
        pmodq[t] = v;
    }
    gpufhe::evalkeygen_host(Kf, kp.s, kp.pkA, kp.pkB, pmodq, modQP, rootQP, 1, 3.19, 202);

    // one context per distinct level, each with the full-QP key
    std::map<uint32_t, gpufhe::DeviceKSContext> ctx;
    std::map<uint32_t, std::pair<std::vector<uint64_t>, std::vector<uint64_t>>> rs;
    uint64_t* d_mods = nullptr;
    ck(cudaMalloc(&d_mods, fullQ * 8), "cudaMalloc");
    ck(cudaMemcpy(d_mods, mod.data(), fullQ * 8, cudaMemcpyHostToDevice), "upload");
    for (uint32_t L : levels) {
        if (ctx.count(L)) continue;
        gpufhe::KeySwitchConstants KL;
        KL.n = n;
        std::vector<uint64_t> ml(mod.begin(), mod.begin() + L);
        gpufhe::compute_keyswitch_constants(KL, ml, P, (L + alpha - 1) / alpha);
        KL.alpha = alpha;
        KL.fullQ = fullQ;
        KL.rootModList = Kf.rootModList;
        KL.rootValList = Kf.rootValList;
        KL.av = Kf.av;
        KL.bv = Kf.bv;
        KL.evalKeyTowers = fullQ + K;
        ctx[L] = gpufhe::ks_context_create(KL);
        gpufhe::native_rescale_consts(rs[L].first, rs[L].second, ml, L - 1);
    }

    // per-chain operands (seeded like the reference driver) and graphs
    std::mt19937_64 rng(7);
    cudaStream_t cap;
    ck(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream");
    std::vector<Chain> ch(levels.size());
    std::vector<std::vector<uint64_t>> host_in;
    for (size_t c = 0; c < ch.size(); ++c) {
        Chain& x = ch[c];
        x.L = levels[c];
        const size_t T = (size_t)x.L * n;
        for (uint64_t** p : {&x.c0a, &x.c1a, &x.c0b, &x.c1b, &x.t0, &x.t1, &x.t2, &x.ba0, &x.ba1, &x.r0, &x.r1})
            ck(cudaMalloc(p, T * 8), "cudaMalloc");
        ck(cudaMalloc(&x.scr, (size_t)n * 8), "cudaMalloc");
        ck(cudaMalloc(&x.drp, (size_t)n * 8), "cudaMalloc");
        for (uint64_t* d : {x.c0a, x.c1a, x.c0b, x.c1b}) {
            std::vector<uint64_t> h(T);
            for (uint32_t t = 0; t < x.L; ++t)
                for (uint32_t k = 0; k < n; ++k) h[(size_t)t * n + k] = rng() % mod[t];
            ck(cudaMemcpy(d, h.data(), T * 8, cudaMemcpyHostToDevice), "upload");
            if (dump != "-") host_in.push_back(std::move(h));
        }
        const gpufhe::DeviceKSContext& C = ctx[x.L];
        x.W = gpufhe::ks_work_create(C);
        cudaGraph_t g;
        ck(cudaStreamBeginCapture(cap, cudaStreamCaptureModeGlobal), "capture");
        LaunchTensor(x.c0a, x.c1a, x.c0b, x.c1b, x.t0, x.t1, x.t2, d_mods, x.L, n, cap);
        gpufhe::keyswitch_resident(x.t2, x.ba0, x.ba1, C, x.W, cap);
        LaunchCombine(x.r0, x.r1, x.t0, x.t1, x.ba0, x.ba1, d_mods, x.L, n, cap);
        gpufhe::rescale_resident_raw(x.r0, x.L, C, rs[x.L].first, rs[x.L].second, x.scr, x.drp, cap);
        gpufhe::rescale_resident_raw(x.r1, x.L, C, rs[x.L].first, rs[x.L].second, x.scr, x.drp, cap);
        ck(cudaStreamEndCapture(cap, &g), "end capture");
        ck(cudaGraphInstantiate(&x.exec, g, nullptr, nullptr, 0), "instantiate");
        ck(cudaGraphDestroy(g), "graph destroy");
    }
    ck(cudaDeviceSynchronize(), "setup");

    constexpr int NS = 16;
    std::vector<cudaStream_t> st(NS);
    for (auto& s : st) ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    cudaEvent_t a, b, fork;
    std::vector<cudaEvent_t> join(NS);
    ck(cudaEventCreate(&a), "event");
    ck(cudaEventCreate(&b), "event");
    ck(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
    for (auto& e : join) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    auto one_stream = [&]() {
        for (auto& x : ch) ck(cudaGraphLaunch(x.exec, st[0]), "launch");
    };
    auto spread = [&]() {
        ck(cudaEventRecord(fork, st[0]), "record");
        for (int s = 1; s < NS; ++s) ck(cudaStreamWaitEvent(st[s], fork, 0), "wait");
        for (size_t c = 0; c < ch.size(); ++c) ck(cudaGraphLaunch(ch[c].exec, st[c % NS]), "launch");
        for (int s = 1; s < NS; ++s) {
            ck(cudaEventRecord(join[s], st[s]), "record");
            ck(cudaStreamWaitEvent(st[0], join[s], 0), "wait");
        }
    };
    auto timed = [&](auto&& f) {
        for (int w = 0; w < 3; ++w) f();
        ck(cudaStreamSynchronize(st[0]), "sync");
        ck(cudaEventRecord(a, st[0]), "record");
        for (uint32_t r = 0; r < reps; ++r) f();
        ck(cudaEventRecord(b, st[0]), "record");
        ck(cudaEventSynchronize(b), "sync");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
        return ms / reps;
    };
    const float ms1 = timed(one_stream);
    const float msn = timed(spread);
    ck(cudaDeviceSynchronize(), "sync");

    if (dump != "-") {
        FILE* f = std::fopen(dump.c_str(), "wb");
        if (!f) { std::perror("dump"); return 1; }
        for (size_t c = 0; c < ch.size(); ++c) {
            const Chain& x = ch[c];
            for (int i = 0; i < 4; ++i) std::fwrite(host_in[4 * c + i].data(), 8, host_in[4 * c + i].size(), f);
            std::vector<uint64_t> o((size_t)(x.L - 1) * n);
            for (uint64_t* d : {x.r0, x.r1}) {
                ck(cudaMemcpy(o.data(), d, o.size() * 8, cudaMemcpyDeviceToHost), "download");
                std::fwrite(o.data(), 8, o.size(), f);
            }
        }
        std::fclose(f);
    }
    std::printf("{\"chains\": %zu, \"one_stream_ms\": %.6f, \"streams16_ms\": %.6f}\n", ch.size(), ms1, msn);

    for (auto& x : ch) {
        cudaGraphExecDestroy(x.exec);
        gpufhe::ks_work_destroy(x.W);
        for (uint64_t* p : {x.c0a, x.c1a, x.c0b, x.c1b, x.t0, x.t1, x.t2, x.ba0, x.ba1, x.r0, x.r1, x.scr, x.drp})
            cudaFree(p);
    }
    for (auto& kv : ctx) gpufhe::ks_context_destroy(kv.second);
    cudaFree(d_mods);
    return 0;
}
