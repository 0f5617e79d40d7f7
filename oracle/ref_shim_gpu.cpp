/*
 * TEST INFRASTRUCTURE ONLY. C entry points over the reference library rebuilt
 * from its own sources for sm_100a (oracle/build_ref.sh -> oracle/_ref/).
 * GPU parity tests and tests/golden/make_golden.py call these to run the
 * reference's own keygen / encrypt / keyswitch_resident / rescale /
 * rotate_ct_device on the same seeded inputs as the oracle and the product.
 * Host buffers in and out; every call synchronizes.
 */
#include "keyswitch.h"            /* reference include/ */
#include "keyswitch_resident.h"
#include "keygen.h"
#include "ntt.h"
#include "intt.h"
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" void LaunchTensor(const uint64_t*, const uint64_t*, const uint64_t*, const uint64_t*,
                             uint64_t*, uint64_t*, uint64_t*, const uint64_t*, uint32_t, uint32_t,
                             cudaStream_t);
extern "C" void LaunchCombine(uint64_t*, uint64_t*, const uint64_t*, const uint64_t*,
                              const uint64_t*, const uint64_t*, const uint64_t*, uint32_t,
                              uint32_t, cudaStream_t);

namespace gpufhe {
void native_rescale_consts(std::vector<uint64_t>&, std::vector<uint64_t>&, const std::vector<uint64_t>&, uint32_t);
void automorphism_eval_host(std::vector<uint64_t>&, uint32_t, uint32_t, uint32_t,
                            const std::vector<uint64_t>&, const std::vector<uint64_t>&);
/* headerless in the reference; declared the way its tests declare them */
void pt_to_eval_host(std::vector<uint64_t>&, const std::vector<int64_t>&, uint32_t, uint32_t,
                     const std::vector<uint64_t>&, const std::vector<uint64_t>&);
void ct_add_ct_host(std::vector<uint64_t>&, std::vector<uint64_t>&, const std::vector<uint64_t>&,
                    const std::vector<uint64_t>&, uint32_t, uint32_t, const std::vector<uint64_t>&);
void ct_mul_pt_host(std::vector<uint64_t>&, std::vector<uint64_t>&, const std::vector<uint64_t>&, uint32_t,
                    uint32_t, const std::vector<uint64_t>&);
void rotate_ct_host(std::vector<uint64_t>&, std::vector<uint64_t>&, uint32_t, const KeySwitchConstants&,
                    uint32_t, uint32_t, const std::vector<uint64_t>&, const std::vector<uint64_t>&);
}

typedef uint64_t u64;
typedef std::vector<u64> vec;

struct RefH {
    uint32_t n, fullQ, K;
    vec Q, P, rQ, rP;
    std::vector<uint32_t> key_np;                 /* numPart the key was made with */
    std::vector<std::vector<vec>> av, bv;         /* [key][part] -> [fullQ+K][n] */
};

static gpufhe::KeySwitchConstants level_consts(const RefH* h, uint32_t L, uint32_t numPart) {
    gpufhe::KeySwitchConstants C;
    C.n = h->n;
    vec q(h->Q.begin(), h->Q.begin() + L);
    gpufhe::compute_keyswitch_constants(C, q, h->P, numPart);
    for (uint32_t i = 0; i < L; ++i) { C.rootModList.push_back(h->Q[i]); C.rootValList.push_back(h->rQ[i]); }
    for (uint32_t j = 0; j < h->K; ++j) { C.rootModList.push_back(h->P[j]); C.rootValList.push_back(h->rP[j]); }
    /* ks_context_create (keyswitch_resident.cpp:73-84) reads av/bv[part] for
     * every part: give it empty per-part vectors until a key is attached. */
    C.av.assign(C.numPart, {});
    C.bv.assign(C.numPart, {});
    return C;
}

static void attach_key(const RefH* h, gpufhe::KeySwitchConstants& C, uint32_t key) {
    C.fullQ = h->fullQ;
    C.evalKeyTowers = h->fullQ + h->K;
    C.av.assign(C.numPart, {}); C.bv.assign(C.numPart, {});
    for (uint32_t p = 0; p < C.numPart; ++p) { C.av[p] = h->av[key][p]; C.bv[p] = h->bv[key][p]; }
}

static u64* dup(const u64* host, size_t words) {
    u64* d = nullptr;
    cudaMalloc(&d, words * 8);
    cudaMemcpy(d, host, words * 8, cudaMemcpyHostToDevice);
    return d;
}

extern "C" {

void* refg_create(uint32_t n, const u64* Q, uint32_t fullQ, const u64* P, uint32_t K, const u64* rootsQP) {
    RefH* h = new RefH();
    h->n = n; h->fullQ = fullQ; h->K = K;
    h->Q.assign(Q, Q + fullQ); h->P.assign(P, P + K);
    h->rQ.assign(rootsQP, rootsQP + fullQ); h->rP.assign(rootsQP + fullQ, rootsQP + fullQ + K);
    return h;
}

void refg_destroy(void* hp) { delete (RefH*)hp; }

void refg_set_hw(uint32_t hw) { gpufhe::set_secret_hamming_weight(hw); }

void refg_keygen(uint32_t n, const u64* mods, uint32_t nm, const u64* roots, u64 ns, double sigma,
                 u64 seed, u64* s, u64* pkA, u64* pkB) {
    vec m(mods, mods + nm), r(roots, roots + nm);
    auto kp = gpufhe::keygen_host(n, m, r, ns, sigma, seed);
    std::memcpy(s, kp.s.data(), kp.s.size() * 8);
    std::memcpy(pkA, kp.pkA.data(), kp.pkA.size() * 8);
    std::memcpy(pkB, kp.pkB.data(), kp.pkB.size() * 8);
}

/* evalkeygen_host_sold over full QP with numPart digits; av/bv out [numPart][fullQ+K][n]. */
void refg_evalkeygen(void* hp, uint32_t numPart, const u64* sQP, const u64* sOld, const u64* pkA,
                     const u64* pkB, u64 ns, double sigma, u64 seed, u64* av, u64* bv) {
    RefH* h = (RefH*)hp;
    const uint32_t QP = h->fullQ + h->K;
    const size_t W = (size_t)QP * h->n;
    auto C = level_consts(h, h->fullQ, numPart);
    vec modQP = h->Q, rootQP = h->rQ;
    modQP.insert(modQP.end(), h->P.begin(), h->P.end());
    rootQP.insert(rootQP.end(), h->rP.begin(), h->rP.end());
    vec PM(QP);
    for (uint32_t t = 0; t < QP; ++t) {
        u64 q = modQP[t], P = 1 % q;
        for (uint32_t j = 0; j < h->K; ++j) P = (u64)(((unsigned __int128)P * (h->P[j] % q)) % q);
        PM[t] = P;
    }
    gpufhe::evalkeygen_host_sold(C, vec(sQP, sQP + W), vec(sOld, sOld + W), vec(pkA, pkA + W),
                                 vec(pkB, pkB + W), PM, modQP, rootQP, ns, sigma, seed);
    for (uint32_t p = 0; p < C.numPart; ++p) {
        std::memcpy(av + p * W, C.av[p].data(), W * 8);
        std::memcpy(bv + p * W, C.bv[p].data(), W * 8);
    }
}

void refg_set_key(void* hp, uint32_t key, uint32_t numPart, const u64* av, const u64* bv) {
    RefH* h = (RefH*)hp;
    const size_t W = (size_t)(h->fullQ + h->K) * h->n;
    if (h->av.size() <= key) { h->av.resize(key + 1); h->bv.resize(key + 1); h->key_np.resize(key + 1); }
    h->key_np[key] = numPart;
    h->av[key].clear(); h->bv[key].clear();
    for (uint32_t p = 0; p < numPart; ++p) {
        h->av[key].emplace_back(av + p * W, av + (p + 1) * W);
        h->bv[key].emplace_back(bv + p * W, bv + (p + 1) * W);
    }
}

void refg_encrypt(uint32_t n, const u64* mods, uint32_t nm, const u64* roots, const int64_t* m,
                  const u64* pkA, const u64* pkB, u64 ns, double sigma, u64 seed, u64* c0, u64* c1) {
    vec md(mods, mods + nm), r(roots, roots + nm), c0v, c1v;
    const size_t W = (size_t)nm * n;
    gpufhe::encrypt_host(c0v, c1v, std::vector<int64_t>(m, m + n), vec(pkA, pkA + W), vec(pkB, pkB + W),
                         n, md, r, ns, sigma, seed);
    std::memcpy(c0, c0v.data(), W * 8);
    std::memcpy(c1, c1v.data(), W * 8);
}

void refg_decrypt(uint32_t n, const u64* mods, uint32_t nm, const u64* roots, const u64* c0,
                  const u64* c1, const u64* s, int64_t* mout) {
    vec md(mods, mods + nm), r(roots, roots + nm);
    const size_t W = (size_t)nm * n;
    std::vector<int64_t> o;
    gpufhe::decrypt_host(o, vec(c0, c0 + W), vec(c1, c1 + W), vec(s, s + W), n, md, r);
    std::memcpy(mout, o.data(), (size_t)n * 8);
}

void refg_automorph_host(uint32_t n, uint32_t towers, uint32_t k, const u64* mods, const u64* roots, u64* v) {
    vec x(v, v + (size_t)towers * n);
    gpufhe::automorphism_eval_host(x, towers, n, k, vec(mods, mods + towers), vec(roots, roots + towers));
    std::memcpy(v, x.data(), x.size() * 8);
}

/* pt_to_eval_host (rotate.cpp:104-112) */
void refg_pt_to_eval(uint32_t n, uint32_t towers, const u64* mods, const u64* roots, const int64_t* m, u64* out) {
    vec o;
    gpufhe::pt_to_eval_host(o, std::vector<int64_t>(m, m + n), towers, n, vec(mods, mods + towers),
                            vec(roots, roots + towers));
    std::memcpy(out, o.data(), o.size() * 8);
}

/* ct_add_ct_host (mul = 0, d1 used) or ct_mul_pt_host (mul = 1, d0 is the
 * plaintext) (ptops.cpp:13-26) */
void refg_ptops(uint32_t n, uint32_t towers, const u64* mods, int mul, u64* c0, u64* c1, const u64* d0,
                const u64* d1) {
    const size_t T = (size_t)towers * n;
    vec a(c0, c0 + T), b(c1, c1 + T), md(mods, mods + towers);
    if (mul) gpufhe::ct_mul_pt_host(a, b, vec(d0, d0 + T), towers, n, md);
    else gpufhe::ct_add_ct_host(a, b, vec(d0, d0 + T), vec(d1, d1 + T), towers, n, md);
    std::memcpy(c0, a.data(), T * 8);
    std::memcpy(c1, b.data(), T * 8);
}

/* rotate_ct_host with rotation key `key` at level L (rotate.cpp:176-188) */
int refg_rotate_host(void* hp, uint32_t key, uint32_t L, uint32_t numPart, uint32_t k, u64* c0, u64* c1) {
    RefH* h = (RefH*)hp;
    auto C = level_consts(h, L, numPart);
    attach_key(h, C, key);
    const size_t T = (size_t)L * h->n;
    vec a(c0, c0 + T), b(c1, c1 + T);
    gpufhe::rotate_ct_host(a, b, k, C, L, h->n, vec(h->Q.begin(), h->Q.begin() + L),
                           vec(h->rQ.begin(), h->rQ.begin() + L));
    std::memcpy(c0, a.data(), T * 8);
    std::memcpy(c1, b.data(), T * 8);
    return (int)cudaGetLastError();
}

/* keyswitch_resident at level L (device path) */
int refg_keyswitch_resident(void* hp, uint32_t key, uint32_t L, uint32_t numPart, const u64* a,
                            u64* ba0, u64* ba1) {
    RefH* h = (RefH*)hp;
    auto C = level_consts(h, L, numPart);
    attach_key(h, C, key);
    auto D = gpufhe::ks_context_create(C);
    auto W = gpufhe::ks_work_create(D);
    const size_t T = (size_t)L * h->n;
    u64 *da = dup(a, T), *d0, *d1;
    cudaMalloc(&d0, T * 8); cudaMalloc(&d1, T * 8);
    gpufhe::keyswitch_resident(da, d0, d1, D, W, 0);
    cudaDeviceSynchronize();
    cudaMemcpy(ba0, d0, T * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(ba1, d1, T * 8, cudaMemcpyDeviceToHost);
    cudaFree(da); cudaFree(d0); cudaFree(d1);
    gpufhe::ks_work_destroy(W); gpufhe::ks_context_destroy(D);
    return (int)cudaGetLastError();
}

/* keyswitch_core_resident at level L (host-orchestrated path) */
int refg_keyswitch_core(void* hp, uint32_t key, uint32_t L, uint32_t numPart, const u64* a, u64* ba0,
                        u64* ba1) {
    RefH* h = (RefH*)hp;
    auto C = level_consts(h, L, numPart);
    attach_key(h, C, key);
    auto R = gpufhe::keyswitch_core_resident(vec(a, a + (size_t)L * h->n), C);
    std::memcpy(ba0, R.ba0.data(), R.ba0.size() * 8);
    std::memcpy(ba1, R.ba1.data(), R.ba1.size() * 8);
    return (int)cudaGetLastError();
}

/* rescale_resident_raw on one [L][n] component with native_rescale_consts */
int refg_rescale(void* hp, uint32_t L, uint32_t numPart, u64* comp) {
    RefH* h = (RefH*)hp;
    auto C = level_consts(h, L, numPart);
    C.fullQ = h->fullQ;
    auto D = gpufhe::ks_context_create(C);
    vec s1, s2;
    gpufhe::native_rescale_consts(s1, s2, vec(h->Q.begin(), h->Q.begin() + L), L - 1);
    const size_t T = (size_t)L * h->n;
    u64 *dc = dup(comp, T), *scr, *drp;
    cudaMalloc(&scr, (size_t)h->n * 8); cudaMalloc(&drp, (size_t)h->n * 8);
    gpufhe::rescale_resident_raw(dc, L, D, s1, s2, scr, drp, 0);
    cudaDeviceSynchronize();
    cudaMemcpy(comp, dc, T * 8, cudaMemcpyDeviceToHost);
    cudaFree(dc); cudaFree(scr); cudaFree(drp);
    gpufhe::ks_context_destroy(D);
    return (int)cudaGetLastError();
}

/* One EvalMult+Rescale exactly as bench_evalmult_resident.cpp:96-100 chains it. */
int refg_evalmult_rescale(void* hp, uint32_t L, uint32_t numPart, const u64* c0a, const u64* c1a,
                          const u64* c0b, const u64* c1b, u64* out0, u64* out1) {
    RefH* h = (RefH*)hp;
    auto C = level_consts(h, L, numPart);
    attach_key(h, C, 0);
    auto D = gpufhe::ks_context_create(C);
    auto W = gpufhe::ks_work_create(D);
    const uint32_t n = h->n;
    const size_t T = (size_t)L * n;
    vec s1, s2;
    gpufhe::native_rescale_consts(s1, s2, vec(h->Q.begin(), h->Q.begin() + L), L - 1);
    u64 *a0 = dup(c0a, T), *a1 = dup(c1a, T), *b0 = dup(c0b, T), *b1 = dup(c1b, T);
    u64 *dm = dup(h->Q.data(), L);
    u64 *t0, *t1, *t2, *x0, *x1, *r0, *r1, *scr, *drp;
    for (u64** p : {&t0, &t1, &t2, &x0, &x1, &r0, &r1}) cudaMalloc(p, T * 8);
    cudaMalloc(&scr, (size_t)n * 8); cudaMalloc(&drp, (size_t)n * 8);
    LaunchTensor(a0, a1, b0, b1, t0, t1, t2, dm, L, n, 0);
    gpufhe::keyswitch_resident(t2, x0, x1, D, W, 0);
    LaunchCombine(r0, r1, t0, t1, x0, x1, dm, L, n, 0);
    gpufhe::rescale_resident_raw(r0, L, D, s1, s2, scr, drp, 0);
    gpufhe::rescale_resident_raw(r1, L, D, s1, s2, scr, drp, 0);
    cudaDeviceSynchronize();
    cudaMemcpy(out0, r0, (size_t)(L - 1) * n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(out1, r1, (size_t)(L - 1) * n * 8, cudaMemcpyDeviceToHost);
    for (u64* p : {a0, a1, b0, b1, dm, t0, t1, t2, x0, x1, r0, r1, scr, drp}) cudaFree(p);
    gpufhe::ks_work_destroy(W); gpufhe::ks_context_destroy(D);
    return (int)cudaGetLastError();
}

/* rotate_ct_device with rotation key `key` at level L (rotate.cpp:118-132) */
int refg_rotate_device(void* hp, uint32_t key, uint32_t L, uint32_t numPart, uint32_t k, u64* c0, u64* c1) {
    RefH* h = (RefH*)hp;
    auto C = level_consts(h, L, numPart);
    attach_key(h, C, key);
    auto D = gpufhe::ks_context_create(C);
    auto W = gpufhe::ks_work_create(D);
    const uint32_t n = h->n;
    const size_t T = (size_t)L * n;
    u64 *d0 = dup(c0, T), *d1 = dup(c1, T), *sc, *b0, *b1;
    cudaMalloc(&sc, (size_t)n * 8); cudaMalloc(&b0, T * 8); cudaMalloc(&b1, T * 8);
    vec mod(h->Q.begin(), h->Q.begin() + L), root(h->rQ.begin(), h->rQ.begin() + L);
    gpufhe::rotate_ct_device(d0, d1, k, D, W, L, n, mod, root, sc, b0, b1, 0);
    cudaDeviceSynchronize();
    cudaMemcpy(c0, d0, T * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(c1, d1, T * 8, cudaMemcpyDeviceToHost);
    for (u64* p : {d0, d1, sc, b0, b1}) cudaFree(p);
    gpufhe::ks_work_destroy(W); gpufhe::ks_context_destroy(D);
    return (int)cudaGetLastError();
}

/* LaunchNTT_CT / LaunchINTT_GS on one tower with tables built from root */
int refg_ntt(u64* x, uint32_t n, u64 q, const u64* fr, const u64* fp, int inverse, u64 ninv, u64 ninvp) {
    u64 *dx = dup(x, n), *dr = dup(fr, n), *dp = dup(fp, n);
    if (inverse) LaunchINTT_GS(dx, dr, dp, n, q, ninv, ninvp, 0);
    else LaunchNTT_CT(dx, dr, dp, n, q, 0);
    cudaDeviceSynchronize();
    cudaMemcpy(x, dx, (size_t)n * 8, cudaMemcpyDeviceToHost);
    cudaFree(dx); cudaFree(dr); cudaFree(dp);
    return (int)cudaGetLastError();
}

}  // extern "C"
