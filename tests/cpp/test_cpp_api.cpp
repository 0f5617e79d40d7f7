// C++ API gate, written the way the reference's own tests call it
// (tests/test_evalmult_rescale.cpp, test_ks_graph.cpp, test_rot_resident.cpp),
// with native primes/roots instead of OpenFHE. Links libgpufhe_b200.so only.
// Prints [PASS]/[FAIL] lines; exit 0 when every gate passes. Writes the
// EvalMult+Rescale output and the keyswitch output to argv[1] (binary) so the
// Python test can compare them with the CPU oracle bit for bit.
#include <cuda_runtime.h>
#include <algorithm>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <vector>

#include "ckks_ops.h"
#include "device_ciphertext.h"
#include "encode.h"
#include "host_ops.h"
#include "keygen.h"
#include "keyswitch.h"
#include "keyswitch_resident.h"
#include "basis_convert.h"
#include "intt.h"
#include "ntt.h"
#include "params.h"
#include "tensor.h"

using u64 = uint64_t;
static u64 mm(u64 a, u64 b, u64 q) { return (u64)(((unsigned __int128)a * b) % q); }
static int fails = 0;
static void gate(bool ok, const char* what) {
    std::printf("[%s] %s\n", ok ? "PASS" : "FAIL", what);
    if (!ok) ++fails;
}

int main(int argc, char** argv) {
    const uint32_t n = 4096, sizeQ = 6, sizeP = 3, numPart = 2;
    const u64 ns = 1;
    std::vector<u64> mod, modP;
    gpufhe::native_primes(mod, 1, 60, n, {});
    { std::vector<u64> mids; gpufhe::native_primes(mids, sizeQ - 1, 50, n, mod); for (u64 m : mids) mod.push_back(m); }
    gpufhe::native_primes(modP, sizeP, 60, n, mod);
    std::vector<u64> modQP = mod, root(sizeQ), rootQP;
    for (u64 p : modP) modQP.push_back(p);
    for (uint32_t i = 0; i < sizeQ; ++i) root[i] = gpufhe::native_root(n, mod[i]);
    rootQP = root;
    for (u64 p : modP) rootQP.push_back(gpufhe::native_root(n, p));
    const uint32_t sizeQlP = sizeQ + sizeP;

    auto KPqp = gpufhe::keygen_host(n, modQP, rootQP, ns, 3.19, 101);
    auto KPq = gpufhe::keygen_host(n, mod, root, ns, 3.19, 101);
    gpufhe::KeySwitchConstants K;
    K.n = n;
    gpufhe::compute_keyswitch_constants(K, mod, modP, numPart);
    for (uint32_t i = 0; i < sizeQ; ++i) { K.rootModList.push_back(mod[i]); K.rootValList.push_back(root[i]); }
    for (uint32_t j = 0; j < sizeP; ++j) { K.rootModList.push_back(modP[j]); K.rootValList.push_back(rootQP[sizeQ + j]); }
    std::vector<u64> PModq(sizeQlP);
    for (uint32_t t = 0; t < sizeQlP; ++t) {
        u64 q = modQP[t], P = 1 % q;
        for (u64 p : modP) P = mm(P, p % q, q);
        PModq[t] = P;
    }
    gpufhe::evalkeygen_host(K, KPqp.s, KPqp.pkA, KPqp.pkB, PModq, modQP, rootQP, ns, 3.19, 202);
    std::vector<u64> s1, s2;
    gpufhe::native_rescale_consts(s1, s2, mod, sizeQ - 1);

    const int64_t D = (int64_t)1 << 40;
    std::vector<int64_t> a1(n, 0), a2(n, 0);
    a1[0] = 3; a1[1] = -2; a2[0] = 4; a2[2] = 5;
    std::vector<int64_t> m1(n), m2(n);
    for (uint32_t k = 0; k < n; ++k) { m1[k] = a1[k] * D; m2[k] = a2[k] * D; }
    std::vector<u64> c0a, c1a, c0b, c1b;
    gpufhe::encrypt_host(c0a, c1a, m1, KPq.pkA, KPq.pkB, n, mod, root, ns, 3.19, 303);
    gpufhe::encrypt_host(c0b, c1b, m2, KPq.pkA, KPq.pkB, n, mod, root, ns, 3.19, 304);

    {   // fresh encryption decrypts (encdec round trip)
        std::vector<int64_t> dec;
        gpufhe::decrypt_host(dec, c0a, c1a, KPq.s, n, mod, root);
        bool ok = true;
        for (uint32_t k = 0; k < n; ++k) ok &= std::llround((double)dec[k] / (double)D) == a1[k];
        gate(ok, "encrypt_host/decrypt_host round trip");
    }

    auto C = gpufhe::ks_context_create(K);
    auto W = gpufhe::ks_work_create(C);
    const size_t T = (size_t)sizeQ * n;
    auto up = [&](const std::vector<u64>& h) { u64* d; cudaMalloc(&d, T * 8); cudaMemcpy(d, h.data(), T * 8, cudaMemcpyHostToDevice); return d; };
    u64 *dc0a = up(c0a), *dc1a = up(c1a), *dc0b = up(c0b), *dc1b = up(c1b);
    u64 *t0, *t1, *t2, *ba0, *ba1, *r0, *r1, *scr, *drp, *dmods;
    for (u64** p : {&t0, &t1, &t2, &ba0, &ba1, &r0, &r1}) cudaMalloc(p, T * 8);
    cudaMalloc(&scr, (size_t)n * 8); cudaMalloc(&drp, (size_t)n * 8);
    cudaMalloc(&dmods, sizeQ * 8);
    cudaMemcpy(dmods, mod.data(), sizeQ * 8, cudaMemcpyHostToDevice);

    LaunchTensor(dc0a, dc1a, dc0b, dc1b, t0, t1, t2, dmods, sizeQ, n, 0);
    gpufhe::keyswitch_resident(t2, ba0, ba1, C, W, 0);
    std::vector<u64> ks0(T), ks1(T);
    cudaDeviceSynchronize();
    cudaMemcpy(ks0.data(), ba0, T * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(ks1.data(), ba1, T * 8, cudaMemcpyDeviceToHost);
    LaunchCombine(r0, r1, t0, t1, ba0, ba1, dmods, sizeQ, n, 0);
    gpufhe::rescale_resident_raw(r0, sizeQ, C, s1, s2, scr, drp, 0);
    gpufhe::rescale_resident_raw(r1, sizeQ, C, s1, s2, scr, drp, 0);
    gate(cudaDeviceSynchronize() == cudaSuccess, "EvalMult+Rescale chain runs");
    std::vector<u64> h0(T), h1(T);
    cudaMemcpy(h0.data(), r0, T * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(h1.data(), r1, T * 8, cudaMemcpyDeviceToHost);
    {
        std::vector<u64> mR(mod.begin(), mod.end() - 1), rR(root.begin(), root.end() - 1);
        auto KPr = gpufhe::keygen_host(n, mR, rR, ns, 3.19, 101);
        std::vector<int64_t> dec;
        gpufhe::decrypt_host(dec, h0, h1, KPr.s, n, mR, rR);
        std::vector<int64_t> expect(n, 0);
        for (uint32_t i = 0; i < n; ++i) if (a1[i]) for (uint32_t j = 0; j < n; ++j) if (a2[j]) {
            uint32_t idx = (i + j) % n; int64_t sg = (i + j) >= n ? -1 : 1; expect[idx] += sg * a1[i] * a2[j]; }
        const long double qLast = (long double)mod[sizeQ - 1], D2 = (long double)D * (long double)D;
        int bad = 0;
        for (uint32_t k = 0; k < n; ++k) if ((int64_t)llroundl((long double)dec[k] * qLast / D2) != expect[k]) ++bad;
        gate(bad == 0, "EvalMult+Rescale decrypts to (3-2x)(4+5x^2) exactly");
    }

    {   // graph replay == direct (test_ks_graph.cpp:45-67), outputs zeroed first
        cudaMemset(ba0, 0, T * 8); cudaMemset(ba1, 0, T * 8);
        cudaStream_t s; cudaStreamCreate(&s);
        cudaGraph_t g; cudaGraphExec_t ge;
        cudaStreamBeginCapture(s, cudaStreamCaptureModeGlobal);
        gpufhe::keyswitch_resident(t2, ba0, ba1, C, W, s);
        cudaStreamEndCapture(s, &g);
        bool ok = cudaGraphInstantiate(&ge, g, nullptr, nullptr, 0) == cudaSuccess;
        ok = ok && cudaGraphLaunch(ge, s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess;
        std::vector<u64> g0(T), g1(T);
        cudaMemcpy(g0.data(), ba0, T * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(g1.data(), ba1, T * 8, cudaMemcpyDeviceToHost);
        ok = ok && g0 == ks0 && g1 == ks1;
        gate(ok, "keyswitch_resident graph replay bit-exact vs direct");
        cudaGraphExecDestroy(ge); cudaGraphDestroy(g); cudaStreamDestroy(s);
    }

    {   // the context's public tables (the reference's names and layouts), used
        // the way a caller composing the Launch* entry points uses them
        bool ok = C.d_av.size() == numPart && C.d_bv.size() == numPart && C.d_qhi.size() == numPart;
        for (uint32_t p = 0; ok && p < numPart; ++p) {   // eval key rows as given
            std::vector<u64> av(K.av[p].size()), bv(K.bv[p].size());
            cudaMemcpy(av.data(), C.d_av[p], av.size() * 8, cudaMemcpyDeviceToHost);
            cudaMemcpy(bv.data(), C.d_bv[p], bv.size() * 8, cudaMemcpyDeviceToHost);
            ok = av == K.av[p] && bv == K.bv[p];
        }
        gate(ok, "DeviceKSContext d_av / d_bv hold the eval key rows");
        // NTT with d_fr / d_fp, inverse with d_ir / d_ip / ninv: a round trip
        // on one 60-bit, one 50-bit and one P tower
        ok = C.modList.size() == sizeQlP && C.d_fr.size() == sizeQlP && C.ninv.size() == sizeQlP;
        u64* dx; cudaMalloc(&dx, (size_t)n * 8);
        for (uint32_t r : {0u, 2u, sizeQ + 1}) {
            if (!ok) break;
            std::vector<u64> x(n), y(n);
            std::mt19937_64 g(77 + r);
            for (auto& v : x) v = g() % C.modList[r];
            cudaMemcpy(dx, x.data(), (size_t)n * 8, cudaMemcpyHostToDevice);
            LaunchNTT_CT(dx, C.d_fr[r], C.d_fp[r], n, C.modList[r], 0);
            cudaMemcpy(y.data(), dx, (size_t)n * 8, cudaMemcpyDeviceToHost);
            LaunchINTT_GS(dx, C.d_ir[r], C.d_ip[r], n, C.modList[r], C.ninv[r], C.ninv_p[r], 0);
            std::vector<u64> z(n);
            cudaMemcpy(z.data(), dx, (size_t)n * 8, cudaMemcpyDeviceToHost);
            ok = y != x && z == x;
        }
        gate(ok, "DeviceKSContext d_fr / d_fp / d_ir / d_ip / ninv: NTT round trip");
        // ApproxSwitchCRTBasis of digit 1 with d_qhi ... d_mhi against the
        // formula on the host: y_i = x_i * QHatInv_i mod q_i, out_j = sum_i
        // y_i * QHatModp[i][j] mod p_j
        {
            const uint32_t p = 1, sp = C.sizePart[p], sc = C.sizeCompl[p], st = C.startIdx[p];
            std::vector<u64> src((size_t)sp * n), dst((size_t)sc * n);
            std::mt19937_64 g(91);
            for (uint32_t i = 0; i < sp; ++i)
                for (uint32_t k = 0; k < n; ++k) src[(size_t)i * n + k] = g() % mod[st + i];
            u64 *dsrc, *ddst;
            cudaMalloc(&dsrc, src.size() * 8); cudaMalloc(&ddst, dst.size() * 8);
            cudaMemcpy(dsrc, src.data(), src.size() * 8, cudaMemcpyHostToDevice);
            LaunchApproxSwitchCRTBasis(dsrc, ddst, C.d_qhi[p], C.d_qhip[p], C.d_srcMod[p], C.d_qmp[p],
                                       C.d_complMod[p], C.d_mlo[p], C.d_mhi[p], sp, sc, n, 0);
            cudaMemcpy(dst.data(), ddst, dst.size() * 8, cudaMemcpyDeviceToHost);
            bool cv = C.complModHost[p] == K.partComplMod[p];
            for (uint32_t j = 0; cv && j < sc; ++j) {
                const u64 pj = K.partComplMod[p][j];
                for (uint32_t k = 0; cv && k < n; ++k) {
                    unsigned __int128 acc = 0;
                    for (uint32_t i = 0; i < sp; ++i) {
                        const u64 qi = mod[st + i], y = mm(src[(size_t)i * n + k], K.partQHatInv[p][i], qi);
                        acc += (unsigned __int128)y * K.partQHatModp[p][(size_t)i * sc + j];
                    }
                    cv = dst[(size_t)j * n + k] == (u64)(acc % pj);
                }
            }
            gate(cv, "DeviceKSContext d_qhi ... d_mhi drive LaunchApproxSwitchCRTBasis");
            cudaFree(dsrc); cudaFree(ddst);
        }
        cudaFree(dx);
        std::vector<u64> mq(sizeQlP), md(sizeQ), pm(sizeP);
        std::vector<uint32_t> kr(sizeQlP);
        cudaMemcpy(mq.data(), C.d_modsQlP, sizeQlP * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(kr.data(), C.d_keyRow, sizeQlP * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(md.data(), C.d_qMod, sizeQ * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(pm.data(), C.d_pMod, sizeP * 8, cudaMemcpyDeviceToHost);
        ok = mq == modQP && md == mod && pm == modP && W.d_res0 && W.d_res1 && W.d_part && W.d_digPtrs;
        for (uint32_t i = 0; i < sizeQlP; ++i) ok = ok && kr[i] == i;   // full level: rows in place
        gate(ok, "DeviceKSContext d_modsQlP / d_keyRow / d_qMod / d_pMod and DeviceKSWork scratch");
    }

    {   // keyswitch_core_resident (host vectors) == keyswitch_resident
        std::vector<u64> t2h(T);
        cudaMemcpy(t2h.data(), t2, T * 8, cudaMemcpyDeviceToHost);
        auto R = gpufhe::keyswitch_core_resident(t2h, K);
        gate(R.ba0 == ks0 && R.ba1 == ks1, "keyswitch_core_resident bit-exact vs keyswitch_resident");
    }

    std::vector<u64> sH, g0, g1;
    {   // rotation: device == resident (test_rot_resident.cpp:141-164), and decrypts rotated
        const u64 k = 5;
        std::vector<u64> sA = KPqp.s;
        // sigma_k(s) over QP through the device automorphism
        u64* ds; cudaMalloc(&ds, sA.size() * 8);
        cudaMemcpy(ds, sA.data(), sA.size() * 8, cudaMemcpyHostToDevice);
        gpufhe::automorphism_eval_device(ds, sizeQlP, n, (uint32_t)k, modQP, rootQP, scr, 0);
        cudaMemcpy(sA.data(), ds, sA.size() * 8, cudaMemcpyDeviceToHost);
        gpufhe::KeySwitchConstants Kr;
        Kr.n = n;
        gpufhe::compute_keyswitch_constants(Kr, mod, modP, numPart);
        Kr.rootModList = K.rootModList; Kr.rootValList = K.rootValList;
        gpufhe::evalkeygen_host_sold(Kr, KPqp.s, sA, KPqp.pkA, KPqp.pkB, PModq, modQP, rootQP, ns, 3.19, 404);
        std::vector<u64> e0 = c0a, e1 = c1a;
        gpufhe::rotate_ct_resident(e0, e1, (uint32_t)k, Kr, sizeQ, n, mod, root);
        auto Cr = gpufhe::ks_context_create(Kr);
        auto Wr = gpufhe::ks_work_create(Cr);
        u64 *d0 = up(c0a), *d1 = up(c1a), *b0, *b1;
        cudaMalloc(&b0, T * 8); cudaMalloc(&b1, T * 8);
        gpufhe::rotate_ct_device(d0, d1, (uint32_t)k, Cr, Wr, sizeQ, n, mod, root, scr, b0, b1, 0);
        cudaDeviceSynchronize();
        std::vector<u64> f0(T), f1(T);
        cudaMemcpy(f0.data(), d0, T * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(f1.data(), d1, T * 8, cudaMemcpyDeviceToHost);
        gate(f0 == e0 && f1 == e1, "rotate_ct_device bit-exact vs rotate_ct_resident");
        // the headerless host forms (test_rotate.cpp:42, test_c2s_engine.cpp:55, 101)
        sH = KPqp.s;
        gpufhe::automorphism_eval_host(sH, sizeQlP, n, (uint32_t)k, modQP, rootQP);
        gate(sH == sA, "automorphism_eval_host bit-exact vs automorphism_eval_device");
        g0 = c0a; g1 = c1a;
        gpufhe::rotate_ct_host(g0, g1, (uint32_t)k, Kr, sizeQ, n, mod, root);
        gate(g0 == e0 && g1 == e1, "rotate_ct_host bit-exact vs rotate_ct_resident");
        bool thrown = false;
        try { std::vector<u64> x = c0a; gpufhe::automorphism_eval_host(x, sizeQ, n, 4, mod, root); }
        catch (const std::invalid_argument&) { thrown = true; }
        gate(thrown, "automorphism_eval_host rejects an even Galois element");
        std::vector<int64_t> dec;
        gpufhe::decrypt_host(dec, f0, f1, KPq.s, n, mod, root);
        // sigma_5 maps X -> X^5: 3 - 2x -> 3 - 2x^5
        bool ok = std::llround((double)dec[0] / D) == 3 && std::llround((double)dec[5] / D) == -2 &&
                  std::llround((double)dec[1] / D) == 0;
        gate(ok, "rotation decrypts to sigma_5(3-2x) = 3-2x^5");
        gpufhe::ks_work_destroy(Wr); gpufhe::ks_context_destroy(Cr);
    }

    {   // DeviceCiphertext + mul_resident + rescale_resident (relin-free chain)
        gpufhe::DeviceTables Tb;
        gpufhe::build_device_tables(Tb, n, mod);
        gpufhe::DeviceCiphertext A(gpufhe::Scheme::CKKS, n, sizeQ), B(gpufhe::Scheme::CKKS, n, sizeQ);
        A.upload(c0a, c1a);
        B.upload(c0b, c1b);
        gpufhe::mul_resident(A, B, Tb, 0);
        gpufhe::rescale_resident(A, Tb, s1, s2, 0, scr, drp);
        cudaDeviceSynchronize();
        std::vector<u64> x0, x1;
        A.to_host(x0, x1);
        bool ok = A.num_towers() == sizeQ - 1 && x0.size() == (size_t)(sizeQ - 1) * n;
        // componentwise product then rescale, host check on tower 0 / coefficient-free spot check
        ok = ok && x0[0] < mod[0] && x1[5] < mod[0];
        gate(ok, "DeviceCiphertext mul_resident + rescale_resident");
        bool thrown = false;
        try { A.upload(c0a, c1a); } catch (const std::runtime_error&) { thrown = true; }
        gate(thrown, "DeviceCiphertext::upload throws on size mismatch");
    }

    // plaintext-ciphertext helpers as test_ptops.cpp:60-95 calls them:
    // (3-2x)*D times the unscaled plaintext 4+5x^2, and the sum of the two
    // ciphertexts, each checked by decryption and word for word
    std::vector<u64> pe, pm0 = c0a, pm1 = c1a, pa0 = c0a, pa1 = c1a;
    {
        gpufhe::pt_to_eval_host(pe, a2, sizeQ, n, mod, root);
        gpufhe::ct_mul_pt_host(pm0, pm1, pe, sizeQ, n, mod);
        gpufhe::ct_add_ct_host(pa0, pa1, c0b, c1b, sizeQ, n, mod);
        bool words = pe.size() == T;
        for (uint32_t t = 0; t < sizeQ && words; ++t)
            for (uint32_t j = 0; j < n; ++j) {
                const size_t x = (size_t)t * n + j;
                const u64 q = mod[t], s0 = c0a[x] + c0b[x], s1 = c1a[x] + c1b[x];
                words &= pm0[x] == mm(c0a[x], pe[x], q) && pm1[x] == mm(c1a[x], pe[x], q) &&
                         pa0[x] == (s0 >= q ? s0 - q : s0) && pa1[x] == (s1 >= q ? s1 - q : s1);
            }
        gate(words, "ct_mul_pt_host / ct_add_ct_host word for word");
        std::vector<int64_t> dm, da;
        gpufhe::decrypt_host(dm, pm0, pm1, KPq.s, n, mod, root);
        gpufhe::decrypt_host(da, pa0, pa1, KPq.s, n, mod, root);
        std::vector<int64_t> prod(n, 0);
        for (uint32_t i = 0; i < n; ++i) if (a1[i]) for (uint32_t j = 0; j < n; ++j) if (a2[j]) {
            uint32_t idx = (i + j) % n; int64_t sg = (i + j) >= n ? -1 : 1; prod[idx] += sg * a1[i] * a2[j]; }
        int bad = 0;
        for (uint32_t j = 0; j < n; ++j) {
            bad += std::llround((double)dm[j] / (double)D) != prod[j];
            bad += std::llround((double)da[j] / (double)D) != a1[j] + a2[j];
        }
        gate(bad == 0, "ct_mul_pt_host decrypts to (3-2x)(4+5x^2), ct_add_ct_host to the sum");
        // fewer towers than the vectors hold: only the first towers*n words change
        std::vector<u64> q0 = c0a, q1 = c1a;
        gpufhe::ct_add_ct_host(q0, q1, c0b, c1b, sizeQ - 1, n, mod);
        const size_t F = (size_t)(sizeQ - 1) * n;
        gate(std::equal(q0.begin(), q0.begin() + F, pa0.begin()) && std::equal(q0.begin() + F, q0.end(), c0a.begin() + F) &&
             std::equal(q1.begin(), q1.begin() + F, pa1.begin()) && q1.size() == T,
             "ct_add_ct_host over fewer towers leaves the rest");
    }

    // canonical encode / decode as the reference's tests call them
    // (test_alpha10.cpp:52-82): seeded slots at scale 2^40
    std::vector<int64_t> em;
    std::vector<std::complex<double>> ez(n / 2), dz;
    {
        std::mt19937_64 zr(11);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        for (auto& v : ez) {
            const double re = u(zr);
            v = {re, u(zr)};
        }
        gpufhe::encode_host(em, ez, n, 1099511627776.0);
        gpufhe::decode_host(dz, em, n, 1099511627776.0);
        double err = 0;
        for (uint32_t k = 0; k < n / 2; ++k) err = std::max(err, std::abs(dz[k] - ez[k]));
        gate(em.size() == n && dz.size() == n / 2 && err < 1e-6, "encode_host / decode_host round trip");
    }

    if (argc > 1) {
        FILE* f = std::fopen(argv[1], "wb");
        std::fwrite(h0.data(), 8, (size_t)(sizeQ - 1) * n, f);
        std::fwrite(h1.data(), 8, (size_t)(sizeQ - 1) * n, f);
        std::fwrite(ks0.data(), 8, T, f);
        std::fwrite(ks1.data(), 8, T, f);
        std::fwrite(ez.data(), 16, n / 2, f);
        std::fwrite(em.data(), 8, n, f);
        std::fwrite(dz.data(), 16, n / 2, f);
        for (const auto* v : {&sH, &g0, &g1, &pe, &pm0, &pm1, &pa0, &pa1}) std::fwrite(v->data(), 8, v->size(), f);
        std::fclose(f);
    }
    gpufhe::ks_work_destroy(W);
    gpufhe::ks_context_destroy(C);
    std::printf("%s\n", fails ? "[FAIL]" : "[PASS] C++ API gates");
    return fails ? 1 : 0;
}
