/*
 * CPU oracle for the resident leveled-CKKS hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the reference result for tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py. It is a scalar restatement of the
 * reference's formulas (samfrazerdutton/GPU-Resident-Library); each function
 * names the reference file:line it follows. No CUDA, no product code.
 *
 * Parity pin: the constants and parameter routines are checked against the
 * reference's own host sources compiled by oracle/build_ref.sh, and the
 * composed path is checked against golden vectors produced by the reference
 * library rebuilt for sm_100a (tests/golden/make_golden.py).
 */
#include "ckks_oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <random>
#include <stdexcept>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;
typedef unsigned __int128 u128;
typedef std::vector<u64> vec;

namespace {

inline u64 mulmod(u64 a, u64 b, u64 q) { return (u64)(((u128)a * b) % q); }
inline u64 addmod(u64 a, u64 b, u64 q) { u64 s = a + b; return s >= q ? s - q : s; }
inline u64 submod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + q - b; }
u64 powmod(u64 b, u64 e, u64 q) {
    u128 r = 1, bb = b % q;
    while (e) { if (e & 1) r = (r * bb) % q; bb = (bb * bb) % q; e >>= 1; }
    return (u64)r;
}
u64 invmod(u64 a, u64 q) { return powmod(a % q, q - 2, q); }
/* floor(w * 2^64 / q), the Shoup precomputation (ks_constants.cpp:19). */
inline u64 precon(u64 w, u64 q) { return (u64)(((u128)w << 64) / q); }
/* Shoup multiply, one correction (ntt_ct.cu:11-16). */
inline u64 shoup(u64 x, u64 w, u64 wp, u64 q) {
    u64 hi = (u64)(((u128)x * wp) >> 64);
    u64 r = x * w - hi * q;
    return r >= q ? r - q : r;
}
inline uint32_t bitrev(uint32_t v, uint32_t b) {
    uint32_t r = 0;
    for (uint32_t k = 0; k < b; k++) { r = (r << 1) | (v & 1); v >>= 1; }
    return r;
}
inline uint32_t ilog2(uint32_t n) { uint32_t l = 0; while ((1u << l) < n) ++l; return l; }

/* Reference-equivalent centered embedding of a small signed integer. */
inline u64 emb(long v, u64 q) { return (u64)((v % (long)q + (long)q) % (long)q); }

bool is_prime(u64 x) {  /* params.cpp:17-25 */
    if (x < 2) return false;
    static const u64 bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (u64 a : bases) if (x % a == 0) return x == a;
    u64 d = x - 1; int s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    for (u64 a : bases) {
        u64 v = powmod(a, d, x);
        if (v == 1 || v == x - 1) continue;
        bool ok = false;
        for (int i = 1; i < s; ++i) { v = mulmod(v, v, x); if (v == x - 1) { ok = true; break; } }
        if (!ok) return false;
    }
    return true;
}

/* overflow-safe mulmod for moduli up to 2^127 (params.cpp:12-15). */
u128 mulmod128(u128 a, u128 b, u128 m) {
    a %= m; u128 r = 0;
    while (b) { if (b & 1) { r += a; if (r >= m) r -= m; } a <<= 1; if (a >= m) a -= m; b >>= 1; }
    return r;
}

struct Tables { vec fr, fp, ir, ip; u64 ninv, ninvp; };

void build_tables(uint32_t n, u64 q, u64 root, Tables& T) {
    /* keyswitch_resident.cpp:53-62: fr[i] = root^bitrev(i), fp = precon */
    uint32_t logn = ilog2(n);
    u64 rinv = invmod(root, q);
    vec pw(n);
    T.fr.resize(n); T.fp.resize(n); T.ir.resize(n); T.ip.resize(n);
    auto fill = [&](u64 base, vec& tr, vec& tp) {
        pw[0] = 1;
        for (uint32_t i = 1; i < n; ++i) pw[i] = mulmod(pw[i - 1], base, q);
        for (uint32_t i = 0; i < n; ++i) { u64 r = pw[bitrev(i, logn)]; tr[i] = r; tp[i] = precon(r, q); }
    };
    fill(root, T.fr, T.fp);
    fill(rinv, T.ir, T.ip);
    T.ninv = invmod(n, q);
    T.ninvp = precon(T.ninv, q);
}

/* Forward CT, standard in -> bit-reversed out (ntt_ct.cu:19-39 per stage and
 * the shared tail ntt_ct.cu:47-88 compute this same loop nest). */
void ntt(u64* x, const u64* fr, const u64* fp, uint32_t n, u64 q) {
    for (uint32_t m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1) {
        for (uint32_t i = 0; i < m; ++i) {
            const u64 w = fr[m + i], wp = fp[m + i];
            const uint32_t j1 = 2 * i * t;
            for (uint32_t j = j1; j < j1 + t; ++j) {
                u64 of = shoup(x[j + t], w, wp, q);
                u64 lo = x[j];
                u64 hi = lo + of; if (hi >= q) hi -= q;
                u64 lv = lo; if (lv < of) lv += q; lv -= of;
                x[j] = hi; x[j + t] = lv;
            }
        }
    }
}

/* Inverse GS, bit-reversed in -> standard out, then x*n^-1 (intt_ct.cu:21-42,
 * 47-84 and the separate scale pass 86-90). */
void intt(u64* x, const u64* ir, const u64* ip, uint32_t n, u64 q, u64 ninv, u64 ninvp) {
    for (uint32_t m = n >> 1, t = 1; m >= 1; m >>= 1, t <<= 1) {
        for (uint32_t i = 0; i < m; ++i) {
            const u64 w = ir[m + i], wp = ip[m + i];
            const uint32_t j1 = 2 * i * t;
            for (uint32_t j = j1; j < j1 + t; ++j) {
                u64 lo = x[j], hi = x[j + t];
                u64 sum = lo + hi; if (sum >= q) sum -= q;
                u64 dif = lo; if (dif < hi) dif += q; dif -= hi;
                x[j] = sum; x[j + t] = shoup(dif, w, wp, q);
            }
        }
        if (m == 1) break;
    }
    for (uint32_t k = 0; k < n; ++k) x[k] = shoup(x[k], ninv, ninvp, q);
}

/* basis_convert.cu:24-55 restated: floor(a*mu/2^128) from partial products,
 * then a_lo - qhat*m with a correction loop. Exact for every input. */
u64 barrett_u128(u128 a, u64 modulus, u128 mu) {
    u64 a_lo = (u64)a, a_hi = (u64)(a >> 64);
    u64 mu_lo = (u64)mu, mu_hi = (u64)(mu >> 64);
    u64 left_hi = (u64)(((u128)a_lo * mu_lo) >> 64);
    u128 mid1 = (u128)a_lo * mu_hi;
    u128 s1 = (u128)(u64)mid1 + left_hi;
    u64 tmp1 = (u64)s1, carry = (u64)(s1 >> 64);
    u64 tmp2 = (u64)(mid1 >> 64) + carry;
    u128 mid2 = (u128)a_hi * mu_lo;
    u128 s2 = (u128)(u64)mid2 + tmp1;
    carry = (u64)(s2 >> 64);
    u64 left_hi2 = (u64)(mid2 >> 64) + carry;
    u64 qhat = a_hi * mu_hi + tmp2 + left_hi2;
    u64 result = a_lo - qhat * modulus;
    while (result >= modulus) result -= modulus;
    return result;
}

/* approx_switch_kernel (basis_convert.cu:61-101), per coefficient. */
void approx_switch(const u64* src, u64* dst, const u64* QHatInv, const u64* QHatInvPrec,
                   const u64* q, const u64* QHatModp, const u64* p, const u64* mulo,
                   const u64* muhi, uint32_t sizeQ, uint32_t sizeP, uint32_t n) {
    std::vector<u64> x(sizeQ);
    for (uint32_t ri = 0; ri < n; ++ri) {
        for (uint32_t i = 0; i < sizeQ; ++i)
            x[i] = shoup(src[(size_t)i * n + ri], QHatInv[i], QHatInvPrec[i], q[i]);
        for (uint32_t j = 0; j < sizeP; ++j) {
            u128 sum = 0;
            for (uint32_t i = 0; i < sizeQ; ++i) sum += (u128)x[i] * QHatModp[(size_t)i * sizeP + j];
            u128 mu = ((u128)muhi[j] << 64) | mulo[j];
            dst[(size_t)j * n + ri] = barrett_u128(sum, p[j], mu);
        }
    }
}

/* ---- keyswitch constants with an explicit partition ----
 * ks_constants.cpp:31-102 derives alpha = ceil(sizeQ/numPart); here alpha is
 * given so one full-QP key serves every level with the same digit boundaries
 * (keyswitch_resident.cpp:91-96 indexing, test_keyreuse.cpp:6-7). When
 * ceil(L/ceil(L/alpha)) == alpha the two derivations coincide exactly. */
struct Part {
    uint32_t start, size;
    vec qhatinv, qhatinvp, src, qhatmodp, compl_, mulo, muhi;
};
struct KSConst {
    uint32_t L, K, alpha, nparts;
    std::vector<Part> parts;
    vec phatinv, phatinvp, phatmodq, mdmulo, mdmuhi, pinvmodq;
};

u64 prod_mod(const u64* mods, uint32_t cnt, u64 q, int skip) {  /* ks_constants.cpp:22-26 */
    u64 r = 1 % q;
    for (uint32_t k = 0; k < cnt; ++k) { if ((int)k == skip) continue; r = mulmod(r, mods[k] % q, q); }
    return r;
}

void ks_constants(KSConst& C, const u64* Q, uint32_t L, const u64* P, uint32_t K, uint32_t alpha) {
    C.L = L; C.K = K; C.alpha = alpha;
    C.nparts = (L + alpha - 1) / alpha;
    /* ModDown family, ks_constants.cpp:45-63 */
    C.pinvmodq.resize(L);
    for (uint32_t i = 0; i < L; ++i) C.pinvmodq[i] = invmod(prod_mod(P, K, Q[i], -1), Q[i]);
    C.phatinv.resize(K); C.phatinvp.resize(K); C.phatmodq.resize((size_t)K * L);
    for (uint32_t j = 0; j < K; ++j) {
        C.phatinv[j] = invmod(prod_mod(P, K, P[j], (int)j), P[j]);
        C.phatinvp[j] = precon(C.phatinv[j], P[j]);
        for (uint32_t i = 0; i < L; ++i) C.phatmodq[(size_t)j * L + i] = prod_mod(P, K, Q[i], (int)j);
    }
    C.mdmulo.resize(L); C.mdmuhi.resize(L);
    for (uint32_t i = 0; i < L; ++i) {
        u128 mu = (~(u128)0) / Q[i];
        C.mdmulo[i] = (u64)mu; C.mdmuhi[i] = (u64)(mu >> 64);
    }
    /* decompose family, ks_constants.cpp:65-101 */
    C.parts.resize(C.nparts);
    for (uint32_t p = 0; p < C.nparts; ++p) {
        Part& pt = C.parts[p];
        pt.start = alpha * p;
        pt.size = (L > pt.start + alpha) ? alpha : (L - pt.start);
        pt.src.assign(Q + pt.start, Q + pt.start + pt.size);
        pt.qhatinv.resize(pt.size); pt.qhatinvp.resize(pt.size);
        for (uint32_t i = 0; i < pt.size; ++i) {
            u64 q = pt.src[i];
            pt.qhatinv[i] = invmod(prod_mod(pt.src.data(), pt.size, q, (int)i), q);
            pt.qhatinvp[i] = precon(pt.qhatinv[i], q);
        }
        pt.compl_.clear();
        for (uint32_t i = 0; i < L; ++i)
            if (i < pt.start || i >= pt.start + pt.size) pt.compl_.push_back(Q[i]);
        for (uint32_t j = 0; j < K; ++j) pt.compl_.push_back(P[j]);
        uint32_t sc = (uint32_t)pt.compl_.size();
        pt.qhatmodp.resize((size_t)pt.size * sc);
        for (uint32_t i = 0; i < pt.size; ++i)
            for (uint32_t j = 0; j < sc; ++j)
                pt.qhatmodp[(size_t)i * sc + j] = prod_mod(pt.src.data(), pt.size, pt.compl_[j], (int)i);
        pt.mulo.resize(sc); pt.muhi.resize(sc);
        for (uint32_t j = 0; j < sc; ++j) {
            u128 mu = (~(u128)0) / pt.compl_[j];
            pt.mulo[j] = (u64)mu; pt.muhi[j] = (u64)(mu >> 64);
        }
    }
}

}  // namespace

/* ===================== oracle context ===================== */
struct OrcCtx {
    uint32_t n, fullQ, K, alpha, dnum;
    vec Q, P, QP, roots;          /* roots parallel to QP */
    std::vector<Tables> tab;      /* parallel to QP */
    std::vector<KSConst> ks;      /* index L (1..fullQ) */
    std::vector<vec> key_av, key_bv;   /* per key id: [dnum][fullQ+K][n] */
    const Tables& T(uint32_t qp_index) const { return tab[qp_index]; }
};

namespace {
uint32_t g_hw = 0;  /* keygen.cpp:18, 53: 0 = uniform ternary */

void intt_one(const OrcCtx* c, u64* v, uint32_t qp) {
    const Tables& T = c->T(qp);
    intt(v, T.ir.data(), T.ip.data(), c->n, c->QP[qp], T.ninv, T.ninvp);
}
void ntt_one(const OrcCtx* c, u64* v, uint32_t qp) {
    const Tables& T = c->T(qp);
    ntt(v, T.fr.data(), T.fp.data(), c->n, c->QP[qp]);
}
/* QP index of the modulus at position i of the level-L QlP order. */
inline uint32_t qlp_index(const OrcCtx* c, uint32_t L, uint32_t i) {
    return i < L ? i : c->fullQ + (i - L);
}

/* Hybrid ModUp of a (eval, L towers) into digits over QlP, eval form
 * (keyswitch_resident.cpp:149-200; keyswitch.cpp:73-118). */
void modup(const OrcCtx* c, uint32_t L, const u64* a, std::vector<vec>& digits) {
    const uint32_t n = c->n, K = c->K, QlP = L + K;
    const KSConst& C = c->ks[L];
    digits.assign(C.nparts, vec());
    for (uint32_t p = 0; p < C.nparts; ++p) {
        const Part& pt = C.parts[p];
        const uint32_t sp = pt.size, st = pt.start, en = st + sp, sc = (uint32_t)pt.compl_.size();
        vec part(a + (size_t)st * n, a + (size_t)en * n);
        for (uint32_t i = 0; i < sp; ++i) intt_one(c, part.data() + (size_t)i * n, st + i);
        vec compl_((size_t)sc * n);
        approx_switch(part.data(), compl_.data(), pt.qhatinv.data(), pt.qhatinvp.data(),
                      pt.src.data(), pt.qhatmodp.data(), pt.compl_.data(), pt.mulo.data(),
                      pt.muhi.data(), sp, sc, n);
        /* complement order: Q towers outside the part, then P (ks_constants.cpp:85-90) */
        for (uint32_t j = 0; j < sc; ++j) {
            uint32_t qi = (j < st) ? j : (j < L - sp ? j + sp : c->fullQ + (j - (L - sp)));
            ntt_one(c, compl_.data() + (size_t)j * n, qi);
        }
        vec& d = digits[p];
        d.resize((size_t)QlP * n);
        for (uint32_t i = 0; i < QlP; ++i) {
            const u64* srcp = (i >= st && i < en) ? a + (size_t)i * n
                            : (i < st) ? compl_.data() + (size_t)i * n
                                       : compl_.data() + (size_t)(i - sp) * n;
            std::memcpy(d.data() + (size_t)i * n, srcp, (size_t)n * 8);
        }
    }
}

/* ks_macc_batched over digits (ks_fastcore.cu:49-69) with keyRow
 * (keyswitch_resident.cpp:91-96): res[i] = sum_p digit_p[i] * key_p[row(i)]. */
void inner_product(const OrcCtx* c, uint32_t key_id, uint32_t L, const std::vector<vec>& digits,
                   vec& res0, vec& res1) {
    const uint32_t n = c->n, K = c->K, QlP = L + K, ET = c->fullQ + K;
    const uint32_t delta = c->fullQ - L;
    res0.assign((size_t)QlP * n, 0); res1.assign((size_t)QlP * n, 0);
    const vec& AV = c->key_av[key_id];
    const vec& BV = c->key_bv[key_id];
    for (uint32_t p = 0; p < digits.size(); ++p) {
        for (uint32_t i = 0; i < QlP; ++i) {
            const u64 q = c->QP[qlp_index(c, L, i)];
            const uint32_t row = (i >= L) ? i + delta : i;
            const u64* bv = BV.data() + ((size_t)p * ET + row) * n;
            const u64* av = AV.data() + ((size_t)p * ET + row) * n;
            const u64* dg = digits[p].data() + (size_t)i * n;
            u64* o0 = res0.data() + (size_t)i * n;
            u64* o1 = res1.data() + (size_t)i * n;
            for (uint32_t k = 0; k < n; ++k) {
                o0[k] = addmod(o0[k], mulmod(dg[k], bv[k], q), q);
                o1[k] = addmod(o1[k], mulmod(dg[k], av[k], q), q);
            }
        }
    }
}

/* ApproxModDown QlP -> Q (keyswitch_resident.cpp:203-224; moddown.cu:10-22). */
void moddown(const OrcCtx* c, uint32_t L, const vec& res, u64* out) {
    const uint32_t n = c->n, K = c->K;
    const KSConst& C = c->ks[L];
    vec pw(res.begin() + (size_t)L * n, res.begin() + (size_t)(L + K) * n);
    for (uint32_t j = 0; j < K; ++j) intt_one(c, pw.data() + (size_t)j * n, c->fullQ + j);
    vec qsw((size_t)L * n);
    approx_switch(pw.data(), qsw.data(), C.phatinv.data(), C.phatinvp.data(), c->P.data(),
                  C.phatmodq.data(), c->Q.data(), C.mdmulo.data(), C.mdmuhi.data(), K, L, n);
    for (uint32_t i = 0; i < L; ++i) {
        ntt_one(c, qsw.data() + (size_t)i * n, i);
        const u64 q = c->Q[i], s = C.pinvmodq[i];
        for (uint32_t k = 0; k < n; ++k) {
            u64 diff = res[(size_t)i * n + k];
            u64 b = qsw[(size_t)i * n + k];
            if (diff < b) diff += q;
            diff -= b;
            out[(size_t)i * n + k] = mulmod(diff, s, q);
        }
    }
}

/* SwitchModulus (switch_modulus.cu:11-42). */
void switch_modulus(u64* v, u64 q_old, u64 q_new, uint32_t n) {
    u64 half = q_old >> 1;
    u64 diff = q_old > q_new ? q_old - q_new : q_new - q_old;
    bool larger = q_new > q_old;
    if (!larger) diff %= q_new;
    for (uint32_t i = 0; i < n; ++i) {
        u64 x = v[i];
        u64 d = x > half ? diff : 0;
        if (larger) v[i] = x + d;
        else { u64 xm = x >= q_new ? x % q_new : x; v[i] = xm >= d ? xm - d : xm + q_new - d; }
    }
}

/* sigma_k on a coefficient-form tower (automorph.cu:9-20). */
void automorph(u64* out, const u64* in, uint32_t n, u64 k, u64 q) {
    const u64 M = 2ull * n;
    for (uint32_t j = 0; j < n; ++j) {
        u64 idx = ((u64)j * k) % M;
        u64 v = in[j];
        if (idx < n) out[idx] = v; else out[idx - n] = v ? q - v : 0;
    }
}

void rescale_comp(const OrcCtx* c, uint32_t L, u64* comp, const vec& s1, const vec& s2) {
    /* rescale_resident_raw (keyswitch_resident.cpp:227-244) */
    const uint32_t n = c->n;
    if (L < 2) return;
    const uint32_t last = L - 1;
    const u64 ql = c->Q[last];
    vec drop(comp + (size_t)last * n, comp + (size_t)L * n);
    intt_one(c, drop.data(), last);
    vec sc(n);
    for (uint32_t t = 0; t < last; ++t) {
        const u64 qi = c->Q[t];
        sc = drop;
        switch_modulus(sc.data(), ql, qi, n);
        ntt_one(c, sc.data(), t);
        u64* a = comp + (size_t)t * n;
        for (uint32_t k = 0; k < n; ++k) {   /* rescale.cu:10-21 */
            u64 t1 = mulmod(a[k], s1[t], qi), t2 = mulmod(sc[k], s2[t], qi);
            u64 s = t1 + t2;
            a[k] = s >= qi ? s - qi : s;
        }
    }
}

void rescale_consts(vec& s1, vec& s2, const u64* mod, uint32_t last) {
    /* params.cpp:54-75 */
    u64 ql = mod[last];
    s1.resize(last); s2.resize(last);
    u64 QlModql = 1 % ql;
    for (uint32_t t = 0; t < last; ++t) QlModql = mulmod(QlModql, mod[t] % ql, ql);
    u64 u = powmod(QlModql, ql - 2, ql);
    for (uint32_t i = 0; i < last; ++i) {
        u64 qi = mod[i];
        s1[i] = powmod(ql % qi, qi - 2, qi);
        u128 mod2 = (u128)ql * qi;
        u128 Ql2 = 1 % mod2;
        for (uint32_t t = 0; t < last; ++t) Ql2 = mulmod128(Ql2, mod[t], mod2);
        u128 prod = mulmod128(Ql2, u, mod2);
        u128 pm1 = (prod == 0) ? mod2 - 1 : prod - 1;
        s2[i] = (u64)((pm1 / ql) % qi);
    }
}

void evalmult_rescale_one(const OrcCtx* c, uint32_t L, const u64* c0a, const u64* c1a,
                          const u64* c0b, const u64* c1b, u64* out0, u64* out1) {
    const uint32_t n = c->n;
    const size_t T = (size_t)L * n;
    vec t0(T), t1(T), t2(T);
    orc_tensor(c0a, c1a, c0b, c1b, t0.data(), t1.data(), t2.data(), c->Q.data(), L, n);
    vec ba0(T), ba1(T);
    orc_keyswitch(c, 0, L, t2.data(), ba0.data(), ba1.data());
    vec r0(T), r1(T);
    orc_combine(r0.data(), r1.data(), t0.data(), t1.data(), ba0.data(), ba1.data(), c->Q.data(), L, n);
    vec s1, s2;
    rescale_consts(s1, s2, c->Q.data(), L - 1);
    rescale_comp(c, L, r0.data(), s1, s2);
    rescale_comp(c, L, r1.data(), s1, s2);
    std::memcpy(out0, r0.data(), (size_t)(L - 1) * n * 8);
    std::memcpy(out1, r1.data(), (size_t)(L - 1) * n * 8);
}
}  // namespace

extern "C" {

int orc_native_primes(u64* out, uint32_t count, uint32_t bits, uint32_t n, const u64* avoid,
                      uint32_t navoid) {
    /* params.cpp:29-39 */
    const u64 M = 2ull * n;
    u64 q = ((1ull << bits) / M) * M + 1;
    uint32_t got = 0;
    while (got < count) {
        if (q < (1ull << (bits - 1))) return -1;
        bool skip = false;
        for (uint32_t a = 0; a < navoid; ++a) if (avoid[a] == q) skip = true;
        if (!skip && is_prime(q)) out[got++] = q;
        q -= M;
    }
    return 0;
}

u64 orc_native_root(uint32_t n, u64 q) {
    /* params.cpp:42-48 */
    const u64 M = 2ull * n;
    for (u64 g = 2; g < q; ++g) {
        u64 c = powmod(g, (q - 1) / M, q);
        if (powmod(c, n, q) == q - 1) return c;
    }
    return 0;
}

void orc_rescale_consts(u64* s1, u64* s2, const u64* mod, uint32_t last) {
    vec a, b;
    rescale_consts(a, b, mod, last);
    std::memcpy(s1, a.data(), last * 8);
    std::memcpy(s2, b.data(), last * 8);
}

void orc_root_tables(uint32_t n, u64 q, u64 root, u64* fr, u64* fp, u64* ir, u64* ip, u64* ninv) {
    Tables T;
    build_tables(n, q, root, T);
    std::memcpy(fr, T.fr.data(), n * 8); std::memcpy(fp, T.fp.data(), n * 8);
    std::memcpy(ir, T.ir.data(), n * 8); std::memcpy(ip, T.ip.data(), n * 8);
    ninv[0] = T.ninv; ninv[1] = T.ninvp;
}

void orc_ntt(u64* x, const u64* fr, const u64* fp, uint32_t n, u64 q) { ntt(x, fr, fp, n, q); }
void orc_intt(u64* x, const u64* ir, const u64* ip, uint32_t n, u64 q, u64 ninv, u64 ninvp) {
    intt(x, ir, ip, n, q, ninv, ninvp);
}

void orc_rns_mult(const u64* a, const u64* b, u64* r, u64 q, uint32_t n) {
    /* rns_arith.cu:21-33: Montgomery twice == plain a*b mod q */
    for (uint32_t i = 0; i < n; ++i) r[i] = mulmod(a[i], b[i], q);
}

void orc_tensor(const u64* c0a, const u64* c1a, const u64* c0b, const u64* c1b, u64* t0, u64* t1,
                u64* t2, const u64* mods, uint32_t sizeQ, uint32_t n) {
    /* tensor.cu:11-27 */
    for (uint32_t t = 0; t < sizeQ; ++t) {
        const u64 q = mods[t];
        for (uint32_t k = 0; k < n; ++k) {
            size_t x = (size_t)t * n + k;
            t0[x] = mulmod(c0a[x], c0b[x], q);
            u64 s = mulmod(c0a[x], c1b[x], q) + mulmod(c1a[x], c0b[x], q);
            t1[x] = s >= q ? s - q : s;
            t2[x] = mulmod(c1a[x], c1b[x], q);
        }
    }
}

void orc_combine(u64* r0, u64* r1, const u64* t0, const u64* t1, const u64* ba0, const u64* ba1,
                 const u64* mods, uint32_t sizeQ, uint32_t n) {
    /* tensor.cu:39-52 */
    for (uint32_t t = 0; t < sizeQ; ++t) {
        const u64 q = mods[t];
        for (uint32_t k = 0; k < n; ++k) {
            size_t x = (size_t)t * n + k;
            u64 a = t0[x] + ba0[x]; r0[x] = a >= q ? a - q : a;
            u64 b = t1[x] + ba1[x]; r1[x] = b >= q ? b - q : b;
        }
    }
}

void orc_switch_modulus(u64* v, u64 q_old, u64 q_new, uint32_t n) { switch_modulus(v, q_old, q_new, n); }

void orc_rescale_fuse(u64* a, const u64* b, u64 s1, u64 s2, u64 q, uint32_t n) {
    for (uint32_t k = 0; k < n; ++k) {
        u64 t1 = mulmod(a[k], s1, q), t2 = mulmod(b[k], s2, q);
        u64 s = t1 + t2;
        a[k] = s >= q ? s - q : s;
    }
}

u64 orc_barrett_u128(u64 a_lo, u64 a_hi, u64 modulus, u64 mu_lo, u64 mu_hi) {
    return barrett_u128(((u128)a_hi << 64) | a_lo, modulus, ((u128)mu_hi << 64) | mu_lo);
}

void orc_approx_switch(const u64* src, u64* dst, const u64* QHatInv, const u64* QHatInvPrec,
                       const u64* q, const u64* QHatModp, const u64* p, const u64* mu_lo,
                       const u64* mu_hi, uint32_t sizeQ, uint32_t sizeP, uint32_t n) {
    approx_switch(src, dst, QHatInv, QHatInvPrec, q, QHatModp, p, mu_lo, mu_hi, sizeQ, sizeP, n);
}

void orc_ks_macc(u64* out0, u64* out1, const u64* digit, const u64* b, const u64* a, u64 q,
                 uint32_t n) {
    /* ks_fastcore.cu:18-31 */
    for (uint32_t k = 0; k < n; ++k) {
        u64 d = digit[k];
        u64 t0 = out0[k] + mulmod(d, b[k], q); if (t0 >= q) t0 -= q;
        u64 t1 = out1[k] + mulmod(d, a[k], q); if (t1 >= q) t1 -= q;
        out0[k] = t0; out1[k] = t1;
    }
}

void orc_moddown_combine(u64* ans, const u64* a, const u64* b, u64 s, u64 q, uint32_t n) {
    for (uint32_t k = 0; k < n; ++k) {   /* moddown.cu:10-22 */
        u64 diff = a[k];
        if (diff < b[k]) diff += q;
        diff -= b[k];
        ans[k] = mulmod(diff, s, q);
    }
}

void orc_automorph(u64* out, const u64* in, uint32_t n, u64 k, u64 q) { automorph(out, in, n, k, q); }

void orc_add_into(u64* a, const u64* b, u64 q, uint32_t n) {
    for (uint32_t k = 0; k < n; ++k) { u64 s = a[k] + b[k]; a[k] = s >= q ? s - q : s; }
}

void orc_ptmulacc(u64* acc0, u64* acc1, const u64* b0, const u64* b1, const u64* d, u64 q,
                  uint32_t n) {
    for (uint32_t k = 0; k < n; ++k) {   /* stage_acc.cu:12-28 */
        u64 p0 = mulmod(b0[k], d[k], q), p1 = mulmod(b1[k], d[k], q);
        u64 s0 = acc0[k] + p0; if (s0 >= q) s0 -= q;
        u64 s1 = acc1[k] + p1; if (s1 >= q) s1 -= q;
        acc0[k] = s0; acc1[k] = s1;
    }
}

u64 orc_ks_constants_size(uint32_t L, uint32_t K, uint32_t alpha) {
    u64 total = 0;
    uint32_t np = (L + alpha - 1) / alpha;
    for (uint32_t p = 0; p < np; ++p) {
        uint32_t st = alpha * p, sp = (L > st + alpha) ? alpha : L - st, sc = L - sp + K;
        total += 3ull * sp + (u64)sp * sc + 3ull * sc;
    }
    total += 2ull * K + (u64)K * L + 3ull * L;
    return total;
}

void orc_ks_constants(u64* out, const u64* Q, uint32_t L, const u64* P, uint32_t K, uint32_t alpha) {
    KSConst C;
    ks_constants(C, Q, L, P, K, alpha);
    u64* o = out;
    auto put = [&](const vec& v) { std::memcpy(o, v.data(), v.size() * 8); o += v.size(); };
    for (auto& pt : C.parts) {
        put(pt.qhatinv); put(pt.qhatinvp); put(pt.src); put(pt.qhatmodp);
        put(pt.compl_); put(pt.mulo); put(pt.muhi);
    }
    put(C.phatinv); put(C.phatinvp); put(C.phatmodq); put(C.mdmulo); put(C.mdmuhi); put(C.pinvmodq);
}

OrcCtx* orc_ctx_create(uint32_t n, const u64* modQ, uint32_t fullQ, const u64* modP, uint32_t sizeP,
                       uint32_t alpha, const u64* rootsQP) {
    OrcCtx* c = new OrcCtx();
    c->n = n; c->fullQ = fullQ; c->K = sizeP; c->alpha = alpha;
    c->dnum = (fullQ + alpha - 1) / alpha;
    c->Q.assign(modQ, modQ + fullQ);
    c->P.assign(modP, modP + sizeP);
    c->QP = c->Q; c->QP.insert(c->QP.end(), c->P.begin(), c->P.end());
    const uint32_t QP = fullQ + sizeP;
    c->roots.resize(QP);
    for (uint32_t i = 0; i < QP; ++i) c->roots[i] = rootsQP ? rootsQP[i] : orc_native_root(n, c->QP[i]);
    c->tab.resize(QP);
    for (uint32_t i = 0; i < QP; ++i) build_tables(n, c->QP[i], c->roots[i], c->tab[i]);
    c->ks.resize(fullQ + 1);
    for (uint32_t L = 1; L <= fullQ; ++L) ks_constants(c->ks[L], c->Q.data(), L, c->P.data(), sizeP, alpha);
    return c;
}

void orc_ctx_destroy(OrcCtx* c) { delete c; }

void orc_ctx_roots(const OrcCtx* c, u64* r) { std::memcpy(r, c->roots.data(), c->roots.size() * 8); }

int orc_ctx_set_key(OrcCtx* c, uint32_t key_id, const u64* av, const u64* bv) {
    if (key_id >= c->key_av.size()) { c->key_av.resize(key_id + 1); c->key_bv.resize(key_id + 1); }
    size_t words = (size_t)c->dnum * (c->fullQ + c->K) * c->n;
    c->key_av[key_id].assign(av, av + words);
    c->key_bv[key_id].assign(bv, bv + words);
    return 0;
}

void orc_set_hamming_weight(uint32_t h) { g_hw = h; }

void orc_keygen(const OrcCtx* c, uint32_t towers, u64 ns, double sigma, u64 seed, u64* s, u64* pkA,
                u64* pkB) {
    /* keygen.cpp:55-112: same mt19937_64 draw order */
    const uint32_t n = c->n;
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, sigma);
    std::vector<int> sc(n), ec(n);
    if (g_hw == 0) {
        for (uint32_t k = 0; k < n; ++k) { int r = (int)(rng() % 3); sc[k] = r - 1; }
    } else {
        std::vector<uint32_t> idx(n);
        for (uint32_t k = 0; k < n; ++k) idx[k] = k;
        for (uint32_t k = n - 1; k > 0; --k) { uint32_t j = (uint32_t)(rng() % (k + 1)); std::swap(idx[k], idx[j]); }
        uint32_t h = g_hw < n ? g_hw : n;
        for (uint32_t k = 0; k < h; ++k) sc[idx[k]] = (rng() & 1ull) ? 1 : -1;
    }
    for (uint32_t k = 0; k < n; ++k) { long e = std::lround(gauss(rng)); ec[k] = (int)e; }
    /* tower t uses modulus QP[t]: the first `towers` moduli of Q||P, as the
     * reference passes moduli = mod (Q key) or modQP (QP key). */
    for (uint32_t t = 0; t < towers; ++t) {
        const uint32_t qp = t;
        const u64 qq = c->QP[qp];
        vec sT(n), eT(n), aT(n);
        for (uint32_t k = 0; k < n; ++k) {
            sT[k] = emb(sc[k], qq); eT[k] = emb(ec[k], qq);
            aT[k] = rng() % qq;
        }
        ntt_one(c, sT.data(), qp);
        ntt_one(c, eT.data(), qp);
        for (uint32_t k = 0; k < n; ++k) {
            u64 as = mulmod(aT[k], sT[k], qq);
            u64 nse = mulmod(ns % qq, eT[k], qq);
            size_t x = (size_t)t * n + k;
            s[x] = sT[k]; pkA[x] = aT[k]; pkB[x] = submod(nse, as, qq);
        }
    }
}

void orc_evalkeygen(const OrcCtx* c, const u64* sQP, const u64* sOld, const u64* pkA_QP,
                    const u64* pkB_QP, u64 ns, double sigma, u64 seed, u64* av, u64* bv) {
    /* evalkeygen.cpp:42-96 at sizeQl = fullQ, sizeQlP = fullQ + K */
    (void)sQP;
    const uint32_t n = c->n, QlP = c->fullQ + c->K, Ql = c->fullQ;
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, sigma);
    vec PModq(QlP);
    for (uint32_t t = 0; t < QlP; ++t) PModq[t] = prod_mod(c->P.data(), c->K, c->QP[t], -1);
    for (uint32_t part = 0; part < c->dnum; ++part) {
        uint32_t st = c->alpha * part;
        uint32_t sp = (Ql > st + c->alpha) ? c->alpha : (Ql - st);
        uint32_t en = st + sp;
        std::vector<int> uc(n), e0c(n), e1c(n);
        for (uint32_t k = 0; k < n; ++k) {
            uc[k] = (int)(rng() % 3) - 1;
            e0c[k] = (int)std::lround(gauss(rng));
            e1c[k] = (int)std::lround(gauss(rng));
        }
        for (uint32_t t = 0; t < QlP; ++t) {
            const u64 q = c->QP[t];
            vec uT(n), e0T(n), e1T(n);
            for (uint32_t k = 0; k < n; ++k) { uT[k] = emb(uc[k], q); e0T[k] = emb(e0c[k], q); e1T[k] = emb(e1c[k], q); }
            ntt_one(c, uT.data(), t); ntt_one(c, e0T.data(), t); ntt_one(c, e1T.data(), t);
            for (uint32_t k = 0; k < n; ++k) {
                size_t x = (size_t)t * n + k;
                u64 p1u = mulmod(pkA_QP[x], uT[k], q);
                u64 p0u = mulmod(pkB_QP[x], uT[k], q);
                u64 a = addmod(p1u, mulmod(ns % q, e1T[k], q), q);
                u64 b = addmod(p0u, mulmod(ns % q, e0T[k], q), q);
                if (t >= st && t < en) b = addmod(b, mulmod(PModq[t] % q, sOld[x], q), q);
                av[((size_t)part * QlP) * n + x] = a;
                bv[((size_t)part * QlP) * n + x] = b;
            }
        }
    }
}

void orc_encrypt(const OrcCtx* c, uint32_t towers, const int64_t* m, const u64* pkA, const u64* pkB,
                 u64 ns, double sigma, u64 seed, u64* c0, u64* c1) {
    /* encdec.cpp:41-64 */
    const uint32_t n = c->n;
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> g(0.0, sigma);
    std::vector<int> vc(n), e0c(n), e1c(n);
    for (uint32_t k = 0; k < n; ++k) {
        vc[k] = (int)(rng() % 3) - 1;
        e0c[k] = (int)std::lround(g(rng));
        e1c[k] = (int)std::lround(g(rng));
    }
    for (uint32_t t = 0; t < towers; ++t) {
        const u64 q = c->QP[t];
        vec vT(n), e0T(n), e1T(n), mT(n);
        for (uint32_t k = 0; k < n; ++k) {
            vT[k] = emb(vc[k], q); e0T[k] = emb(e0c[k], q); e1T[k] = emb(e1c[k], q);
            mT[k] = emb((long)m[k], q);
        }
        ntt_one(c, vT.data(), t); ntt_one(c, e0T.data(), t); ntt_one(c, e1T.data(), t); ntt_one(c, mT.data(), t);
        for (uint32_t k = 0; k < n; ++k) {
            size_t x = (size_t)t * n + k;
            u64 b = addmod(mulmod(pkB[x], vT[k], q), mulmod(ns % q, e0T[k], q), q);
            u64 a = addmod(mulmod(pkA[x], vT[k], q), mulmod(ns % q, e1T[k], q), q);
            c0[x] = addmod(b, mT[k], q);
            c1[x] = a;
        }
    }
}

void orc_decrypt(const OrcCtx* c, uint32_t towers, const u64* c0, const u64* c1, const u64* s,
                 int64_t* mout) {
    /* encdec.cpp:68-81: tower 0 only */
    (void)towers;
    const uint32_t n = c->n;
    const u64 q = c->Q[0];
    vec ph(n);
    for (uint32_t k = 0; k < n; ++k) ph[k] = addmod(c0[k], mulmod(c1[k], s[k], q), q);
    intt_one(c, ph.data(), 0);
    for (uint32_t k = 0; k < n; ++k) { u64 v = ph[k]; mout[k] = v > q / 2 ? (int64_t)v - (int64_t)q : (int64_t)v; }
}

void orc_modraise(const OrcCtx* c, uint32_t towers, const u64* c0, const u64* c1, u64* out0, u64* out1) {
    /* tests/test_modraise.cpp:50-58: per component, decrypt_host with a zero
     * partner (encdec.cpp:68-81: tower-0 INTT, centre v > q0/2 -> v - q0),
     * then pt_to_eval_host over `towers` towers (rotate.cpp:104-112:
     * ((v % q) + q) % q, NTT per tower) */
    const uint32_t n = c->n;
    const u64 q0 = c->Q[0];
    const u64* in[2] = {c0, c1};
    u64* out[2] = {out0, out1};
    vec x(n);
    for (int p = 0; p < 2; ++p) {
        std::memcpy(x.data(), in[p], (size_t)n * 8);
        intt_one(c, x.data(), 0);
        for (uint32_t t = 0; t < towers; ++t) {
            const long long q = (long long)c->Q[t];
            u64* o = out[p] + (size_t)t * n;
            for (uint32_t k = 0; k < n; ++k) {
                const long long v = x[k] > q0 / 2 ? (long long)x[k] - (long long)q0 : (long long)x[k];
                o[k] = (u64)((v % q + q) % q);
            }
            ntt_one(c, o, t);
        }
    }
}

void orc_phase_coeff(const OrcCtx* c, uint32_t towers, const u64* c0, const u64* c1, const u64* s,
                     u64* phase) {
    const uint32_t n = c->n;
    for (uint32_t t = 0; t < towers; ++t) {
        const u64 q = c->Q[t];
        for (uint32_t k = 0; k < n; ++k) {
            size_t x = (size_t)t * n + k;
            phase[x] = addmod(c0[x], mulmod(c1[x], s[x], q), q);
        }
        intt_one(c, phase + (size_t)t * n, t);
    }
}

void orc_keyswitch(const OrcCtx* c, uint32_t key_id, uint32_t L, const u64* a, u64* ba0, u64* ba1) {
    std::vector<vec> digits;
    modup(c, L, a, digits);
    vec res0, res1;
    inner_product(c, key_id, L, digits, res0, res1);
    moddown(c, L, res0, ba0);
    moddown(c, L, res1, ba1);
}

void orc_rescale(const OrcCtx* c, uint32_t L, u64* comp) {
    vec s1, s2;
    rescale_consts(s1, s2, c->Q.data(), L - 1);
    rescale_comp(c, L, comp, s1, s2);
}

void orc_evalmult_rescale(const OrcCtx* c, uint32_t L, const u64* c0a, const u64* c1a,
                          const u64* c0b, const u64* c1b, u64* out0, u64* out1) {
    evalmult_rescale_one(c, L, c0a, c1a, c0b, c1b, out0, out1);
}

void orc_evalmult_rescale_batch(const OrcCtx* c, uint32_t npairs, const uint32_t* L,
                                const u64* const* c0a, const u64* const* c1a,
                                const u64* const* c0b, const u64* const* c1b, u64* const* out0,
                                u64* const* out1, int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int64_t p = 0; p < (int64_t)npairs; ++p)
        evalmult_rescale_one(c, L[p], c0a[p], c1a[p], c0b[p], c1b[p], out0[p], out1[p]);
    (void)nthreads;
}

void orc_automorph_eval(const OrcCtx* c, uint32_t towers, uint32_t k, u64* v, int qp_order) {
    /* rotate.cpp:87-101: INTT -> permute -> NTT per tower */
    (void)qp_order;  /* tower t always uses QP[t] (Q towers first, then P) */
    const uint32_t n = c->n;
    vec o(n);
    for (uint32_t t = 0; t < towers; ++t) {
        const uint32_t qp = t;
        u64* col = v + (size_t)t * n;
        intt_one(c, col, qp);
        automorph(o.data(), col, n, k, c->QP[qp]);
        std::memcpy(col, o.data(), (size_t)n * 8);
        ntt_one(c, col, qp);
    }
}

void orc_rotate(const OrcCtx* c, uint32_t key_id, uint32_t L, uint32_t k, u64* c0, u64* c1) {
    /* rotate_ct_host (rotate.cpp:176-188) */
    const uint32_t n = c->n;
    orc_automorph_eval(c, L, k, c0, 1);
    orc_automorph_eval(c, L, k, c1, 1);
    vec ba0((size_t)L * n), ba1((size_t)L * n);
    orc_keyswitch(c, key_id, L, c1, ba0.data(), ba1.data());
    for (uint32_t t = 0; t < L; ++t) {
        const u64 q = c->Q[t];
        for (uint32_t kk = 0; kk < n; ++kk) { size_t x = (size_t)t * n + kk; c0[x] = addmod(c0[x], ba0[x], q); }
    }
    std::memcpy(c1, ba1.data(), (size_t)L * n * 8);
}

void orc_rotate_hoisted(const OrcCtx* c, uint32_t L, uint32_t nrot, const uint32_t* ks,
                        const uint32_t* key_ids, const u64* c0, const u64* c1, u64* const* out0,
                        u64* const* out1) {
    /* One ModUp of c1 shared by every rotation: digits are automorphed over
     * QlP in eval form, then inner product with the rotation key and ModDown. */
    const uint32_t n = c->n, QlP = L + c->K;
    std::vector<vec> digits;
    modup(c, L, c1, digits);
    std::vector<uint32_t> qpi(QlP);
    for (uint32_t i = 0; i < QlP; ++i) qpi[i] = qlp_index(c, L, i);
    for (uint32_t r = 0; r < nrot; ++r) {
        std::vector<vec> dg = digits;
        vec o(n);
        for (auto& d : dg)
            for (uint32_t i = 0; i < QlP; ++i) {
                u64* col = d.data() + (size_t)i * n;
                intt_one(c, col, qpi[i]);
                automorph(o.data(), col, n, ks[r], c->QP[qpi[i]]);
                std::memcpy(col, o.data(), (size_t)n * 8);
                ntt_one(c, col, qpi[i]);
            }
        vec res0, res1;
        inner_product(c, key_ids[r], L, dg, res0, res1);
        moddown(c, L, res0, out0[r]);
        moddown(c, L, res1, out1[r]);
        vec a0(c0, c0 + (size_t)L * n);
        orc_automorph_eval(c, L, ks[r], a0.data(), 1);
        for (uint32_t t = 0; t < L; ++t) {
            const u64 q = c->Q[t];
            for (uint32_t kk = 0; kk < n; ++kk) {
                size_t x = (size_t)t * n + kk;
                out0[r][x] = addmod(a0[x], out0[r][x], q);
            }
        }
    }
}

void orc_lintrans_bsgs(const OrcCtx* c, uint32_t L, uint32_t n1, uint32_t n2, const u64* c0, const u64* c1,
                       const u64* const* diag, int hoisted, u64* out0, u64* out1) {
    /* Baby-step giant-step linear transform, the sequence of the reference's
     * tests/test_c2s_bsgs.cpp:129-151: baby rotations rot_b(x), b < n1 (rot_0 = x);
     * for every giant step g < n2: in_g = sum_b diag[g*n1+b] (.) rot_b(x)
     * (ct_mul_pt_host then ct_add_ct_host, ptops.cpp:13-26), in_g rotated by
     * g*n1 slots when g > 0 (rotate_ct_host), accumulated. Rotation by r slots
     * uses Galois element 5^r mod 2n and the key stored under that element.
     * hoisted != 0: the baby rotations share one ModUp (orc_rotate_hoisted). */
    const uint32_t n = c->n, M = 2 * n;
    const size_t T = (size_t)L * n;
    auto gal = [&](uint32_t r) { u64 k = 1; for (uint32_t t = 0; t < r; ++t) k = (k * 5) % M; return (uint32_t)k; };
    std::vector<vec> B0(n1, vec(c0, c0 + T)), B1(n1, vec(c1, c1 + T));
    if (n1 > 1) {
        if (hoisted) {
            std::vector<uint32_t> ks(n1 - 1);
            std::vector<u64*> o0(n1 - 1), o1(n1 - 1);
            for (uint32_t b = 1; b < n1; ++b) { ks[b - 1] = gal(b); o0[b - 1] = B0[b].data(); o1[b - 1] = B1[b].data(); }
            orc_rotate_hoisted(c, L, n1 - 1, ks.data(), ks.data(), c0, c1, o0.data(), o1.data());
        } else {
            for (uint32_t b = 1; b < n1; ++b) orc_rotate(c, gal(b), L, gal(b), B0[b].data(), B1[b].data());
        }
    }
    vec acc0(T, 0), acc1(T, 0);
    for (uint32_t g = 0; g < n2; ++g) {
        vec in0(T, 0), in1(T, 0);
        for (uint32_t b = 0; b < n1; ++b) {
            const u64* d = diag[(size_t)g * n1 + b];
            if (!d) continue;
            for (uint32_t t = 0; t < L; ++t)
                orc_ptmulacc(in0.data() + (size_t)t * n, in1.data() + (size_t)t * n, B0[b].data() + (size_t)t * n,
                             B1[b].data() + (size_t)t * n, d + (size_t)t * n, c->Q[t], n);
        }
        if (g > 0) orc_rotate(c, gal(g * n1), L, gal(g * n1), in0.data(), in1.data());
        for (uint32_t t = 0; t < L; ++t) {
            orc_add_into(acc0.data() + (size_t)t * n, in0.data() + (size_t)t * n, c->Q[t], n);
            orc_add_into(acc1.data() + (size_t)t * n, in1.data() + (size_t)t * n, c->Q[t], n);
        }
    }
    std::memcpy(out0, acc0.data(), T * 8);
    std::memcpy(out1, acc1.data(), T * 8);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Canonical encode / decode (reference src/encode.cpp:13-44): slots
 * z_0..z_{N/2-1} <-> integer coefficients at scale Delta with
 * r_k = 5^k mod 2N and the twiddle table tw[t] = polar(1, -+pi t / N).
 *   encode: m_j = llround((2 Delta / N) * sum_k (Re z_k Re tw[j r_k] - Im z_k Im tw[j r_k]))
 *   decode: z_k = (sum_j m_j tw[j r_k]) / Delta
 * Sums run in index order with separate products and sums (no fused
 * multiply-add), so the doubles equal the reference's. */
void orc_encode(int64_t* m, const double* zre, const double* zim, uint32_t N, double Delta) {
    const uint32_t M = 2 * N, S = N / 2;
    std::vector<double> twr(M), twi(M);
    for (uint32_t t = 0; t < M; ++t) {
        const std::complex<double> w = std::polar(1.0, -M_PI * (double)t / (double)N);
        twr[t] = w.real();
        twi[t] = w.imag();
    }
    std::vector<uint64_t> r(S);
    uint64_t rk = 1;
    for (uint32_t k = 0; k < S; ++k) { r[k] = rk; rk = (rk * 5) % M; }
    const double sc = 2.0 * Delta / (double)N;
    for (uint32_t j = 0; j < N; ++j) {
        double acc = 0;
        for (uint32_t k = 0; k < S; ++k) {
            const uint64_t t = ((uint64_t)j * r[k]) % M;
            const double a = zre[k] * twr[t];
            const double b = zim[k] * twi[t];
            acc += a - b;
        }
        m[j] = (int64_t)llround(sc * acc);
    }
}

void orc_decode(double* zre, double* zim, const int64_t* m, uint32_t N, double Delta) {
    const uint32_t M = 2 * N, S = N / 2;
    std::vector<double> twr(M), twi(M);
    for (uint32_t t = 0; t < M; ++t) {
        const std::complex<double> w = std::polar(1.0, +M_PI * (double)t / (double)N);
        twr[t] = w.real();
        twi[t] = w.imag();
    }
    uint64_t rk = 1;
    for (uint32_t k = 0; k < S; ++k) {
        double ar = 0, ai = 0;
        for (uint32_t j = 0; j < N; ++j) {
            const uint64_t t = ((uint64_t)j * rk) % M;
            const double mj = (double)m[j];
            ar += mj * twr[t];
            ai += mj * twi[t];
        }
        zre[k] = ar / Delta;
        zim[k] = ai / Delta;
        rk = (rk * 5) % M;
    }
}

}  // extern "C"
