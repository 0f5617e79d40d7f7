/*
 * CPU oracle for the resident leveled-CKKS EvalMult / Rescale / Rotate path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a scalar, CUDA-free restatement of the
 * reference library's arithmetic (samfrazerdutton/GPU-Resident-Library), used
 * by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker. Nothing in the product library links or calls it.
 *
 * Every array is uint64 residues, tower-major [tower][coeff]. Eval form is the
 * bit-reversed NTT order produced by orc_ntt.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- parameter generation (params.cpp:29-75) ---- */
int      orc_native_primes(uint64_t* out, uint32_t count, uint32_t bits, uint32_t n,
                           const uint64_t* avoid, uint32_t navoid);
uint64_t orc_native_root(uint32_t n, uint64_t q);
void     orc_rescale_consts(uint64_t* s1, uint64_t* s2, const uint64_t* mod, uint32_t last);

/* ---- twiddle tables (keyswitch_resident.cpp:47-68) ---- */
void orc_root_tables(uint32_t n, uint64_t q, uint64_t root,
                     uint64_t* fr, uint64_t* fp, uint64_t* ir, uint64_t* ip,
                     uint64_t* ninv_out /* [2]: n^-1, precon */);

/* ---- per-tower primitives (reference kernels directory) ---- */
void orc_ntt(uint64_t* x, const uint64_t* fr, const uint64_t* fp, uint32_t n, uint64_t q);
void orc_intt(uint64_t* x, const uint64_t* ir, const uint64_t* ip, uint32_t n, uint64_t q,
              uint64_t ninv, uint64_t ninv_precon);
void orc_rns_mult(const uint64_t* a, const uint64_t* b, uint64_t* r, uint64_t q, uint32_t n);
void orc_tensor(const uint64_t* c0a, const uint64_t* c1a, const uint64_t* c0b, const uint64_t* c1b,
                uint64_t* t0, uint64_t* t1, uint64_t* t2, const uint64_t* mods,
                uint32_t sizeQ, uint32_t n);
void orc_combine(uint64_t* r0, uint64_t* r1, const uint64_t* t0, const uint64_t* t1,
                 const uint64_t* ba0, const uint64_t* ba1, const uint64_t* mods,
                 uint32_t sizeQ, uint32_t n);
void orc_switch_modulus(uint64_t* v, uint64_t q_old, uint64_t q_new, uint32_t n);
void orc_rescale_fuse(uint64_t* a, const uint64_t* b, uint64_t s1, uint64_t s2, uint64_t q, uint32_t n);
uint64_t orc_barrett_u128(uint64_t a_lo, uint64_t a_hi, uint64_t modulus, uint64_t mu_lo, uint64_t mu_hi);
void orc_approx_switch(const uint64_t* src, uint64_t* dst,
                       const uint64_t* QHatInv, const uint64_t* QHatInvPrec, const uint64_t* q,
                       const uint64_t* QHatModp, const uint64_t* p,
                       const uint64_t* mu_lo, const uint64_t* mu_hi,
                       uint32_t sizeQ, uint32_t sizeP, uint32_t n);
void orc_ks_macc(uint64_t* out0, uint64_t* out1, const uint64_t* digit,
                 const uint64_t* b, const uint64_t* a, uint64_t q, uint32_t n);
void orc_moddown_combine(uint64_t* ans, const uint64_t* a, const uint64_t* b,
                         uint64_t s, uint64_t q, uint32_t n);
void orc_automorph(uint64_t* out, const uint64_t* in, uint32_t n, uint64_t k, uint64_t q);
void orc_add_into(uint64_t* a, const uint64_t* b, uint64_t q, uint32_t n);
void orc_ptmulacc(uint64_t* acc0, uint64_t* acc1, const uint64_t* b0, const uint64_t* b1,
                  const uint64_t* d, uint64_t q, uint32_t n);

/* ---- keyswitch constants (ks_constants.cpp:31-102), explicit partition ----
 * Layout of the flat output (sizes in uint64 words), for nparts digits of
 * alpha towers each (last one ragged):
 *   per part p: QHatInv[sp], QHatInvPrec[sp], srcMod[sp], QHatModp[sp*sc],
 *               complMod[sc], muLo[sc], muHi[sc]
 *   moddown:    pHatInv[K], pHatInvPrec[K], pHatModq[K*L], mdMuLo[L], mdMuHi[L], pInvModq[L]
 * orc_ks_constants_size returns the total word count. */
uint64_t orc_ks_constants_size(uint32_t sizeQ, uint32_t sizeP, uint32_t alpha);
void     orc_ks_constants(uint64_t* out, const uint64_t* modQ, uint32_t sizeQ,
                          const uint64_t* modP, uint32_t sizeP, uint32_t alpha);

/* ---- oracle context: chain + tables + keys ---- */
typedef struct OrcCtx OrcCtx;
/* roots may be NULL: then native_root(n, q) is used for every modulus. */
OrcCtx* orc_ctx_create(uint32_t n, const uint64_t* modQ, uint32_t fullQ,
                       const uint64_t* modP, uint32_t sizeP, uint32_t alpha,
                       const uint64_t* rootsQP);
void    orc_ctx_destroy(OrcCtx* c);
void    orc_ctx_roots(const OrcCtx* c, uint64_t* rootsQP);
/* Installs a key (av/bv: [dnum][fullQ+K][n], eval form). Key id 0 = relin. */
int     orc_ctx_set_key(OrcCtx* c, uint32_t key_id, const uint64_t* av, const uint64_t* bv);

/* keygen/evalkeygen/enc/dec (keygen.cpp:55-112, evalkeygen.cpp:42-113, encdec.cpp:41-81) */
void orc_set_hamming_weight(uint32_t h);
/* s, pkA, pkB: [towers][n] eval over the first `towers` moduli of QP order
 * (Q towers first, then P). towers==fullQ+K gives the QP key. */
void orc_keygen(const OrcCtx* c, uint32_t towers, uint64_t ns, double sigma, uint64_t seed,
                uint64_t* s, uint64_t* pkA, uint64_t* pkB);
/* Relin (sOld = s^2) or rotation (sOld = sigma_k(s)) key over full QP with the
 * context's partition. av/bv out: [dnum][fullQ+K][n]. */
void orc_evalkeygen(const OrcCtx* c, const uint64_t* sQP, const uint64_t* sOld,
                    const uint64_t* pkA_QP, const uint64_t* pkB_QP,
                    uint64_t ns, double sigma, uint64_t seed, uint64_t* av, uint64_t* bv);
void orc_encrypt(const OrcCtx* c, uint32_t towers, const int64_t* m,
                 const uint64_t* pkA, const uint64_t* pkB, uint64_t ns, double sigma,
                 uint64_t seed, uint64_t* c0, uint64_t* c1);
/* tower-0 decrypt exactly as decrypt_host */
void orc_decrypt(const OrcCtx* c, uint32_t towers, const uint64_t* c0, const uint64_t* c1,
                 const uint64_t* s, int64_t* mout);
/* per-tower phase c0 + c1*s in coefficient form (for full-CRT decryption) */
void orc_phase_coeff(const OrcCtx* c, uint32_t towers, const uint64_t* c0, const uint64_t* c1,
                     const uint64_t* s, uint64_t* phase);

/* ---- composite path (keyswitch_resident.cpp:139-244, rotate.cpp:70-132) ---- */
void orc_keyswitch(const OrcCtx* c, uint32_t key_id, uint32_t L, const uint64_t* a,
                   uint64_t* ba0, uint64_t* ba1);
/* rescale_resident_raw on one component: [L][n] -> first L-1 towers rewritten */
void orc_rescale(const OrcCtx* c, uint32_t L, uint64_t* comp);
/* tensor -> keyswitch -> combine -> rescale x2; out0/out1: [L-1][n] */
void orc_evalmult_rescale(const OrcCtx* c, uint32_t L,
                          const uint64_t* c0a, const uint64_t* c1a,
                          const uint64_t* c0b, const uint64_t* c1b,
                          uint64_t* out0, uint64_t* out1);
/* batch of independent pairs with OpenMP over pairs; ptr arrays of length npairs */
void orc_evalmult_rescale_batch(const OrcCtx* c, uint32_t npairs, const uint32_t* L,
                                const uint64_t* const* c0a, const uint64_t* const* c1a,
                                const uint64_t* const* c0b, const uint64_t* const* c1b,
                                uint64_t* const* out0, uint64_t* const* out1, int nthreads);
/* sigma_k on every tower of an eval-form poly (rotate.cpp:87-101) */
void orc_automorph_eval(const OrcCtx* c, uint32_t towers, uint32_t k, uint64_t* v, int qp_order);
/* rotate_ct_host: automorph c0,c1; keyswitch c1 with key_id; c0 += ba0; c1 = ba1 */
void orc_modraise(const OrcCtx* c, uint32_t towers, const uint64_t* c0, const uint64_t* c1, uint64_t* out0,
                  uint64_t* out1);
void orc_rotate(const OrcCtx* c, uint32_t key_id, uint32_t L, uint32_t k, uint64_t* c0, uint64_t* c1);
/* hoisted: one ModUp of c1 shared by nrot rotations (automorph the digits). */
void orc_lintrans_bsgs(const OrcCtx* c, uint32_t L, uint32_t n1, uint32_t n2, const uint64_t* c0, const uint64_t* c1,
                       const uint64_t* const* diag, int hoisted, uint64_t* out0, uint64_t* out1);
void orc_rotate_hoisted(const OrcCtx* c, uint32_t L, uint32_t nrot, const uint32_t* ks,
                        const uint32_t* key_ids, const uint64_t* c0, const uint64_t* c1,
                        uint64_t* const* out0, uint64_t* const* out1);
int orc_num_threads(void);

/* Canonical encode / decode (reference src/encode.cpp:13-44): z as separate
 * real / imaginary arrays of N/2 slots, m of N coefficients. */
void orc_encode(int64_t* m, const double* zre, const double* zim, uint32_t N, double Delta);
void orc_decode(double* zre, double* zim, const int64_t* m, uint32_t N, double Delta);

#ifdef __cplusplus
}
#endif
