/*
 * gpufhe_b200 — B200-native resident leveled-CKKS hot path, C ABI.
 *
 * The reference (samfrazerdutton/GPU-Resident-Library) exposes its hot path
 * as 14 extern "C" Launch* kernels (ntt.h, intt.h, rns_arith.h, ...; same
 * names and semantics are exported by this library, see those headers) and a
 * C++ API (device_ciphertext.h, ckks_ops.h, keyswitch_resident.h, keygen.h).
 * This header adds the batched / serving entry points that the reference has
 * no counterpart for, as plain C: opaque handles, raw pointers, sizes, and an
 * int status (0 = success, negative = error; gpufhe_last_error() explains).
 *
 * Data layout everywhere: tower-major [tower][coeff] uint64 residues in
 * [0, q), eval form = the reference's bit-reversed NTT order.
 */
#ifndef GPUFHE_B200_H
#define GPUFHE_B200_H

#include <cuda_runtime.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPUFHE_OK 0
#define GPUFHE_EINVAL (-1)   /* bad argument, unsupported size, missing key */
#define GPUFHE_ECUDA (-2)    /* a CUDA call failed */
#define GPUFHE_ENOMEM (-3)   /* workspace or HBM budget too small */
#define GPUFHE_EBUSY (-4)    /* server queue full / request not admitted yet */
#define GPUFHE_ETIMEOUT (-5) /* bounded wait expired */

typedef struct gpufhe_ctx gpufhe_ctx;

const char* gpufhe_last_error(void);

/* ---------------------------------------------------------------- context
 * Modulus chain Q[0..fullQ) and special primes P[0..K), digit width alpha
 * (towers per Hybrid digit, fixed across levels so one full-QP key serves
 * every level). roots_qp: the 2n-th roots for Q then P, or NULL for the
 * smallest-generator roots (the reference's native_root). Builds twiddle
 * tables and every per-level constant on `device`. Replaces the per-call
 * setup of ks_context_create (reference keyswitch_resident.cpp:32-101). */
int  gpufhe_ctx_create(uint32_t n, const uint64_t* Q, uint32_t fullQ, const uint64_t* P, uint32_t K,
                       uint32_t alpha, const uint64_t* roots_qp, int device, gpufhe_ctx** out);
/* Ends the handle. The context's device state is freed at once, or, while
 * plans, linear-transform plans or servers built on it still exist, when the
 * last of them is destroyed (they stay valid until then). */
void gpufhe_ctx_destroy(gpufhe_ctx* ctx);
int  gpufhe_ctx_roots(const gpufhe_ctx* ctx, uint64_t* roots_qp);
/* Key over full QP, host [dnum][fullQ+K][n] (dnum = ceil(fullQ/alpha)),
 * canonical eval form (reference KeySwitchConstants::av/bv, keyswitch.h:35-39).
 * key_id 0 = relinearisation key; rotation keys use their Galois element. */
int  gpufhe_ctx_set_key(gpufhe_ctx* ctx, uint64_t key_id, const uint64_t* av, const uint64_t* bv);
uint64_t gpufhe_ctx_resident_bytes(const gpufhe_ctx* ctx);
/* Rotation-key residency (the key management the reference leaves to its
 * caller: every ks_context_create uploads one key per call, reference
 * keyswitch_resident.cpp:32-101). bytes = 0 (the default) keeps every key
 * resident. Otherwise the device holds at most `bytes` of keys: each key set
 * after the budget keeps a pinned host copy, the least recently used key no
 * plan holds is evicted to make room, and a plan built over a batch uploads
 * the batch's evicted keys and pins them for its lifetime. A batch whose keys
 * do not fit returns GPUFHE_ENOMEM from plan creation. A budget below one
 * key's bytes is GPUFHE_EINVAL. */
int  gpufhe_ctx_set_key_budget(gpufhe_ctx* ctx, uint64_t bytes);
/* out[6] = {keys known, keys resident, resident key bytes, uploads from host
 * copies, evictions, budget}. */
int  gpufhe_ctx_key_stats(const gpufhe_ctx* ctx, uint64_t* out);
/* Synchronises the context's device and returns (then clears) its device
 * status word: 0 when every bounded wait inside this library's kernels was
 * met; otherwise bit 0 = a key-tile wait, bit 1 = a stage wait of a consumer,
 * bit 2 = a stage-release wait of the producer in the TMA form of the key
 * inner product expired (the kernel then left without writing that tile's
 * results). No counterpart in the reference. */
int  gpufhe_ctx_device_status(gpufhe_ctx* ctx, uint32_t* out);

/* ---------------------------------------------------------------- keys and encryption
 * Seeded key generation, eval-key generation, encryption and decryption on
 * the device. The random draws are the reference's (std::mt19937_64,
 * std::normal_distribution + lround, in its order), made on the host; the
 * same seed gives the same keys and ciphertexts, bit for bit. Embedding into
 * the towers, the NTTs and the products run as batched launches. Every call
 * returns after its work on `stream` has completed. Tower t uses QP modulus t
 * (Q towers, then P). */
/* Secret s, public key (pkA, pkB) over the first `towers` QP moduli, eval
 * form, device [towers][n] each; hw = 0: uniform ternary secret, else exactly
 * hw nonzero coefficients (reference keygen_host, src/keygen.cpp:55-112, with
 * set_secret_hamming_weight). */
int gpufhe_keygen(gpufhe_ctx* ctx, uint32_t towers, uint32_t hw, uint64_t ns, double sigma, uint64_t seed,
                  uint64_t* d_s, uint64_t* d_pkA, uint64_t* d_pkB, cudaStream_t stream);
/* `count` eval keys over the full QP basis, key i switching sOld -> s with
 * sOld = s^2 (galois[i] = 0, relinearisation) or sigma_galois[i](s), drawn
 * from seeds[i] and installed in the context under key_ids[i] (reference
 * evalkeygen_host / evalkeygen_host_sold, src/evalkeygen.cpp:42-113, followed
 * by the key upload of ks_context_create, keyswitch_resident.cpp:32-101).
 * d_sQP, d_pkA, d_pkB: device [fullQ+K][n] from gpufhe_keygen over all QP
 * towers. d_av_out / d_bv_out: optional host arrays of count device pointers
 * ([dnum][fullQ+K][n] each, may be null) that receive the canonical keys. */
int gpufhe_evalkeygen(gpufhe_ctx* ctx, uint32_t count, const uint64_t* key_ids, const uint64_t* galois,
                      const uint64_t* seeds, const uint64_t* d_sQP, const uint64_t* d_pkA, const uint64_t* d_pkB,
                      uint64_t ns, double sigma, uint64_t* const* d_av_out, uint64_t* const* d_bv_out,
                      cudaStream_t stream);
/* gpufhe_ctx_set_key from device arrays. */
int gpufhe_ctx_set_key_device(gpufhe_ctx* ctx, uint64_t key_id, const uint64_t* d_av, const uint64_t* d_bv);
/* Encrypts `count` integer-coefficient messages m (host [count][n]) under
 * (d_pkA, d_pkB) ([towers][n] eval form), message i with seeds[i], into the
 * device buffers d_c0[i], d_c1[i] ([towers][n] each; host arrays of device
 * pointers) (reference encrypt_host, src/encdec.cpp:41-64). */
int gpufhe_encrypt_batch(gpufhe_ctx* ctx, uint32_t count, uint32_t towers, const int64_t* m, const uint64_t* seeds,
                         const uint64_t* d_pkA, const uint64_t* d_pkB, uint64_t ns, double sigma,
                         uint64_t* const* d_c0, uint64_t* const* d_c1, cudaStream_t stream);
/* Decrypts `count` ciphertexts with the secret d_s, the reference's way: the
 * phase c0 + c1*s in tower 0 only, centred mod q0 (reference decrypt_host,
 * src/encdec.cpp:68-81); m_out host [count][n]. */
int gpufhe_decrypt_batch(gpufhe_ctx* ctx, uint32_t count, const uint64_t* const* d_c0, const uint64_t* const* d_c1,
                         const uint64_t* d_s, int64_t* m_out, cudaStream_t stream);
/* Exact decryption over the first `towers` Q towers: the phase in every
 * tower, centred CRT reconstruction (Garner) of each coefficient as a
 * two's-complement 128-bit integer, out128 host [count][n][2] = {low, high}
 * words; exact while |coefficient| < 2^127. No counterpart in the reference
 * (which recovers from tower 0 only). */
int gpufhe_decrypt_crt_batch(gpufhe_ctx* ctx, uint32_t count, uint32_t towers, const uint64_t* const* d_c0,
                             const uint64_t* const* d_c1, const uint64_t* d_s, uint64_t* out128,
                             cudaStream_t stream);
/* ---------------------------------------------------------------- ciphertext arithmetic
 * Batched arithmetic without a keyswitch on eval-form ciphertexts at any
 * level (towers = the operation's level, the first `towers` Q moduli), with
 * the reference's formulas and so its bits: the host loops of
 * src/ptops.cpp:13-26 (ct_add_ct_host, ct_mul_pt_host) and the subtract,
 * plaintext subtract and scale-by-integer loops its tests write around them
 * (tests/test_evalmod.cpp:100-113). All operations run in one launch; an
 * output may be its own input. Device buffers are [towers][n]:
 *   ADD      o = a + b          (both components; b0, b1)
 *   SUB      o = a - b          (both components; b0, b1)
 *   MUL_PT   o = a (.) b0       (both components times the plaintext b0)
 *   ADD_PT   o0 = a0 + b0, o1 = a1
 *   SUB_PT   o0 = a0 - b0, o1 = a1
 *   MUL_INT  o = a * scalar mod q (both components) */
#define GPUFHE_PW_ADD 0u
#define GPUFHE_PW_SUB 1u
#define GPUFHE_PW_MUL_PT 2u
#define GPUFHE_PW_ADD_PT 3u
#define GPUFHE_PW_SUB_PT 4u
#define GPUFHE_PW_MUL_INT 5u
typedef struct gpufhe_pw_op {
    uint32_t kind;
    uint32_t towers;
    const uint64_t* a0;
    const uint64_t* a1;
    const uint64_t* b0;
    const uint64_t* b1;
    uint64_t* o0;
    uint64_t* o1;
    uint64_t scalar;
} gpufhe_pw_op;
/* Asynchronous on `stream`; at most 65535 operations per call. */
int gpufhe_pointwise_batch(gpufhe_ctx* ctx, uint32_t count, const gpufhe_pw_op* ops, cudaStream_t stream);

/* Integer plaintexts to eval form: message i (device int64, d_m + i*n)
 * embedded mod each of the first `towers` Q towers (((v % q) + q) % q) and
 * transformed into d_out[i] (host array of count device pointers to
 * [towers][n]), with one embedding launch and one batched NTT launch pair
 * for the whole batch. Replaces the reference's pt_to_eval_host
 * (src/rotate.cpp:104-112), which its linear transforms call once per
 * diagonal. At most 65535 plaintexts per call. Asynchronous on `stream`. */
int gpufhe_pt_to_eval_batch(gpufhe_ctx* ctx, uint32_t count, uint32_t towers, const int64_t* d_m,
                            uint64_t* const* d_out, cudaStream_t stream);
/* ModRaise of `count` ciphertexts from tower q0 alone to the first `towers`
 * towers of Q: each component's tower 0 goes to coefficients, is centred mod
 * q0 (v > q0/2 -> v - q0) and embedded mod every q_t, and every tower goes
 * back to eval form. The raised ciphertext decrypts to the original phase
 * plus q0*I for a small integer polynomial I. Replaces the sequence the
 * reference composes on the host in tests/test_modraise.cpp:50-58
 * (decrypt_host with a zero partner, src/encdec.cpp:68-81, then
 * pt_to_eval_host, src/rotate.cpp:104-112). d_c0_in / d_c1_in: host arrays
 * of count device pointers, tower 0 = their first n words; d_c0_out /
 * d_c1_out: host arrays of count device pointers to [towers][n], distinct
 * from one another; an output may be its own input. At most 32767
 * ciphertexts per call. Asynchronous on `stream`. */
int gpufhe_modraise_batch(gpufhe_ctx* ctx, uint32_t count, uint32_t towers, const uint64_t* const* d_c0_in,
                          const uint64_t* const* d_c1_in, uint64_t* const* d_c0_out, uint64_t* const* d_c1_out,
                          cudaStream_t stream);

/* ---------------------------------------------------------------- canonical encode / decode
 * The reference's encode_host / decode_host (src/encode.cpp:13-44): slots
 * z_0..z_{n/2-1} (complex, interleaved re/im doubles) <-> n integer
 * coefficients at scale delta, with the same summation order, rounding and
 * twiddle table, so results equal the reference's bit for bit; one thread
 * per output index, a batch of messages per launch. The encoder holds the
 * twiddle table (32n bytes) and the rotation-group exponents on `device`;
 * calls must run with that device current. Buffers are host memory; each
 * call returns after its work on `stream` has completed. */
typedef struct gpufhe_encoder gpufhe_encoder;
int  gpufhe_encoder_create(uint32_t n, int device, gpufhe_encoder** out);
void gpufhe_encoder_destroy(gpufhe_encoder* enc);
/* z: [count][n/2][2] doubles; m: [count][n] */
int  gpufhe_encode_batch(gpufhe_encoder* enc, uint32_t count, const double* z, double delta, int64_t* m,
                         cudaStream_t stream);
int  gpufhe_decode_batch(gpufhe_encoder* enc, uint32_t count, const int64_t* m, double delta, double* z,
                         cudaStream_t stream);
/* The same maps by an O(n log n) transform over the rotation group instead
 * of the reference's O(n^2) sums (no counterpart in the reference): encoded
 * coefficients equal the reference's or differ by one where the exact value
 * lies within rounding error of a half-integer; decoded slots agree to
 * about n * 2^-52 relative. For serving paths where encoding would otherwise
 * cost more than encryption. */
int  gpufhe_encode_batch_fast(gpufhe_encoder* enc, uint32_t count, const double* z, double delta, int64_t* m,
                              cudaStream_t stream);
int  gpufhe_decode_batch_fast(gpufhe_encoder* enc, uint32_t count, const int64_t* m, double delta, double* z,
                              cudaStream_t stream);

/* ---------------------------------------------------------------- parameters
 * C forms of the reference's native parameter routines (include/params.h;
 * reference src/params.cpp:29-75). */
int      gpufhe_native_primes(uint64_t* out, uint32_t count, uint32_t bits, uint32_t n, const uint64_t* avoid,
                              uint32_t navoid);
uint64_t gpufhe_native_root(uint32_t n, uint64_t q);
int      gpufhe_rescale_consts(uint64_t* s1, uint64_t* s2, const uint64_t* mod, uint32_t last);

/* ---------------------------------------------------------------- transforms
 * Batched forward/inverse NTT of npolys x towers tower-polys stored
 * contiguously ([poly][tower][n]); tower t uses modulus first_tower + t in
 * Q||P order. d_jobs: device scratch of npolys*towers*gpufhe_ntt_job_bytes()
 * bytes that receives the job list; gpufhe_ntt_run_jobs re-launches a
 * prepared list (capturable in a CUDA graph). */
int gpufhe_ntt_batch(gpufhe_ctx* ctx, uint64_t* d_data, uint32_t npolys, uint32_t towers, uint32_t first_tower,
                     int inverse, uint64_t* d_jobs, cudaStream_t stream);
uint64_t gpufhe_ntt_job_bytes(void);
int gpufhe_ntt_run_jobs(gpufhe_ctx* ctx, const uint64_t* d_jobs, uint32_t njobs, int inverse,
                        cudaStream_t stream);
/* Batched RNS multiply out = a * b mod q over [npolys][towers][n] (tower t
 * uses modulus first_tower + t): plain residues in and out, the result of
 * LaunchRNSMultTower (reference rns_arith.cu:13-56) for every tower in one
 * launch. Buffers 16-byte aligned, n >= 2048; out may alias a or b. */
int gpufhe_rns_mult_batch(gpufhe_ctx* ctx, const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_out,
                          uint32_t npolys, uint32_t towers, uint32_t first_tower, cudaStream_t stream);
/* ApproxSwitchCRTBasis in a chosen form: the arguments and the result of
 * LaunchApproxSwitchCRTBasis (reference kernels/basis_convert.cu:14-114), bit
 * for bit. The tensor-core forms split every x_i and QHatModp[i][j] into
 * bytes; the fifteen byte-shift classes of the exact sum are unsigned 8-bit
 * matrix products with 32-bit sums (tcgen05.mma kind::i8 with the sums in
 * tensor memory, or the warp-level mma.sync m16n8k32), recombined into the
 * exact 128-bit sum before the same Barrett reduction. The integer form is
 * 128-bit multiply-adds on the integer pipes. LaunchApproxSwitchCRTBasis
 * itself takes the tcgen05 form wherever its shape allows (sizeQ <= 12,
 * sizeP <= 64, n a multiple of 128; n may span several polynomials, the
 * conversion is per coefficient), else the integer form. The mma.sync form
 * takes the same limits with n a multiple of 16. No counterpart in the
 * reference. */
#define GPUFHE_CONVERT_TCGEN05 0
#define GPUFHE_CONVERT_MMA_SYNC 1
#define GPUFHE_CONVERT_INTEGER 2
int gpufhe_approx_switch(const uint64_t* d_src, uint64_t* d_dst, const uint64_t* d_QHatInvModq,
                         const uint64_t* d_QHatInvModqPrecon, const uint64_t* d_q, const uint64_t* d_QHatModp,
                         const uint64_t* d_p, const uint64_t* d_mu_lo, const uint64_t* d_mu_hi, uint32_t sizeQ,
                         uint32_t sizeP, uint32_t n, int form, cudaStream_t stream);
/* Synchronizes the device and returns (then clears) the tensor-core
 * conversion's status word: 0, or 1 when a tcgen05 batch did not complete
 * within its bounded wait (its outputs are then not valid). */
int gpufhe_approx_switch_status(uint32_t* out);


/* ---------------------------------------------------------------- batched ops
 * One entry per ciphertext operation; a batch may mix levels and modes.
 *   GPUFHE_EVALMULT_RESCALE: in = {c0a, c1a, c0b, c1b} ([level][n] each),
 *       out = {r0, r1} ([level-1][n]): tensor -> Hybrid relinearisation ->
 *       combine -> rescale, the reference's bench_evalmult_resident.cpp:96-100
 *       chain, bit-exact.
 *   GPUFHE_KEYSWITCH: in[0] = a, out = {ba0, ba1} (keyswitch_resident,
 *       keyswitch_resident.cpp:139-225) with key `key_id`.
 *   GPUFHE_ROTATE: in = {c0, c1}, out = {sigma(c0)+ba0, ba1} with Galois
 *       element `galois` and the rotation key `key_id` (rotate_ct_device,
 *       rotate.cpp:118-132). Outputs must not alias inputs.
 *   GPUFHE_RESCALE: in[0] = comp [level][n] -> out[0] [level-1][n]
 *       (rescale_resident_raw, keyswitch_resident.cpp:227-244); out may alias in.
 *   GPUFHE_ROTATE_HOISTED: as GPUFHE_ROTATE, but every such operation of the
 *       batch with the same in[1] (c1) buffer and level shares one ModUp of c1,
 *       computed by the first of them; each rotation applies sigma_k to the
 *       shared digits in eval form before its key product. No counterpart in
 *       the reference (its rotate_ct_device, rotate.cpp:118-132, does one ModUp
 *       per rotation); the result differs from GPUFHE_ROTATE by the
 *       approximate-basis-conversion term, as hoisting always does.
 * Device pointers, 16-byte aligned; ring sizes 2^10..2^16. */
#define GPUFHE_EVALMULT_RESCALE 0u
#define GPUFHE_KEYSWITCH 1u
#define GPUFHE_ROTATE 2u
#define GPUFHE_RESCALE 3u
#define GPUFHE_ROTATE_HOISTED 4u

typedef struct gpufhe_op {
    uint32_t level;
    uint32_t mode;
    uint64_t key_id;
    uint64_t galois;
    const uint64_t* in[4];
    uint64_t* out[2];
} gpufhe_op;

typedef struct gpufhe_plan gpufhe_plan;

/* Device workspace one operation at `level` needs (sum over a batch). */
uint64_t gpufhe_op_workspace_bytes(gpufhe_ctx* ctx, uint32_t level);
/* Builds the per-phase job tables of a batch (one small device allocation).
 * d_ws: caller workspace of ws_bytes, or NULL for a plan-owned one. */
int  gpufhe_plan_create(gpufhe_ctx* ctx, uint32_t nops, const gpufhe_op* ops, uint64_t* d_ws, uint64_t ws_bytes,
                        gpufhe_plan** out);
/* Launches the phase kernels for the whole batch on `stream` (kernel
 * launches only: capturable in a CUDA graph). The first launch outside
 * capture runs the autotuner, which re-runs the batch to time the candidate
 * schedules (skipped for in-place rescales). */
int  gpufhe_plan_launch(gpufhe_plan* plan, cudaStream_t stream);
void gpufhe_plan_destroy(gpufhe_plan* plan);
/* One phase (0..8 = P1..P9) only, for per-kernel timing. */
int  gpufhe_plan_launch_phase(gpufhe_plan* plan, uint32_t phase, cudaStream_t stream);
/* Number of kernels one gpufhe_plan_launch enqueues. */
uint32_t gpufhe_plan_kernel_count(const gpufhe_plan* plan);
/* Launch schedule chosen by the autotuner (first gpufhe_plan_launch outside
 * graph capture, cached per context and batch shape): bits 0-1 = P5 form
 * (0 register prefetch, 128 threads x 4 words; 1 cp.async pipelined;
 * 2 register prefetch, 256 threads x 2 words; 3 bulk-copy (TMA) stage ring
 * with mbarriers, one producer warp and 128 consumer threads), bit 2 = every phase launches
 * its integer and FP64 transform jobs interleaved in one launch, bits 3-4 =
 * P3 form (0 plain; 1 warp-specialised, 128 conversion threads, two CTAs per
 * SM; 2 warp-specialised, 256 conversion threads, one CTA per SM: conversion
 * warps overlap the transform warps), bit 5 = tuned, bit 6 = the key inner
 * product (P5) of Q towers with q < 2^50 on the FP64 pipe (exact FP64 modular
 * products) beside the chosen integer form for the other rows, bit 7 = that
 * FP64 form's occupancy (0: four digits' loads in flight, four CTAs per SM;
 * 1: two digits, five CTAs), bit 17 = those FP64 rows on a second stream
 * beside the integer rows (forked and joined inside the launch, graph-
 * capturable), bit 18 = those FP64 rows through the bulk-copy (TMA) stage
 * ring of form 3 instead, of three stages (bit 7 clear) or two (bit 7 set),
 * bits 8-16 = the
 * phases (bit 8 + k for phase k+1) launched interleaved (the others as two
 * launches). */
uint32_t gpufhe_plan_schedule(const gpufhe_plan* plan);
/* Fixes the schedule (bits 0-4, 6-7 and 8-18 as above; bit 2 sets every phase
 * interleaved) and skips the autotuner; every schedule computes the same bits. */
int      gpufhe_plan_set_schedule(gpufhe_plan* plan, uint32_t schedule);
/* Host-buffer form: copies h_in[4*i+k] (host, level*n words) into op i's
 * device inputs, launches the batch and copies each op's outputs back into
 * h_out[2*i+k]; synchronizes `stream`. NULL entries are skipped. Pinned host
 * memory gives full PCIe bandwidth. */
int  gpufhe_plan_launch_host(gpufhe_plan* plan, const uint64_t* const* h_in, uint64_t* const* h_out,
                             cudaStream_t stream);
/* The same without the final synchronisation: copies and kernels are queued
 * on `stream`. Host buffers must be pinned and left untouched until the
 * stream reaches this point; two plans over separate device buffers on two
 * streams let one batch's host->device copies overlap another's transform
 * and device->host copies. */
int  gpufhe_plan_launch_host_async(gpufhe_plan* plan, const uint64_t* const* h_in, uint64_t* const* h_out,
                                   cudaStream_t stream);
/* Batch form of the above: h_in is one pinned host buffer holding every op's
 * inputs back to back in op order (each op's input components, level*n words
 * each), h_out one pinned buffer for all outputs in op order. Where the ops'
 * device buffers continue each other inside one device allocation, the
 * copies merge into one transfer each way (large copies reach PCIe's full
 * rate; a batch of 2-6 MB copies does not). No counterpart in the
 * reference. */
int  gpufhe_plan_launch_host_batch_async(gpufhe_plan* plan, const uint64_t* h_in, uint64_t* h_out,
                                         cudaStream_t stream);
/* create + launch + synchronize + destroy */
int  gpufhe_run_ops(gpufhe_ctx* ctx, uint32_t nops, const gpufhe_op* ops, cudaStream_t stream);

/* ---------------------------------------------------------------- linear transform
 * Baby-step giant-step homomorphic linear transform of the ciphertext
 * (d_c0, d_c1) at `level` (eval form, [level][n] each):
 *   y = sum_{g<n2} rot_{g*n1}( sum_{b<n1} diag[g*n1+b] (.) rot_b(x) ),
 * the sequence of the reference's tests/test_c2s_bsgs.cpp:129-151
 * (rotate_ct per step, ct_mul_pt + ct_add_ct for the inner sums). diag: host
 * array of n1*n2 device pointers to eval-form plaintext diagonals ([level][n])
 * or NULL for a zero diagonal. Rotation by r slots uses Galois element
 * 5^r mod 2n and needs the key stored under that element (baby steps
 * r = 1..n1-1, giant steps r = g*n1). hoisted != 0 computes the baby
 * rotations with one shared ModUp (GPUFHE_ROTATE_HOISTED; different bits from
 * the reference's per-rotation ModUp). Allocates scratch, runs the baby
 * rotations, the inner sums, the giant rotations and the final sum as four
 * batched launches on `stream`, and synchronises it. */
int gpufhe_lintrans_bsgs(gpufhe_ctx* ctx, uint32_t level, const uint64_t* d_c0, const uint64_t* d_c1, uint32_t n1,
                         uint32_t n2, const uint64_t* const* diag, int hoisted, uint64_t* d_out0, uint64_t* d_out1,
                         cudaStream_t stream);
/* Plan form of the same transform for repeated use: creation checks the
 * rotation keys, allocates the scratch, uploads the pointer tables and builds
 * the baby and giant rotation batches (which keep their keys resident while
 * the plan lives); launching enqueues the four steps on `stream` with no
 * allocation and no host transfer, so a launch can be captured in a CUDA graph
 * and replayed. Input, diagonals and output buffers are fixed at creation.
 * The reference runs the sequence as separate rotate / multiply / add calls
 * per step (tests/test_c2s_bsgs.cpp:129-151). */
typedef struct gpufhe_lintrans_plan gpufhe_lintrans_plan;
int  gpufhe_lintrans_plan_create(gpufhe_ctx* ctx, uint32_t level, const uint64_t* d_c0, const uint64_t* d_c1,
                                 uint32_t n1, uint32_t n2, const uint64_t* const* diag, int hoisted,
                                 uint64_t* d_out0, uint64_t* d_out1, gpufhe_lintrans_plan** out);
int  gpufhe_lintrans_plan_launch(gpufhe_lintrans_plan* plan, cudaStream_t stream);
void gpufhe_lintrans_plan_destroy(gpufhe_lintrans_plan* plan);

/* ---------------------------------------------------------------- no allocation
 * No counterpart in the reference. Rescale of one eval-form component
 * d_comp ([level][n], in place: the first level-1 towers receive the result)
 * that calls no cudaMalloc / cudaFree: for hosts that own the device-memory
 * budget through their own pool and forbid a library from allocating
 * (cudaMalloc can fail under a fixed budget, cudaFree synchronizes the
 * device), and for serving threads that must not block on an allocation.
 * Same result, bit for bit, as GPUFHE_RESCALE and rescale_resident_raw.
 * Its scratch is a static device array of gpufhe_rescale_noalloc_max_words()
 * uint64 words (8 MiB, held by every GPU that loads the library until the
 * process exits); level * n above that returns GPUFHE_ENOMEM. The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress), so
 * make it before any stream capture. All calls share the array: calls that
 * overlap on the GPU race. */
int      gpufhe_rescale_noalloc(gpufhe_ctx* ctx, uint32_t level, uint64_t* d_comp, cudaStream_t stream);
uint64_t gpufhe_rescale_noalloc_max_words(void);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference (its multi-ciphertext driver runs chains on
 * separate streams, bench/bench_batch.cpp:95-105). A continuous-batching
 * server over one or more contexts (ring sizes) on one device. A request is
 * a chain of EvalMult+Rescale (the ciphertext times itself) and rotation
 * operations on one ciphertext. Each step queues the next operation of every
 * admitted request as one batched plan per context; two steps stay in
 * flight. Requests are admitted FIFO, once arrived, while the device arena
 * (budget_bytes minus the contexts' resident tables and keys) has room for
 * two ciphertexts at their start level plus their workspace; a request's
 * memory returns to the arena when the step finishing it completes.
 * max_active caps admitted requests (0 = budget only); batch_cap caps the
 * operations of one plan (0 = none); plain != 0 runs one request at a time
 * (the plain one-chain-at-a-time form). */
typedef struct gpufhe_server gpufhe_server;

typedef struct gpufhe_req_op {
    uint32_t mode;      /* GPUFHE_EVALMULT_RESCALE or GPUFHE_ROTATE */
    uint32_t reserved;
    uint64_t galois;    /* GPUFHE_ROTATE: Galois element, also the key id */
} gpufhe_req_op;

typedef struct gpufhe_server_stats {
    uint64_t steps, ops, emr_ops, completed, peak_active, max_batch;
    uint64_t peak_bytes;       /* most arena bytes in use */
    uint64_t arena_bytes;      /* arena capacity */
    uint64_t resident_bytes;   /* tables + keys of every context */
    double busy_s;             /* first admission to last completion */
    double host_build_s;       /* host time building and launching steps */
    double host_wait_s;        /* host time blocked on a step still running on the GPU */
} gpufhe_server_stats;

typedef struct gpufhe_request_record {
    uint64_t id;
    uint32_t ctx, start_level, final_level, nops;
    /* seconds since the epoch (gpufhe_server_start); t_finish is the device
     * time at which the step holding the request's last operation completed */
    double t_arrival, t_admit, t_finish;
} gpufhe_request_record;

int      gpufhe_server_create(gpufhe_ctx* const* ctxs, uint32_t nctx, uint64_t budget_bytes, uint32_t max_active,
                              uint32_t batch_cap, int plain, gpufhe_server** out);
void     gpufhe_server_destroy(gpufhe_server* srv);
/* Arena bytes one request of context ctx starting at `level` holds. */
uint64_t gpufhe_server_request_bytes(gpufhe_server* srv, uint32_t ctx, uint32_t level);
/* Queues a request that arrives arrival_s seconds after the epoch. h_in:
 * host ciphertext [2][level][n] uploaded on admission, or NULL for seeded
 * residues generated on the device (SplitMix64 of seed, component, tower,
 * index). h_out: host buffer [2][final level][n] that receives the result,
 * or NULL. Pinned host buffers keep the copies asynchronous. GPUFHE_EINVAL
 * for an invalid chain (EvalMult+Rescale below level 2, a missing key),
 * GPUFHE_ENOMEM for a request larger than the whole arena. */
int      gpufhe_server_submit(gpufhe_server* srv, uint32_t ctx, uint32_t level, const gpufhe_req_op* ops,
                              uint32_t nops, double arrival_s, uint64_t seed, const uint64_t* h_in, uint64_t* h_out,
                              uint64_t* id);
/* Autotunes every context's launch schedule on EvalMult+Rescale batches of
 * 1, 2, 4, ... max_batch (0 = 256) operations, on zero-filled arena buffers,
 * so that serving steps (which only read the tuning cache) use measured
 * schedules; call while the server is idle. *tuned = batch shapes tuned. */
int      gpufhe_server_tune(gpufhe_server* srv, uint32_t max_batch, uint32_t* tuned);
/* Sets the epoch to now. */
int      gpufhe_server_start(gpufhe_server* srv);
/* One scheduling step; *queued = operations queued (0 when idle). */
int      gpufhe_server_step(gpufhe_server* srv, uint32_t* queued);
/* Steps until every request finished; GPUFHE_ETIMEOUT after max_seconds. */
int      gpufhe_server_drain(gpufhe_server* srv, double max_seconds);
uint64_t gpufhe_server_pending(gpufhe_server* srv);
int      gpufhe_server_get_stats(gpufhe_server* srv, gpufhe_server_stats* out);
/* Finished requests in completion order: *count = how many finished; up to
 * cap records are written to out (out may be NULL to ask for the count). */
int      gpufhe_server_records(gpufhe_server* srv, gpufhe_request_record* out, uint32_t cap, uint32_t* count);

#ifdef __cplusplus
}
#endif
#endif /* GPUFHE_B200_H */
