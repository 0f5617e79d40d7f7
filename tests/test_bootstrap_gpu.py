"""The reference's composed CKKS bootstrap (tests/test_boot.cpp) run on the
GPU entry points, in the reference test's order and with its parameters.

n = 8192 (4096 slots); Q = one 60-bit and twenty-nine 55-bit primes, P = two
60-bit primes; every key has digits of two towers; the secret has exactly 64
nonzero coefficients (test_boot.cpp:40-56). A message z encoded at
Delta_in = 2^54 * sqrt(n / 1024) * 8 is encrypted at q0 alone, then

1. ModRaise lifts it to all 30 towers (gpufhe_modraise_batch); the raised
   ciphertext decrypts over q0 q1 to a_k = m_k + q0 I_k (the reference's
   congruence gate, test_boot.cpp:123-160).
2. CoeffsToSlots: three merged radix-2^4 FFT stages (test_boot.cpp:200-300),
   each a sum of diagonal (.) rotation terms over 16 or 31 diagonals, then a
   rescale. The slots become y_k = a_k / q0 in bit-reversed order.
3. The real / imaginary split: conj(y) by the Galois element 2n - 1, then
   y + conj(y) and y - conj(y) (test_boot.cpp:318-330).
4. EvalMod on both branches: affine map, degree-10 Chebyshev series of cos,
   seven double-angle steps, each ciphertext product relinearised with a key
   made for its own level (test_boot.cpp:333-432).
5. SlotsToCoeffs: the three forward FFT stages, the imaginary branch folded
   into the first one (test_boot.cpp:456-520).
6. Decrypt at the output level and decode: every slot within the reference
   test's bound of z (|boot(z) - z| < 2e-2, test_boot.cpp:555).

On the device: every key (public, the 75 rotation keys and the conjugation
key with the reference's seeds, one relinearisation key per level), the
encryption, every encoding (gpufhe_encode_batch), every plaintext eval form
(gpufhe_pt_to_eval_batch), the rotations (batched, gpufhe_run_ops), every
product, sum and rescale, and the decryption. The FFT-stage diagonals are
computed on the host in double precision, as the reference does.
"""
import ctypes as C
import math
import time

import numpy as np
import pytest

from gpu_util import empty, host, ptr, sync

pytestmark = pytest.mark.gpu

N = 8192
S = N // 2
M = 2 * N
SQ, SP, HW = 30, 2, 64
LGS = 12
LST, RST = 3, 4                      # three merged stages of four radix-2 stages each
DELTA_IN = 2.0 ** 54 * math.sqrt(N / 1024.0) * 8.0
DELTA_PT = 2.0 ** 50
DELTA_W = 2.0 ** 55
DEG = 10
RDBL = int(math.ceil(math.log2(2 * math.pi * (2.5 * math.sqrt(HW) + 0.25))))   # 7
RK = np.array([pow(5, k, M) for k in range(S)], np.int64)


def parr(ts):
    return (C.c_void_p * len(ts))(*[ptr(t) for t in ts])


def to_int128(lo, hi):
    """Two's-complement 128-bit integer from its low and high 64-bit words."""
    v = int(lo) | (int(hi) << 64)
    return v - (1 << 128) if v >> 127 else v


def brev(i):
    return int(format(i, f"0{LGS}b")[::-1], 2)


def twd(k, st):
    return np.exp(2j * np.pi * ((RK[k] << st) % M) / M)


def stage_diagonals(g, forward):
    """Diagonals of merged FFT stage g as the reference derives them: the
    stage applied to every unit vector, entry (i, (i + d) mod S) of the
    result filed under diagonal d, a diagonal kept when any entry exceeds
    1e-12 (test_boot.cpp:222-239 for CoeffsToSlots, 465-488 for
    SlotsToCoeffs). Returns (offsets, [count][S] complex)."""
    V = np.eye(S, dtype=np.complex128)
    sts = list(range(g * RST, (g + 1) * RST))
    for st in (reversed(sts) if forward else sts):
        h = S >> (st + 1)
        W = V.reshape(S // (2 * h), 2, h, S)
        a, b = W[:, 0], W[:, 1]
        t = twd(np.arange(h), st)[None, :, None]
        o = np.stack([a + t * b, a - t * b] if forward else [(a + b) * 0.5, (a - b) / (2.0 * t)], axis=1)
        V = o.reshape(S, S)
    i = np.arange(S)
    offs, dg = [], []
    for d in range(S):
        col = V[i, (i + d) % S]
        if np.any(np.abs(col) > 1e-12):
            offs.append(d)
            dg.append(col)
    return offs, np.array(dg)


class Ct:
    def __init__(self, c0, c1, tw, scale):
        self.c0, self.c1, self.tw, self.scale = c0, c1, tw, scale


class Boot:
    """The reference's helper lambdas (mulK, subK, mulCt, lvl, x2, subC,
    rescaleAt) on the device entry points."""

    def __init__(self):
        import torch
        import gpufhe_b200 as G
        self.G, self.torch = G, torch
        q0 = G.native_primes(1, 60, N)
        self.Q = np.concatenate([q0, G.native_primes(SQ - 1, 55, N, avoid=list(q0))])
        self.P = G.native_primes(SP, 60, N, avoid=list(self.Q))
        self.qd = [float(q) for q in self.Q]
        self.full = G.Context(N, self.Q, self.P, 2)
        self.enc = G.Encoder(N)
        T = SQ + SP
        self.s, self.pkA, self.pkB = empty(T * N), empty(T * N), empty(T * N)
        G.check(G.lib().gpufhe_keygen(self.full.h, T, HW, 1, 3.19, 101, ptr(self.s), ptr(self.pkA),
                                      ptr(self.pkB), None))
        self.lev = {}

    # ---------------------------------------------------------------- keys
    def rotation_keys(self, gal_seeds, copy=()):
        """Full-QP rotation keys installed under their Galois elements; the
        canonical words of those in `copy` are returned as {galois: (av, bv)}."""
        gal = [g for g, _ in gal_seeds]
        ids = (C.c_uint64 * len(gal))(*gal)
        seeds = (C.c_uint64 * len(gal))(*[s for _, s in gal_seeds])
        words = 15 * (SQ + SP) * N
        kept = {g: (empty(words), empty(words)) for g in gal if g in set(copy)}
        av = (C.c_void_p * len(gal))(*[ptr(kept[g][0]) if g in kept else None for g in gal])
        bv = (C.c_void_p * len(gal))(*[ptr(kept[g][1]) if g in kept else None for g in gal])
        self.G.check(self.G.lib().gpufhe_evalkeygen(self.full.h, len(gal), ids, ids, seeds, ptr(self.s),
                                                    ptr(self.pkA), ptr(self.pkB), 1, 3.19, av, bv, None))
        return kept

    def relin_ctx(self, tw):
        """buildK(tw): a relinearisation key over (q_0 .. q_{tw-1}, P) from
        the chain's secret and public key, seed 202 (test_boot.cpp:342-360)."""
        if tw not in self.lev:
            G, t = self.G, self.torch
            g = G.Context(N, self.Q[:tw], self.P, 2)
            sl = lambda v: t.cat([v[:tw * N], v[SQ * N:(SQ + SP) * N]]).contiguous()
            ls, la, lb = sl(self.s), sl(self.pkA), sl(self.pkB)
            one = C.c_uint64 * 1
            G.check(G.lib().gpufhe_evalkeygen(g.h, 1, one(0), one(0), one(202), ptr(ls), ptr(la), ptr(lb), 1,
                                              3.19, None, None, None))
            self.lev[tw] = g
        return self.lev[tw]

    # ---------------------------------------------------------------- primitives
    def encode(self, z, scale):
        return self.enc.encode(np.asarray(z, np.complex128), scale)

    def pt_eval(self, ms, tw):
        ms = np.ascontiguousarray(np.atleast_2d(ms), np.int64)
        outs = [empty(tw * N) for _ in range(ms.shape[0])]
        dm = self.torch.from_numpy(ms).cuda()
        self.G.check(self.G.lib().gpufhe_pt_to_eval_batch(self.full.h, len(outs), tw, dm.data_ptr(), parr(outs),
                                                          None))
        return outs

    def pw(self, ops):
        self.G.pointwise(self.full, ops)

    def op(self, kind, a, b, tw, scalar=0, out=None):
        o0, o1 = out if out is not None else (empty(tw * N), empty(tw * N))
        bb = () if b is None else tuple(ptr(x) for x in b)
        self.pw([dict(kind=kind, towers=tw, a=(ptr(a[0]), ptr(a[1])), b=bb, o=(ptr(o0), ptr(o1)), scalar=scalar)])
        return o0, o1

    def rescale(self, a, tw):
        c0, c1 = a[0][:tw * N].clone(), a[1][:tw * N].clone()
        R = self.G.RESCALE
        self.G.run_ops(self.full, [dict(level=tw, mode=R, inp=[ptr(c0)], out=[ptr(c0)]),
                                   dict(level=tw, mode=R, inp=[ptr(c1)], out=[ptr(c1)])])
        return c0[:(tw - 1) * N], c1[:(tw - 1) * N]

    def rotate_many(self, src, gals, tw):
        outs = [(empty(tw * N), empty(tw * N)) for _ in gals]
        self.G.run_ops(self.full, [dict(level=tw, mode=self.G.ROTATE, key_id=k, galois=k,
                                        inp=[ptr(src[0]), ptr(src[1])], out=[ptr(o[0]), ptr(o[1])])
                                   for k, o in zip(gals, outs)])
        return outs

    def decrypt(self, a):
        dec = np.zeros((1, N), np.int64)
        self.G.check(self.G.lib().gpufhe_decrypt_batch(self.full.h, 1, parr([a[0]]), parr([a[1]]), ptr(self.s),
                                                       dec.ctypes.data, None))
        return dec[0]

    def decrypt_crt(self, a, towers):
        out = np.zeros((1, N, 2), np.uint64)
        self.G.check(self.G.lib().gpufhe_decrypt_crt_batch(self.full.h, 1, towers, parr([a[0]]), parr([a[1]]),
                                                           ptr(self.s), out.ctypes.data, None))
        return [to_int128(lo, hi) for lo, hi in out[0]]

    # ---------------------------------------------------------------- the reference's lambdas
    def lvl(self, A, tw):
        return Ct(A.c0[:tw * N], A.c1[:tw * N], tw, A.scale)

    def x2(self, A):
        c = self.op(self.G.PW_MUL_INT, (A.c0, A.c1), None, A.tw, scalar=2)
        return Ct(c[0], c[1], A.tw, A.scale)

    def sub_ct(self, A, B):
        c = self.op(self.G.PW_SUB, (A.c0, A.c1), (B.c0, B.c1), A.tw)
        return Ct(c[0], c[1], A.tw, A.scale)

    def sub_k(self, A, v):
        p = self.pt_eval(self.encode(np.full(S, v, np.complex128), A.scale), A.tw)[0]
        c = self.op(self.G.PW_SUB_PT, (A.c0, A.c1), (p,), A.tw)
        return Ct(c[0], c[1], A.tw, A.scale)

    def mul_k(self, A, v):
        p = self.pt_eval(self.encode(np.full(S, v, np.complex128), DELTA_W), A.tw)[0]
        c = self.rescale(self.op(self.G.PW_MUL_PT, (A.c0, A.c1), (p,), A.tw), A.tw)
        return Ct(c[0], c[1], A.tw - 1, A.scale * DELTA_W / self.qd[A.tw - 1])

    def mul_ct(self, A, B):
        tw = A.tw
        o0, o1 = empty((tw - 1) * N), empty((tw - 1) * N)
        self.G.run_ops(self.relin_ctx(tw), [dict(level=tw, inp=[ptr(A.c0), ptr(A.c1), ptr(B.c0), ptr(B.c1)],
                                                 out=[ptr(o0), ptr(o1)])])
        return Ct(o0, o1, tw - 1, A.scale * B.scale / self.qd[tw - 1])

    def fft_stage(self, srcs, offs, dg, tw, dpt):
        """One merged stage: sum over sources (ciphertext, factor) and
        diagonals d of encode(factor * diag_d, dpt) (.) rot_d(ciphertext),
        then a rescale (test_boot.cpp:283-296, 494-513)."""
        G = self.G
        terms, msgs = [], []
        for (src, fac) in srcs:
            rots = self.rotate_many(src, [pow(5, d, M) for d in offs if d], tw)
            it = iter(rots)
            for d, diag in zip(offs, dg):
                terms.append(next(it) if d else (src[0][:tw * N], src[1][:tw * N]))
                msgs.append(diag * fac)
        pts = self.pt_eval(self.encode(np.array(msgs), dpt), tw)
        prods = [(empty(tw * N), empty(tw * N)) for _ in terms]
        self.pw([dict(kind=G.PW_MUL_PT, towers=tw, a=(ptr(t[0]), ptr(t[1])), b=(ptr(p),),
                      o=(ptr(o[0]), ptr(o[1]))) for t, p, o in zip(terms, pts, prods)])
        acc = prods[0]
        for o in prods[1:]:
            self.op(G.PW_ADD, acc, o, tw, out=acc)
        return self.rescale(acc, tw)

    def evalmod(self, X, aff, cc, baff):
        """test_boot.cpp:407-432."""
        U = self.sub_k(self.mul_k(X, aff), complex(-baff, 0))
        T = [None, U, self.sub_k(self.x2(self.mul_ct(U, U)), 1.0)]
        for k in range(3, DEG + 1):
            ul = self.lvl(U, T[k - 1].tw)
            p = self.x2(self.mul_ct(ul, T[k - 1]))
            T.append(self.sub_ct(p, self.lvl(T[k - 2], p.tw)))
        low = T[DEG].tw
        terms = [self.lvl(T[k], low) for k in range(1, DEG + 1)]
        pts = self.pt_eval(self.encode(np.array([np.full(S, cc[k], np.complex128) for k in range(1, DEG + 1)]),
                                       DELTA_W), low)
        prods = [(empty(low * N), empty(low * N)) for _ in terms]
        self.pw([dict(kind=self.G.PW_MUL_PT, towers=low, a=(ptr(t.c0), ptr(t.c1)), b=(ptr(p),),
                      o=(ptr(o[0]), ptr(o[1]))) for t, p, o in zip(terms, pts, prods)])
        acc = prods[0]
        for o in prods[1:]:
            self.op(self.G.PW_ADD, acc, o, low, out=acc)
        r = self.rescale(acc, low)
        A = self.sub_k(Ct(r[0], r[1], low - 1, terms[0].scale * DELTA_W / self.qd[low - 1]), complex(-cc[0], 0))
        for _ in range(RDBL):
            A = self.sub_k(self.x2(self.mul_ct(A, A)), 1.0)
        return A


def chebyshev_cos(deg):
    """Chebyshev coefficients of cos(x) on [-1, 1] by 4(deg+1)-point
    quadrature (test_boot.cpp:400-405)."""
    nq = 4 * (deg + 1)
    cc = []
    for k in range(deg + 1):
        s = 0.0
        for j in range(nq):
            th = math.pi * (j + 0.5) / nq
            s += math.cos(math.cos(th)) * math.cos(k * th)
        cc.append(2.0 * s / nq)
    cc[0] *= 0.5
    return cc


def negacyclic_int(a, s):
    """a * s in Z[x]/(x^n + 1) with Python integers; s sparse."""
    out = [0] * N
    for j in np.nonzero(s)[0].tolist():
        sj = int(s[j])
        for i in range(N):
            k = i + j
            if k < N:
                out[k] += sj * a[i]
            else:
                out[k - N] -= sj * a[i]
    return out


def test_bootstrap():
    B = Boot()
    G, Q = B.G, B.Q
    q0 = int(Q[0])

    # message, public key over q0 alone (keygen_host over mod1, seed 101), encryption at q0
    i = np.arange(S)
    z = 0.35 * np.sin(0.02 * i) + 1j * 0.25 * np.cos(0.017 * i)
    mz = B.encode(z, DELTA_IN)
    s1, a1, b1 = empty(N), empty(N), empty(N)
    G.check(G.lib().gpufhe_keygen(B.full.h, 1, HW, 1, 3.19, 101, ptr(s1), ptr(a1), ptr(b1), None))
    assert B.torch.equal(s1, B.s[:N])
    c0, c1 = empty(N), empty(N)
    G.check(G.lib().gpufhe_encrypt_batch(B.full.h, 1, 1, np.ascontiguousarray(mz).ctypes.data,
                                         (C.c_uint64 * 1)(303), ptr(a1), ptr(b1), 1, 3.19, parr([c0]), parr([c1]),
                                         None))
    # stage clock as the reference's (test_boot.cpp:112, 536-543), checks excluded
    laps, mark = {}, [0.0]

    def lap(name=None):
        sync()
        now = time.time()
        if name:
            laps[name] = laps.get(name, 0.0) + now - mark[0]
        mark[0] = now

    lap()

    # 1. ModRaise and the reference's congruence gate
    R0, R1 = empty(SQ * N), empty(SQ * N)
    G.check(G.lib().gpufhe_modraise_batch(B.full.h, 1, SQ, parr([c0]), parr([c1]), parr([R0]), parr([R1]), None))
    lap("modraise")
    zero = empty(N)
    a0c = B.decrypt((c0, zero))                      # centred c0, c1 at q0 (decrypt_host with a zero partner)
    a1c = B.decrypt((c1, zero))
    scoef = B.decrypt((B.s[:N], zero))               # the secret's coefficients
    assert int(np.count_nonzero(scoef)) == HW and set(np.unique(scoef).tolist()) <= {-1, 0, 1}
    prod = negacyclic_int([int(v) for v in a1c], scoef)
    aref = [int(a0c[k]) + prod[k] for k in range(N)]
    dec1 = B.decrypt((c0, c1))
    bad = sum((aref[k] - int(dec1[k])) % q0 != 0 for k in range(N))
    assert bad == 0
    assert B.decrypt_crt((R0, R1), 2) == aref        # Garner over q0 q1 of the raised ciphertext
    aq = np.array([float(v) / q0 for v in aref])     # slots after C2S: y_k = (a_k + i a_{k+S}) / q0

    # rotation keys: every stage offset, seed 4000 + offset; conjugation, seed 7400
    lap()
    c2s = [stage_diagonals(g, False) for g in range(LST)]
    s2c = {g: stage_diagonals(g, True) for g in range(LST)}
    lap("diagonals")
    offsets = sorted(({d for o, _ in c2s for d in o} | {d for g in s2c for d in s2c[g][0]}) - {0})
    assert len(offsets) == 75
    keys0 = B.rotation_keys([(pow(5, d, M), 4000 + d) for d in offsets] + [(M - 1, 7400)],
                            copy=[pow(5, d, M) for d in c2s[0][0] if d])
    lap("rotation_keys")

    # 2. CoeffsToSlots: declared input scale q0, the scale held flat through
    #    the first two stages (diagonals encoded at the modulus being dropped)
    ct, tw, sc = (R0, R1), SQ, float(q0)
    for g in range(LST):
        offs, dg = c2s[g]
        dpt = B.qd[tw - 1] if g + 1 < LST else DELTA_PT
        ct = B.fft_stage([(ct, 1.0)], offs, dg, tw, dpt)
        if g == 0:
            stage0 = ct
        sc = sc * dpt / B.qd[tw - 1]
        tw -= 1
    nt, s_out = tw, sc
    lap("c2s")
    v = B.enc.decode(B.decrypt(ct), s_out)
    ref = aq[:S] + 1j * aq[S:]
    perm = np.array([brev(k) for k in range(S)])
    err_c2s = np.max(np.abs(v[perm] - ref))

    # 3. real / imaginary split by conjugation
    lap()
    (k0, k1), = B.rotate_many(ct, [M - 1], nt)
    ctR = Ct(*B.op(G.PW_ADD, ct, (k0, k1), nt), nt, s_out)
    ctI = Ct(*B.op(G.PW_SUB, ct, (k0, k1), nt), nt, s_out)
    lap("split")

    # 4. EvalMod on both branches
    aaff, baff = 2 * math.pi / 2.0 ** RDBL, -(math.pi / 2) / 2.0 ** RDBL
    cc = chebyshev_cos(DEG)
    oR = B.evalmod(ctR, complex(aaff / 2.0, 0), cc, baff)
    oI = B.evalmod(ctI, complex(0, -aaff / 2.0), cc, baff)
    lap("evalmod")
    assert oR.tw == oI.tw == nt - (1 + (DEG - 1) + 1 + RDBL)
    vR = B.enc.decode(B.decrypt((oR.c0, oR.c1)), oR.scale)
    err_mod = np.max(np.abs(vR.real - np.sin(2 * math.pi * aq[perm])))

    # 5. SlotsToCoeffs: the imaginary branch folded into the first stage
    lap()
    ct, tw, sc = None, oR.tw, oR.scale
    for g in range(LST - 1, -1, -1):
        offs, dg = s2c[g]
        dpt = B.qd[tw - 1] if g > 0 else DELTA_PT
        srcs = ([((oR.c0, oR.c1), 1.0), ((oI.c0, oI.c1), 1j)] if g == LST - 1 else [(ct, 1.0)])
        ct = B.fft_stage(srcs, offs, dg, tw, dpt)
        sc = sc * dpt / B.qd[tw - 1]
        tw -= 1
    lap("s2c")

    # 6. decrypt, decode at the final scale, compare with z
    d_final = sc * 2 * math.pi * DELTA_IN / q0
    zf = B.enc.decode(B.decrypt(ct), d_final)
    lap("decrypt_decode")
    err = np.max(np.abs(zf - z))
    print(f"\nbootstrap n={N}: ModRaise congruence mismatches {bad}; C2S slot err {err_c2s:.3e}; "
          f"EvalMod(R) err {err_mod:.3e}; output towers {tw}; {len(offsets) + 1} rotation keys; "
          f"max |boot(z) - z| = {err:.3e}")
    print(f"  z[0]={z[0]:.6g} got={zf[0]:.6g}  z[1]={z[1]:.6g} got={zf[1]:.6g}")
    print("bootstrap seconds (checks excluded; diagonals: the six stages' diagonals in numpy on the host; "
          "evalmod includes its per-level relinearisation keys): "
          + ", ".join(f"{k} {v:.3f}" for k, v in laps.items()) + f"; total {sum(laps.values()):.3f}")
    assert tw == SQ - 2 * LST - (1 + (DEG - 1) + 1 + RDBL)
    assert err < 2e-2, err

    # the oracle on the same keys and inputs: ModRaise and the first
    # CoeffsToSlots stage (15 rotations at 30 towers, 16 diagonal products,
    # the sum and the rescale) bit for bit
    w0, w1, r0, r1 = oracle_stage0(B, c0, c1, c2s[0], keys0)
    assert np.array_equal(host(R0), w0) and np.array_equal(host(R1), w1)
    assert np.array_equal(host(stage0[0]), r0) and np.array_equal(host(stage0[1]), r1)


def oracle_stage0(B, c0, c1, stage, keys):
    """The oracle's restatement of ModRaise (tests/test_modraise.cpp:50-58)
    and of one CoeffsToSlots stage as the reference composes it
    (test_boot.cpp:283-296: encode_host, pt_to_eval_host, rotate_ct_host,
    ct_mul_pt_host, ct_add_ct_host, rescale_resident_raw)."""
    import oracle as O
    o = O.Ctx(N, B.Q, B.P, 2)
    for k, (av, bv) in keys.items():
        o.set_key(k, host(av), host(bv))
    w0, w1 = o.modraise(SQ, host(c0), host(c1))
    dpt = B.qd[SQ - 1]
    tables = [O.root_tables(N, int(B.Q[t]), int(o.roots[t]))[:2] for t in range(SQ)]
    acc = None
    for d, diag in zip(*stage):
        m = O.encode(diag, N, dpt)
        pt = [O.ntt(np.mod(m, np.int64(B.Q[t])).astype(np.uint64), N, int(B.Q[t]), *tables[t]) for t in range(SQ)]
        t0, t1 = (w0, w1) if d == 0 else o.rotate(SQ, pow(5, d, M), w0, w1, pow(5, d, M))
        prod = []
        for comp in (t0, t1):
            out = np.empty(SQ * N, np.uint64)
            for t in range(SQ):
                sl = slice(t * N, (t + 1) * N)
                r = np.empty(N, np.uint64)
                O.lib().orc_rns_mult(np.ascontiguousarray(comp[sl]), pt[t], r, int(B.Q[t]), N)
                out[sl] = r
            prod.append(out)
        if acc is None:
            acc = prod
        else:
            qv = np.repeat(B.Q[:SQ].astype(np.uint64), N)
            acc = [np.where(a + p >= qv, a + p - qv, a + p) for a, p in zip(acc, prod)]
    return w0, w1, o.rescale(SQ, acc[0]), o.rescale(SQ, acc[1])
