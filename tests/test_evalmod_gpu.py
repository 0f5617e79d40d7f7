"""EvalMod, the homomorphic reduction mod 1 of bootstrapping, in the exact
sequence of the reference's tests/test_evalmod.cpp, run once on the GPU
entry points and once on the oracle, written once against two backends.

n = 1024, Q = one 60-bit and fourteen 50-bit primes, P = two 60-bit primes,
scale 2^50; slots x = m + I with |m| <= 0.04 and I in [-2, 2]. The affine map
y = (pi/8) x - pi/32, a degree-8 Chebyshev series of cos(y) (T_2 .. T_8 by the
recurrence), one rescale of the coefficient sum, then four double-angle steps
c <- 2c^2 - 1 give cos(16 y) = sin(2 pi x), and sin(2 pi x) / (2 pi) ~ m: the
integer part is gone. As in the reference, every level tw has its own
relinearisation key over (q_0 .. q_{tw-1}, P) with digits of at most two
towers, made with seed 202 from the secret and public key of one keygen over
the whole chain.

On the GPU: keys (gpufhe_keygen, gpufhe_evalkeygen per level), encryption,
every encoding (gpufhe_encode_batch), plaintext embeddings
(gpufhe_pt_to_eval_batch), EvalMult+Rescale and rescale (the batched
pipeline), and every add / subtract / plaintext product / doubling
(gpufhe_pointwise_batch). The final ciphertext equals the oracle's bit for
bit and meets the reference test's own bound (|y / 2 pi - m| < 1e-3).
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as O
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

N, SQ, SP = 1024, 15, 2
S = N // 2
DELTA = 2.0 ** 50


def alpha_for(tw):
    """Digit width of the reference's per-level keys: numPart = 1 for tw <= 2,
    else (tw + 1) / 2 (test_evalmod.cpp:37)."""
    parts = 1 if tw <= 2 else (tw + 1) // 2
    return -(-tw // parts)


def parr(ts):
    return (C.c_void_p * len(ts))(*[ptr(t) for t in ts])


def chain():
    q0 = O.native_primes(1, 60, N)
    Q = np.concatenate([q0, O.native_primes(SQ - 1, 50, N, avoid=list(q0))])
    P = O.native_primes(SP, 60, N, avoid=list(Q))
    return Q, P


def slice_qp(v, tw):
    """Rows q_0..q_{tw-1} and the P rows of a [SQ+SP][n] array."""
    return np.concatenate([v[:tw * N], v[SQ * N:(SQ + SP) * N]])


class Ct:
    def __init__(self, c0, c1, tw, scale):
        self.c0, self.c1, self.tw, self.scale = c0, c1, tw, scale


class Gpu:
    def __init__(self, Q, P, s, pkA, pkB):
        import torch
        import gpufhe_b200 as G
        self.G, self.torch, self.Q = G, torch, Q
        self.full = G.Context(N, Q, P, 2)
        self.enc = G.Encoder(N)
        T = SQ + SP                   # one keygen over the whole chain, as the reference's
        ds, da, db = empty(T * N), empty(T * N), empty(T * N)
        G.check(G.lib().gpufhe_keygen(self.full.h, T, 0, 1, 3.19, 101, ptr(ds), ptr(da), ptr(db), None))
        assert np.array_equal(host(ds), s) and np.array_equal(host(da), pkA) and np.array_equal(host(db), pkB)
        self.s, self.pkA, self.pkB = ds, da, db
        self.lev = {}
        for tw in range(2, SQ + 1):
            g = G.Context(N, Q[:tw], P, alpha_for(tw))
            ls, la, lb = dev(slice_qp(s, tw)), dev(slice_qp(pkA, tw)), dev(slice_qp(pkB, tw))
            one = C.c_uint64 * 1
            G.check(G.lib().gpufhe_evalkeygen(g.h, 1, one(0), one(0), one(202), ptr(ls), ptr(la), ptr(lb), 1, 3.19,
                                              None, None, None))
            self.lev[tw] = g

    def encode(self, z, scale):
        return self.enc.encode(np.asarray(z, np.complex128), scale)

    def encrypt(self, m):
        c0, c1 = empty(SQ * N), empty(SQ * N)
        self.G.check(self.G.lib().gpufhe_encrypt_batch(self.full.h, 1, SQ, np.ascontiguousarray(m).ctypes.data,
                                                       (C.c_uint64 * 1)(303), ptr(self.pkA), ptr(self.pkB), 1, 3.19,
                                                       parr([c0]), parr([c1]), None))
        return c0, c1

    def pt_eval(self, m, tw):
        out = empty(tw * N)
        dm = self.torch.from_numpy(np.ascontiguousarray(m, np.int64)).cuda()
        self.G.check(self.G.lib().gpufhe_pt_to_eval_batch(self.full.h, 1, tw, dm.data_ptr(), parr([out]), None))
        return out

    def pw(self, kind, a, b, tw, scalar=0):
        o0, o1 = empty(tw * N), empty(tw * N)
        bb = () if b is None else tuple(ptr(x) for x in b)
        self.G.pointwise(self.full, [dict(kind=kind, towers=tw, a=(ptr(a[0]), ptr(a[1])), b=bb,
                                          o=(ptr(o0), ptr(o1)), scalar=scalar)])
        return o0, o1

    def add(self, a, b, tw): return self.pw(self.G.PW_ADD, a, b, tw)
    def sub(self, a, b, tw): return self.pw(self.G.PW_SUB, a, b, tw)
    def mul_pt(self, a, p, tw): return self.pw(self.G.PW_MUL_PT, a, (p,), tw)
    def sub_pt(self, a, p, tw): return self.pw(self.G.PW_SUB_PT, a, (p,), tw)
    def double(self, a, tw): return self.pw(self.G.PW_MUL_INT, a, None, tw, scalar=2)

    def rescale(self, a, tw):
        c0, c1 = a[0].clone(), a[1].clone()
        self.G.run_ops(self.full, [dict(level=tw, mode=self.G.RESCALE, inp=[ptr(c0)], out=[ptr(c0)]),
                                   dict(level=tw, mode=self.G.RESCALE, inp=[ptr(c1)], out=[ptr(c1)])])
        return c0[:(tw - 1) * N], c1[:(tw - 1) * N]

    def emr(self, a, b, tw):
        o0, o1 = empty((tw - 1) * N), empty((tw - 1) * N)
        self.G.run_ops(self.lev[tw], [dict(level=tw, inp=[ptr(a[0]), ptr(a[1]), ptr(b[0]), ptr(b[1])],
                                           out=[ptr(o0), ptr(o1)])])
        return o0, o1

    def head(self, a, tw):
        return a[0][:tw * N], a[1][:tw * N]

    def decrypt(self, a):
        dec = np.zeros((1, N), np.int64)
        self.G.check(self.G.lib().gpufhe_decrypt_batch(self.full.h, 1, parr([a[0]]), parr([a[1]]), ptr(self.s),
                                                       dec.ctypes.data, None))
        return dec[0]

    def words(self, a):
        sync()
        return host(a[0]), host(a[1])


class Oracle:
    def __init__(self, Q, P, s, pkA, pkB):
        self.Q, self.s, self.pkA, self.pkB = Q, s, pkA, pkB
        self.full = O.Ctx(N, Q, P, 2)
        self.roots = self.full.roots
        self.lev = {}
        for tw in range(2, SQ + 1):
            o = O.Ctx(N, Q[:tw], P, alpha_for(tw))
            sl = slice_qp(s, tw)
            sq = np.concatenate([np.array([(int(x) * int(x)) % int(q) for x in sl[t * N:(t + 1) * N].tolist()],
                                          np.uint64) for t, q in enumerate(o.QP)])
            av, bv = o.evalkeygen(sl, sq, slice_qp(pkA, tw), slice_qp(pkB, tw), seed=202)
            o.set_key(0, av, bv)
            self.lev[tw] = o

    def encode(self, z, scale):
        return O.encode(np.asarray(z, np.complex128), N, scale)

    def encrypt(self, m):
        return self.full.encrypt(SQ, m, self.pkA[:SQ * N], self.pkB[:SQ * N], seed=303)

    def pt_eval(self, m, tw):
        parts = []
        for t in range(tw):
            q = int(self.Q[t])
            fr, fp, _, _, _, _ = O.root_tables(N, q, int(self.roots[t]))
            parts.append(O.ntt(np.array([v % q for v in np.asarray(m).tolist()], np.uint64), N, q, fr, fp))
        return np.concatenate(parts)

    def _tw(self, f, a, b, tw):
        o = []
        for c in range(2):
            out = np.empty(tw * N, np.uint64)
            for t in range(tw):
                sl = slice(t * N, (t + 1) * N)
                out[sl] = f(a[c][sl], b[c][sl] if b is not None else None, np.uint64(self.Q[t]), t)
            o.append(out)
        return o[0], o[1]

    def add(self, a, b, tw):
        return self._tw(lambda x, y, q, t: np.where(x + y >= q, x + y - q, x + y), a, b, tw)

    def sub(self, a, b, tw):
        return self._tw(lambda x, y, q, t: np.where(x >= y, x - y, x + q - y), a, b, tw)

    def mul_pt(self, a, p, tw):
        def f(x, y, q, t):
            r = np.empty_like(x)
            O.lib().orc_rns_mult(x.copy(), p[t * N:(t + 1) * N].copy(), r, int(q), N)
            return r
        return self._tw(f, a, None, tw)

    def sub_pt(self, a, p, tw):
        c0 = a[0][:tw * N].copy()
        for t in range(tw):
            q, sl = np.uint64(self.Q[t]), slice(t * N, (t + 1) * N)
            x, y = c0[sl], p[sl]
            c0[sl] = np.where(x >= y, x - y, x + q - y)
        return c0, a[1][:tw * N].copy()

    def double(self, a, tw):
        return self._tw(lambda x, y, q, t: (x * np.uint64(2)) % q, a, None, tw)

    def rescale(self, a, tw):
        return self.full.rescale(tw, a[0][:tw * N]), self.full.rescale(tw, a[1][:tw * N])

    def emr(self, a, b, tw):
        return self.lev[tw].evalmult_rescale(tw, a[0][:tw * N], a[1][:tw * N], b[0][:tw * N], b[1][:tw * N])

    def head(self, a, tw):
        return a[0][:tw * N], a[1][:tw * N]

    def decrypt(self, a):
        return self.full.decrypt(1, a[0], a[1], self.s)

    def words(self, a):
        return a[0], a[1]


def evalmod(B, Q, xin):
    """tests/test_evalmod.cpp:125-190 against backend B."""
    qd = [float(q) for q in Q]
    full = lambda v: np.full(S, v, np.complex128)

    def mul_const(A, v):          # times encode(v, Delta), then rescale
        p = B.pt_eval(B.encode(full(v), DELTA), A.tw)
        o = B.rescale(B.mul_pt((A.c0, A.c1), p, A.tw), A.tw)
        return Ct(o[0], o[1], A.tw - 1, A.scale * DELTA / qd[A.tw - 1])

    def sub_const(A, v):          # c0 -= encode(v, A.scale)
        p = B.pt_eval(B.encode(full(v), A.scale), A.tw)
        c0, c1 = B.sub_pt((A.c0, A.c1), p, A.tw)
        return Ct(c0, c1, A.tw, A.scale)

    def mul_ct(A, Bc):
        o = B.emr((A.c0, A.c1), (Bc.c0, Bc.c1), A.tw)
        return Ct(o[0], o[1], A.tw - 1, A.scale * Bc.scale / qd[A.tw - 1])

    def reduce(A, tw):
        c0, c1 = B.head((A.c0, A.c1), tw)
        return Ct(c0, c1, tw, A.scale)

    def double(A):
        c0, c1 = B.double((A.c0, A.c1), A.tw)
        return Ct(c0, c1, A.tw, A.scale)

    def sub_ct(A, Bc):
        c0, c1 = B.sub((A.c0, A.c1), (Bc.c0, Bc.c1), A.tw)
        return Ct(c0, c1, A.tw, A.scale)

    c0, c1 = B.encrypt(B.encode(xin, DELTA))
    X = Ct(c0, c1, SQ, DELTA)
    a_, b_ = math.pi / 8.0, -math.pi / 32.0
    U = sub_const(mul_const(X, a_), -b_)
    deg, nq = 8, 36
    c = []
    for k in range(deg + 1):
        s = 0.0
        for j in range(nq):
            th = math.pi * (j + 0.5) / nq
            s += math.cos(math.cos(th)) * math.cos(k * th)
        c.append(2.0 * s / nq)
    c[0] *= 0.5
    T = [None, U, sub_const(double(mul_ct(U, U)), 1.0)]
    for k in range(3, deg + 1):
        p = double(mul_ct(reduce(U, T[k - 1].tw), T[k - 1]))
        T.append(sub_ct(p, reduce(T[k - 2], p.tw)))
    low = T[deg].tw
    acc = None
    for k in range(1, deg + 1):
        t = reduce(T[k], low)
        p = B.pt_eval(B.encode(full(c[k]), DELTA), low)
        m0, m1 = B.mul_pt((t.c0, t.c1), p, low)
        if acc is None:
            acc = Ct(m0, m1, low, t.scale * DELTA)
        else:
            s0, s1 = B.add((acc.c0, acc.c1), (m0, m1), low)
            acc = Ct(s0, s1, low, acc.scale)
    r0, r1 = B.rescale((acc.c0, acc.c1), low)
    acc = sub_const(Ct(r0, r1, low - 1, acc.scale / qd[low - 1]), -c[0])
    for _ in range(4):
        acc = sub_const(double(mul_ct(acc, acc)), 1.0)
    return acc


def test_evalmod():
    Q, P = chain()
    octx = O.Ctx(N, Q, P, 2)
    s, pkA, pkB = octx.keygen(SQ + SP, seed=101)
    i = np.arange(S)
    mtrue = 0.04 * np.sin(0.021 * i)
    xin = (mtrue + (i % 5) - 2).astype(np.complex128)
    g = evalmod(Gpu(Q, P, s, pkA, pkB), Q, xin)
    o = evalmod(Oracle(Q, P, s, pkA, pkB), Q, xin)
    assert g.tw == o.tw == 2 and g.scale == o.scale
    gw, ow = Gpu.words(None, (g.c0, g.c1)), (o.c0, o.c1)
    assert np.array_equal(gw[0], ow[0]) and np.array_equal(gw[1], ow[1])
    dec = O.Ctx(N, Q, P, 2).decrypt(1, gw[0], gw[1], s)
    y = O.decode(dec, N, g.scale)
    err_mod = np.max(np.abs(y.real / (2 * math.pi) - mtrue))
    assert err_mod < 1e-3, err_mod
