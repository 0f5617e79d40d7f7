"""The reference's homomorphic linear-transform engine test
(tests/test_c2s_engine.cpp) run on the GPU entry points: n = 1024, four
50-bit Q primes, two 51-bit P primes, two digits; an arbitrary real,
diagonal-dominant 512 x 512 matrix U applied to encrypt(x) as
sum_j diag_j (.) rot_j(ct) over all 512 diagonals, then one rescale.

Keys (secret, public, 511 rotation keys with the reference's seeds 900 + j),
the encryption (seed 303), the canonical encodings of x and of every
diagonal, the plaintexts' eval forms (gpufhe_pt_to_eval_batch), the 511
rotations with their products and sums (gpufhe_lintrans_bsgs with one giant
step) and the rescale all run on the device. The result equals the oracle's
restatement of the same sequence bit for bit, and decodes to U x within the
reference test's own bound (5e-3).
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

N, SQ, SP, ALPHA = 1024, 4, 2, 2
S = N // 2
DELTA = 2.0 ** 35


def parr(ts):
    return (C.c_void_p * len(ts))(*[ptr(t) for t in ts])


def test_c2s_engine():
    import torch
    import gpufhe_b200 as G
    Q = O.native_primes(SQ, 50, N)
    P = O.native_primes(SP, 51, N, avoid=list(Q))
    g = G.Context(N, Q, P, ALPHA)
    octx = O.Ctx(N, Q, P, ALPHA)
    T = SQ + SP
    ds, da, db = empty(T * N), empty(T * N), empty(T * N)
    G.check(G.lib().gpufhe_keygen(g.h, T, 0, 1, 3.19, 101, ptr(ds), ptr(da), ptr(db), None))
    M = 2 * N
    gal = [pow(5, j, M) for j in range(1, S)]
    cnt = len(gal)
    dnum = -(-SQ // ALPHA)
    av = [empty(dnum * T * N) for _ in range(cnt)]
    bv = [empty(dnum * T * N) for _ in range(cnt)]
    ids = (C.c_uint64 * cnt)(*gal)
    seeds = (C.c_uint64 * cnt)(*[900 + j for j in range(1, S)])
    G.check(G.lib().gpufhe_evalkeygen(g.h, cnt, ids, ids, seeds, ptr(ds), ptr(da), ptr(db), 1, 3.19,
                                      parr(av), parr(bv), None))

    # slots and matrix as the reference test builds them
    i = np.arange(S, dtype=np.float64)
    x = (0.3 * np.sin(0.1 * i)).astype(np.complex128)
    U = 0.02 * np.cos((0.03 * i[:, None]) * i[None, :] + 0.1) + 0.5 * np.eye(S)
    diags = np.stack([U[np.arange(S), (np.arange(S) + j) % S] for j in range(S)]).astype(np.complex128)
    enc = G.Encoder(N)
    mx = enc.encode(x, DELTA)
    md = enc.encode(diags, DELTA)                      # [512][1024]

    c0, c1 = empty(SQ * N), empty(SQ * N)
    G.check(G.lib().gpufhe_encrypt_batch(g.h, 1, SQ, np.ascontiguousarray(mx).ctypes.data, (C.c_uint64 * 1)(303),
                                         ptr(da), ptr(db), 1, 3.19, parr([c0]), parr([c1]), None))
    dm = torch.from_numpy(np.ascontiguousarray(md)).cuda()
    dev_diag = [empty(SQ * N) for _ in range(S)]
    G.check(G.lib().gpufhe_pt_to_eval_batch(g.h, S, SQ, dm.data_ptr(), parr(dev_diag), None))
    o0, o1 = empty(SQ * N), empty(SQ * N)
    G.lintrans_bsgs(g, SQ, ptr(c0), ptr(c1), S, 1, [ptr(d) for d in dev_diag], ptr(o0), ptr(o1))
    sync()
    pre0, pre1 = host(o0), host(o1)
    G.run_ops(g, [dict(level=SQ, mode=G.RESCALE, inp=[ptr(o0)], out=[ptr(o0)]),
                  dict(level=SQ, mode=G.RESCALE, inp=[ptr(o1)], out=[ptr(o1)])])
    sync()
    r0, r1 = host(o0)[:(SQ - 1) * N], host(o1)[:(SQ - 1) * N]

    # the oracle on the same keys and inputs
    for k, a, b in zip(gal, av, bv):
        octx.set_key(k, host(a), host(b))
    s_h, a_h, b_h = host(ds), host(da), host(db)
    w0, w1 = octx.encrypt(SQ, mx, a_h[:SQ * N], b_h[:SQ * N], seed=303)
    assert np.array_equal(host(c0), w0) and np.array_equal(host(c1), w1)
    want_diag = []
    for j in range(S):
        parts = []
        for t in range(SQ):
            q = int(Q[t])
            fr, fp, _, _, _, _ = O.root_tables(N, q, int(octx.roots[t]))
            parts.append(O.ntt(np.array([v % q for v in md[j].tolist()], np.uint64), N, q, fr, fp))
        want_diag.append(np.concatenate(parts))
    for j in (0, 1, 255, 511):
        assert np.array_equal(host(dev_diag[j]), want_diag[j]), j
    e0, e1 = octx.lintrans_bsgs(SQ, S, 1, w0, w1, want_diag)
    assert np.array_equal(pre0, e0) and np.array_equal(pre1, e1)
    f0, f1 = e0.copy(), e1.copy()
    f0 = octx.rescale(SQ, f0)[:(SQ - 1) * N]
    f1 = octx.rescale(SQ, f1)[:(SQ - 1) * N]
    assert np.array_equal(r0, f0) and np.array_equal(r1, f1)

    # decrypt at the reduced level, decode, compare with U x
    dec = np.zeros((1, N), np.int64)
    G.check(G.lib().gpufhe_decrypt_batch(g.h, 1, parr([o0]), parr([o1]), ptr(ds), dec.ctypes.data, None))
    y = enc.decode(dec[0], DELTA * DELTA / float(Q[SQ - 1]))
    err = np.max(np.abs(y.real - (U @ x.real)))
    assert err < 5e-3, err
