"""Key generation, eval-key generation, encryption and decryption on the GPU
(gpufhe_keygen / gpufhe_evalkeygen / gpufhe_encrypt_batch /
gpufhe_decrypt_batch / gpufhe_decrypt_crt_batch), bit-exact against the CPU
oracle's restatement of the reference's seeded routines (keygen.cpp:55-112,
evalkeygen.cpp:42-113, encdec.cpp:41-81) and, where the reference rebuild is
present, against the reference's own keygen_host / evalkeygen_host /
encrypt_host / decrypt_host. Keys made on the GPU then drive EvalMult+Rescale
and rotation to the oracle's bits."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from ckks_setup import chain, square_mod
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

REFG = O.load_ref_gpu()
N, FULLQ, K, ALPHA = 4096, 6, 3, 3
T = FULLQ + K


def parr(ts):
    return (C.c_void_p * len(ts))(*[ptr(t) for t in ts])


@pytest.fixture(scope="module")
def env():
    import gpufhe_b200 as G
    Q, P = chain(N, FULLQ, K)
    octx = O.Ctx(N, Q, P, ALPHA)
    g = G.Context(N, Q, P, ALPHA)
    ds, da, db = empty(T * N), empty(T * N), empty(T * N)
    G.check(G.lib().gpufhe_keygen(g.h, T, 0, 1, 3.19, 101, ptr(ds), ptr(da), ptr(db), None))
    one = (C.c_uint64 * 1)
    G.check(G.lib().gpufhe_evalkeygen(g.h, 1, one(0), one(0), one(202), ptr(ds), ptr(da), ptr(db), 1, 3.19,
                                      None, None, None))
    return dict(G=G, Q=Q, P=P, octx=octx, g=g, ds=ds, da=da, db=db)


@pytest.mark.parametrize("hw", [0, 64])
def test_keygen(env, hw):
    G, g, octx = env["G"], env["g"], env["octx"]
    ds, da, db = empty(T * N), empty(T * N), empty(T * N)
    G.check(G.lib().gpufhe_keygen(g.h, T, hw, 1, 3.19, 111, ptr(ds), ptr(da), ptr(db), None))
    O.set_hamming_weight(hw)
    try:
        s, a, b = octx.keygen(T, seed=111)
    finally:
        O.set_hamming_weight(0)
    assert np.array_equal(host(ds), s)
    assert np.array_equal(host(da), a)
    assert np.array_equal(host(db), b)
    if REFG is not None:
        rs, ra, rb = (np.zeros(T * N, np.uint64) for _ in range(3))
        REFG.refg_set_hw(hw)
        try:
            REFG.refg_keygen(N, octx.QP, T, octx.roots, 1, 3.19, 111, rs, ra, rb)
        finally:
            REFG.refg_set_hw(0)
        assert np.array_equal(host(ds), rs) and np.array_equal(host(db), rb)


def test_evalkeygen_relin_and_rotation(env):
    G, g, octx = env["G"], env["g"], env["octx"]
    s, a, b = host(env["ds"]), host(env["da"]), host(env["db"])
    gm2 = O.galois_element(-2, N)
    ids, gal, seeds = [0, 5, gm2], [0, 5, gm2], [202, 405, 406]
    dnum = -(-FULLQ // ALPHA)
    W = dnum * T * N
    avs, bvs = [empty(W) for _ in ids], [empty(W) for _ in ids]
    arr = lambda xs: (C.c_uint64 * len(xs))(*xs)
    G.check(G.lib().gpufhe_evalkeygen(g.h, len(ids), arr(ids), arr(gal), arr(seeds), ptr(env["ds"]),
                                      ptr(env["da"]), ptr(env["db"]), 1, 3.19, parr(avs), parr(bvs), None))
    for i, k in enumerate(gal):
        s_old = square_mod(s, octx.QP, N) if k == 0 else octx.automorph_eval(T, k, s)
        av, bv = octx.evalkeygen(s, s_old, a, b, seed=seeds[i])
        assert np.array_equal(host(avs[i]), av), k
        assert np.array_equal(host(bvs[i]), bv), k
        octx.set_key(ids[i], av, bv)
        if REFG is not None and k == 0:
            h = REFG.refg_create(N, env["Q"], FULLQ, env["P"], K, octx.roots)
            rav, rbv = np.zeros(W, np.uint64), np.zeros(W, np.uint64)
            REFG.refg_evalkeygen(h, dnum, s, s_old, a, b, 1, 3.19, seeds[i], rav, rbv)
            REFG.refg_destroy(h)
            assert np.array_equal(host(avs[i]), rav) and np.array_equal(host(bvs[i]), rbv)
    # the installed keys drive the batched pipeline to the oracle's bits
    rng = np.random.default_rng(9)
    L = FULLQ
    ins = [np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in env["Q"][:L]]) for _ in range(4)]
    d = [dev(x) for x in ins]
    out = [empty((L - 1) * N) for _ in range(2)]
    G.run_ops(g, [dict(level=L, mode=G.EVALMULT_RESCALE, inp=[ptr(t) for t in d], out=[ptr(t) for t in out])])
    sync()
    want = octx.evalmult_rescale(L, *ins)
    assert all(np.array_equal(host(o), w) for o, w in zip(out, want))
    r0, r1 = empty(L * N), empty(L * N)
    G.run_ops(g, [dict(level=L, mode=G.ROTATE, key_id=gm2, galois=gm2, inp=[ptr(d[0]), ptr(d[1])],
                       out=[ptr(r0), ptr(r1)])])
    sync()
    w0, w1 = octx.rotate(L, gm2, ins[0], ins[1], gm2)
    assert np.array_equal(host(r0), w0) and np.array_equal(host(r1), w1)


def test_encrypt_decrypt_batch(env):
    G, g, octx = env["G"], env["g"], env["octx"]
    s, a, b = host(env["ds"]), host(env["da"]), host(env["db"])
    L, count = FULLQ, 3
    rng = np.random.default_rng(17)
    m = rng.integers(-(1 << 40), 1 << 40, size=(count, N), dtype=np.int64)
    m[0, :4] = [np.iinfo(np.int64).min + 1, np.iinfo(np.int64).max, -1, 0]   # any int64 embeds
    seeds = [303, 304, 305]
    c0s, c1s = [empty(L * N) for _ in range(count)], [empty(L * N) for _ in range(count)]
    G.check(G.lib().gpufhe_encrypt_batch(g.h, count, L, np.ascontiguousarray(m).ctypes.data,
                                         (C.c_uint64 * count)(*seeds), ptr(env["da"]), ptr(env["db"]), 1, 3.19,
                                         parr(c0s), parr(c1s), None))
    for i in range(count):
        w0, w1 = octx.encrypt(L, m[i], a[:L * N], b[:L * N], seed=seeds[i])
        assert np.array_equal(host(c0s[i]), w0) and np.array_equal(host(c1s[i]), w1), i
        if REFG is not None:
            r0, r1 = np.zeros(L * N, np.uint64), np.zeros(L * N, np.uint64)
            REFG.refg_encrypt(N, octx.QP, L, octx.roots, np.ascontiguousarray(m[i]), a, b, 1, 3.19, seeds[i], r0, r1)
            assert np.array_equal(host(c0s[i]), r0) and np.array_equal(host(c1s[i]), r1), i
    dec = np.zeros((count, N), np.int64)
    G.check(G.lib().gpufhe_decrypt_batch(g.h, count, parr(c0s), parr(c1s), ptr(env["ds"]), dec.ctypes.data, None))
    for i in range(count):
        assert np.array_equal(dec[i], octx.decrypt(L, host(c0s[i]), host(c1s[i]), s)), i
    # exact CRT decryption: message plus small noise, and the oracle's big-integer CRT
    crt = np.zeros((count, N, 2), np.uint64)
    G.check(G.lib().gpufhe_decrypt_crt_batch(g.h, count, L, parr(c0s), parr(c1s), ptr(env["ds"]),
                                             crt.ctypes.data, None))
    for i in range(count):
        vals = [int(lo) | (int(hi) << 64) for lo, hi in crt[i]]
        vals = [v - (1 << 128) if v >= 1 << 127 else v for v in vals]
        want = octx.decrypt_crt(L, host(c0s[i]), host(c1s[i]), s)
        assert vals == want, i
        assert max(abs(v - int(x)) for v, x in zip(vals, m[i])) < 1 << 20


def test_decrypt_crt_after_evalmult(env):
    """128-bit coefficients: EvalMult+Rescale of two encryptions of messages
    near 2^60 gives coefficients near 2^76; the GPU CRT decryption equals the
    oracle's big-integer CRT."""
    G, g, octx = env["G"], env["g"], env["octx"]
    s = host(env["ds"])
    L = FULLQ
    rng = np.random.default_rng(23)
    m = rng.integers(-(1 << 60), 1 << 60, size=(2, N), dtype=np.int64)
    cts = []
    for i in range(2):
        c0, c1 = empty(L * N), empty(L * N)
        G.check(G.lib().gpufhe_encrypt_batch(g.h, 1, L, np.ascontiguousarray(m[i]).ctypes.data,
                                             (C.c_uint64 * 1)(700 + i), ptr(env["da"]), ptr(env["db"]), 1, 3.19,
                                             parr([c0]), parr([c1]), None))
        cts.append((c0, c1))
    out = [empty((L - 1) * N) for _ in range(2)]
    G.run_ops(g, [dict(level=L, mode=G.EVALMULT_RESCALE, inp=[ptr(cts[0][0]), ptr(cts[0][1]), ptr(cts[1][0]),
                                                              ptr(cts[1][1])], out=[ptr(t) for t in out])])
    sync()
    crt = np.zeros((1, N, 2), np.uint64)
    G.check(G.lib().gpufhe_decrypt_crt_batch(g.h, 1, L - 1, parr([out[0]]), parr([out[1]]), ptr(env["ds"]),
                                             crt.ctypes.data, None))
    vals = [int(lo) | (int(hi) << 64) for lo, hi in crt[0]]
    vals = [v - (1 << 128) if v >= 1 << 127 else v for v in vals]
    assert vals == octx.decrypt_crt(L - 1, host(out[0]), host(out[1]), s)
    assert max(abs(v) for v in vals) > 1 << 64


def test_bad_arguments(env):
    G, g = env["G"], env["g"]
    d = empty(T * N)
    assert G.lib().gpufhe_keygen(g.h, T + 1, 0, 1, 3.19, 1, ptr(d), ptr(d), ptr(d), None) != 0
    one = (C.c_uint64 * 1)(4)   # even Galois element
    assert G.lib().gpufhe_evalkeygen(g.h, 1, one, one, one, ptr(d), ptr(d), ptr(d), 1, 3.19, None, None,
                                     None) != 0
