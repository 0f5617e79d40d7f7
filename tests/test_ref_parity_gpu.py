"""Parity against the reference library itself: its own sources rebuilt for
sm_100a (oracle/_ref/libref_gpu.so, built by oracle/build_ref.sh), run on the
same seeded inputs as the CPU oracle and this library. Pins the oracle's
keygen / evalkeygen / encrypt / keyswitch / rescale / rotation against the
reference's routines, and this library against both."""
import numpy as np
import pytest

import oracle as O
from ckks_setup import chain, square_mod
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

REFG = O.load_ref_gpu()
needs_ref = pytest.mark.skipif(REFG is None, reason="oracle/_ref/libref_gpu.so not built")

N, FULLQ, K, ALPHA = 4096, 12, 3, 3
DNUM = -(-FULLQ // ALPHA)


@pytest.fixture(scope="module")
def env():
    Q, P = chain(N, FULLQ, K)
    octx = O.Ctx(N, Q, P, ALPHA)
    roots = octx.roots
    h = REFG.refg_create(N, Q, FULLQ, P, K, roots)
    QP = octx.QP
    T = FULLQ + K
    s, a, b = (np.zeros(T * N, np.uint64) for _ in range(3))
    REFG.refg_keygen(N, QP, T, roots, 1, 3.19, 101, s, a, b)
    av = np.zeros(DNUM * T * N, np.uint64)
    bv = np.zeros_like(av)
    s2 = square_mod(s, QP, N)
    REFG.refg_evalkeygen(h, DNUM, s, s2, a, b, 1, 3.19, 202, av, bv)
    REFG.refg_set_key(h, 0, DNUM, av, bv)
    octx.set_key(0, av, bv)
    import gpufhe_b200 as G
    g = G.Context(N, Q, P, ALPHA)
    g.set_key(0, av, bv)
    yield dict(Q=Q, P=P, octx=octx, roots=roots, h=h, s=s, a=a, b=b, av=av, bv=bv, s2=s2, G=G, g=g)
    REFG.refg_destroy(h)


def _ref_alpha_matches(L):
    numpart = -(-L // ALPHA)
    return -(-L // numpart) == ALPHA, numpart


@needs_ref
def test_keygen_evalkeygen_match_reference(env):
    octx = env["octx"]
    s, a, b = octx.keygen(FULLQ + K, seed=101)
    assert np.array_equal(s, env["s"]) and np.array_equal(a, env["a"]) and np.array_equal(b, env["b"])
    av, bv = octx.evalkeygen(s, env["s2"], a, b, seed=202)
    assert np.array_equal(av, env["av"]) and np.array_equal(bv, env["bv"])


@needs_ref
def test_encrypt_decrypt_match_reference(env):
    octx, Q, roots = env["octx"], env["Q"], env["roots"]
    L = 5
    sq, pa, pb = (np.zeros(L * N, np.uint64) for _ in range(3))
    REFG.refg_keygen(N, Q[:L].copy(), L, roots[:L].copy(), 1, 3.19, 101, sq, pa, pb)
    rng = np.random.default_rng(3)
    m = rng.integers(-(1 << 40), 1 << 40, N).astype(np.int64)
    c0, c1 = np.zeros(L * N, np.uint64), np.zeros(L * N, np.uint64)
    REFG.refg_encrypt(N, Q[:L].copy(), L, roots[:L].copy(), m, pa, pb, 1, 3.19, 303, c0, c1)
    e0, e1 = octx.encrypt(L, m, pa, pb, seed=303)
    assert np.array_equal(c0, e0) and np.array_equal(c1, e1)
    d = np.zeros(N, np.int64)
    REFG.refg_decrypt(N, Q[:L].copy(), L, roots[:L].copy(), c0, c1, sq, d)
    assert np.array_equal(d, octx.decrypt(L, c0, c1, sq))


@needs_ref
@pytest.mark.parametrize("L", [12, 9, 5, 3])
def test_keyswitch_matches_reference(env, L):
    ok, numpart = _ref_alpha_matches(L)
    assert ok
    rng = np.random.default_rng(88 + L)
    a = np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in env["Q"][:L]])
    r0, r1 = np.zeros(L * N, np.uint64), np.zeros(L * N, np.uint64)
    assert REFG.refg_keyswitch_resident(env["h"], 0, L, numpart, a, r0, r1) == 0
    h0, h1 = np.zeros(L * N, np.uint64), np.zeros(L * N, np.uint64)
    assert REFG.refg_keyswitch_core(env["h"], 0, L, numpart, a, h0, h1) == 0
    assert np.array_equal(r0, h0) and np.array_equal(r1, h1)          # reference: resident == host-orchestrated
    e0, e1 = env["octx"].keyswitch(L, a)
    assert np.array_equal(r0, e0) and np.array_equal(r1, e1)          # oracle == reference
    G = env["G"]
    da, b0, b1 = dev(a), empty(L * N), empty(L * N)
    G.run_ops(env["g"], [dict(level=L, mode=G.KEYSWITCH, inp=[ptr(da)], out=[ptr(b0), ptr(b1)])])
    assert np.array_equal(host(b0), r0) and np.array_equal(host(b1), r1)   # this library == reference


@needs_ref
@pytest.mark.parametrize("L", [12, 8, 6, 3])
def test_evalmult_rescale_matches_reference(env, L):
    ok, numpart = _ref_alpha_matches(L)
    assert ok
    rng = np.random.default_rng(7 + L)
    ins = [np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in env["Q"][:L]]) for _ in range(4)]
    r0, r1 = np.zeros((L - 1) * N, np.uint64), np.zeros((L - 1) * N, np.uint64)
    assert REFG.refg_evalmult_rescale(env["h"], L, numpart, *ins, r0, r1) == 0
    e0, e1 = env["octx"].evalmult_rescale(L, *ins)
    assert np.array_equal(r0, e0) and np.array_equal(r1, e1)
    G = env["G"]
    d = [dev(x) for x in ins]
    o0, o1 = empty((L - 1) * N), empty((L - 1) * N)
    G.run_ops(env["g"], [dict(level=L, inp=[ptr(x) for x in d], out=[ptr(o0), ptr(o1)])])
    assert np.array_equal(host(o0), r0) and np.array_equal(host(o1), r1)


@needs_ref
def test_rescale_matches_reference(env):
    L = 7
    ok, numpart = _ref_alpha_matches(L)
    rng = np.random.default_rng(17)
    c = np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in env["Q"][:L]])
    r = c.copy()
    assert REFG.refg_rescale(env["h"], L, numpart, r) == 0
    assert np.array_equal(r[: (L - 1) * N], env["octx"].rescale(L, c))


@needs_ref
@pytest.mark.parametrize("r", [1, -4])
def test_rotation_matches_reference(env, r):
    octx, Q, P, roots = env["octx"], env["Q"], env["P"], env["roots"]
    k = O.galois_element(r, N)
    T = FULLQ + K
    sa = env["s"].copy()
    REFG.refg_automorph_host(N, T, k, octx.QP.copy(), roots.copy(), sa)
    assert np.array_equal(sa, octx.automorph_eval(T, k, env["s"]))
    av = np.zeros(DNUM * T * N, np.uint64)
    bv = np.zeros_like(av)
    REFG.refg_evalkeygen(env["h"], DNUM, env["s"], sa, env["a"], env["b"], 1, 3.19, 900 + k, av, bv)
    REFG.refg_set_key(env["h"], 1, DNUM, av, bv)
    octx.set_key(k, av, bv)
    env["g"].set_key(k, av, bv)
    L = 9
    ok, numpart = _ref_alpha_matches(L)
    rng = np.random.default_rng(k)
    c0 = np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in Q[:L]])
    c1 = np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in Q[:L]])
    r0, r1 = c0.copy(), c1.copy()
    assert REFG.refg_rotate_device(env["h"], 1, L, numpart, k, r0, r1) == 0
    e0, e1 = octx.rotate(L, k, c0, c1, k)
    assert np.array_equal(r0, e0) and np.array_equal(r1, e1)
    G = env["G"]
    d0, d1, o0, o1 = dev(c0), dev(c1), empty(L * N), empty(L * N)
    G.run_ops(env["g"], [dict(level=L, mode=G.ROTATE, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)],
                              out=[ptr(o0), ptr(o1)])])
    assert np.array_equal(host(o0), r0) and np.array_equal(host(o1), r1)


@needs_ref
def test_reference_ntt_kernels_match(env):
    q = int(env["Q"][3])
    fr, fp, ir, ip, ni, nip = O.root_tables(N, q, int(env["roots"][3]))
    rng = np.random.default_rng(5)
    x = rng.integers(0, q, N, dtype=np.uint64)
    y = x.copy()
    assert REFG.refg_ntt(y, N, q, fr, fp, 0, 0, 0) == 0
    assert np.array_equal(y, O.ntt(x, N, q, fr, fp))
    z = y.copy()
    assert REFG.refg_ntt(z, N, q, ir, ip, 1, ni, nip) == 0
    assert np.array_equal(z, x)
