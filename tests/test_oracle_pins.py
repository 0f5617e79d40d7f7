"""Pins the CPU oracle against the reference's own host sources (compiled by
oracle/build_ref.sh) and against the reference's known-answer tests."""
import numpy as np
import pytest

import oracle as O

REF = O.load_ref_host()
needs_ref = pytest.mark.skipif(REF is None, reason="oracle/_ref/libref_host.so not built")


@needs_ref
@pytest.mark.parametrize("count,bits,n", [(4, 50, 1024), (3, 60, 4096), (12, 50, 65536), (3, 60, 65536), (4, 35, 32768)])
def test_native_primes_match_reference(count, bits, n):
    a = O.native_primes(count, bits, n)
    b = np.zeros(count, np.uint64)
    assert REF.ref_native_primes(b, count, bits, n, None, 0) == 0
    assert np.array_equal(a, b)
    for q in a:
        assert int(q) % (2 * n) == 1


@needs_ref
@pytest.mark.parametrize("n", [1024, 4096, 65536])
def test_native_root_matches_reference(n):
    for q in O.native_primes(3, 50, n):
        r = O.native_root(n, int(q))
        assert r == REF.ref_native_root(n, int(q))
        assert pow(r, n, int(q)) == int(q) - 1


@needs_ref
@pytest.mark.parametrize("L", [2, 4, 7, 12])
def test_rescale_consts_match_reference(L):
    n = 4096
    mods = np.concatenate([O.native_primes(1, 60, n), O.native_primes(L - 1, 50, n)])
    s1, s2 = O.rescale_consts(mods, L - 1)
    r1, r2 = np.zeros(L - 1, np.uint64), np.zeros(L - 1, np.uint64)
    REF.ref_rescale_consts(r1, r2, mods, L, L - 1)
    assert np.array_equal(s1, r1) and np.array_equal(s2, r2)
    # definition: s2 = floor(Ql * (Ql^-1 mod ql) / ql) mod q_i, big-int check
    Ql = 1
    for q in mods[: L - 1]:
        Ql *= int(q)
    ql = int(mods[L - 1])
    D = Ql * pow(Ql % ql, -1, ql) // ql
    assert [D % int(q) for q in mods[: L - 1]] == [int(x) for x in s2]


@needs_ref
@pytest.mark.parametrize("L,alpha", [(4, 2), (12, 3), (9, 3), (5, 3), (11, 4), (3, 3), (30, 10)])
def test_ks_constants_match_reference(L, alpha):
    n = 1024
    Q = np.concatenate([O.native_primes(1, 60, n), O.native_primes(L - 1, 50, n)])
    P = O.native_primes(3, 60, n, avoid=list(Q))
    numPart = -(-L // alpha)
    a = O.ks_constants(Q, P, alpha)
    b = np.zeros_like(a)
    ref_alpha = REF.ref_ks_constants(b, Q, L, P, len(P), numPart)
    if ref_alpha == alpha:
        assert np.array_equal(a, b)
    else:
        # the reference derives alpha = ceil(L / numPart): a full-QP key made
        # with digit width alpha no longer lines up at this level
        assert ref_alpha < alpha


def test_ks_constants_big_int_definition():
    n = 1024
    Q = np.concatenate([O.native_primes(1, 60, n), O.native_primes(6, 50, n)])
    P = O.native_primes(2, 60, n, avoid=list(Q))
    alpha, L, K = 3, 7, 2
    flat = O.ks_constants(Q, P, alpha)
    off = 0
    Qi = [int(x) for x in Q]
    Pi = [int(x) for x in P]
    for p in range(-(-L // alpha)):
        st, sp = alpha * p, min(alpha, L - alpha * p)
        src = Qi[st:st + sp]
        compl = [q for i, q in enumerate(Qi[:L]) if not (st <= i < st + sp)] + Pi
        sc = len(compl)
        prod = 1
        for q in src:
            prod *= q
        qhatinv = flat[off:off + sp]; off += 3 * sp
        qhatmodp = flat[off:off + sp * sc].reshape(sp, sc); off += sp * sc
        assert [int(x) for x in flat[off:off + sc]] == compl; off += 3 * sc
        for i, q in enumerate(src):
            assert int(qhatinv[i]) == pow((prod // q) % q, -1, q)
            for j, m in enumerate(compl):
                assert int(qhatmodp[i, j]) == (prod // q) % m


def test_barrett_u128_is_exact():
    rng = np.random.default_rng(1)
    for bits in (35, 50, 60):
        q = int(O.native_primes(1, bits, 1024)[0])
        mu = ((1 << 128) - 1) // q
        for _ in range(2000):
            a = int(rng.integers(0, 1 << 62)) * int(rng.integers(0, 1 << 62)) * int(rng.integers(1, 16))
            a &= (1 << 128) - 1
            r = O.lib().orc_barrett_u128(a & (2**64 - 1), a >> 64, q, mu & (2**64 - 1), mu >> 64)
            assert r == a % q


@pytest.mark.parametrize("n", [16, 256, 1024])
def test_ntt_is_negacyclic_evaluation(n):
    q = int(O.native_primes(1, 50, n)[0])
    psi = O.native_root(n, q)
    fr, fp, ir, ip, ni, nip = O.root_tables(n, q, psi)
    rng = np.random.default_rng(n)
    x = rng.integers(0, q, n, dtype=np.uint64)
    y = O.ntt(x, n, q, fr, fp)
    logn = n.bit_length() - 1
    brv = lambda v: int(format(v, f"0{logn}b")[::-1], 2)
    xs = [int(v) for v in x]
    for j in range(0, n, max(1, n // 16)):
        e = 2 * brv(j) + 1
        w = pow(psi, e, q)
        acc, p = 0, 1
        for i in range(n):
            acc = (acc + xs[i] * p) % q
            p = p * w % q
        assert int(y[j]) == acc
    z = O.intt(y, n, q, ir, ip, ni, nip)
    assert np.array_equal(z, x)


def _small_chain(n, L=4, K=2, alpha=2, bitsQ=50):
    Q = np.concatenate([O.native_primes(1, 60, n), O.native_primes(L - 1, bitsQ, n)])
    P = O.native_primes(K, 60, n, avoid=list(Q))
    return Q, P, alpha


def _relin_ctx(n, L, K, alpha, bitsQ=50):
    Q, P, alpha = _small_chain(n, L, K, alpha, bitsQ)
    ctx = O.Ctx(n, Q, P, alpha)
    T = L + K
    s, pkA, pkB = ctx.keygen(T, seed=101)
    s2 = [(int(a) * int(a)) % int(ctx.QP[i // n]) for i, a in enumerate(s)]
    av, bv = ctx.evalkeygen(s, np.array(s2, np.uint64), pkA, pkB, seed=202)
    ctx.set_key(0, av, bv)
    return ctx


def test_evalmult_rescale_known_answer():
    """test_evalmult_rescale.cpp:82-93: (3-2x)(4+5x^2) recovered exactly."""
    n, L = 1024, 4
    ctx = _relin_ctx(n, L, 2, 2, bitsQ=35)
    sQ, pkA, pkB = ctx.keygen(L, seed=101)
    D = 1 << 25
    m1 = np.zeros(n, np.int64); m1[0], m1[1] = 3 * D, -2 * D
    m2 = np.zeros(n, np.int64); m2[0], m2[2] = 4 * D, 5 * D
    c0a, c1a = ctx.encrypt(L, m1, pkA, pkB, seed=303)
    c0b, c1b = ctx.encrypt(L, m2, pkA, pkB, seed=304)
    o0, o1 = ctx.evalmult_rescale(L, c0a, c1a, c0b, c1b)
    sR, _, _ = ctx.keygen(L - 1, seed=101)
    dec = ctx.decrypt(L - 1, o0, o1, sR)
    ql = int(ctx.Q[L - 1])
    got = [round(int(v) * ql / (D * D)) for v in dec]
    expect = [0] * n
    expect[0], expect[1], expect[2], expect[3] = 12, -8, 15, -10
    assert got == expect


def test_keyswitch_reuse_across_levels():
    """test_keyreuse.cpp: one full-QP key, delta = fullQ - L at every level."""
    n, fullQ, K, alpha = 1024, 6, 2, 2
    ctx = _relin_ctx(n, fullQ, K, alpha)
    D = 1 << 40
    for L in (6, 5, 4, 3):
        sQ, pkA, pkB = ctx.keygen(L, seed=101)
        m = np.zeros(n, np.int64); m[0], m[5] = 2 * D, -3 * D
        c0, c1 = ctx.encrypt(L, m, pkA, pkB, seed=505)
        o0, o1 = ctx.evalmult_rescale(L, c0, c1, c0, c1)
        sR, _, _ = ctx.keygen(L - 1, seed=101)
        dec = ctx.decrypt_crt(L - 1, o0, o1, sR)
        ql = int(ctx.Q[L - 1])
        got = [round(v * ql / (D * D)) for v in dec[:11]]
        assert got == [4, 0, 0, 0, 0, -12, 0, 0, 0, 0, 9], L


@needs_ref
@pytest.mark.parametrize("L", [2, 4, 7, 12, 24])
def test_library_rescale_consts_match_reference(L):
    """The library's own rescale constants (host code, no GPU call): s1 from
    the inverse of the dropped prime, s2 = q_i - s1 by the exact-division
    identity. Same values as the reference's params.cpp and as the big-integer
    definition floor(Ql * (Ql^-1 mod ql) / ql) mod q_i."""
    import gpufhe_b200 as G
    n = 1 << 14
    mods = np.concatenate([O.native_primes(1, 60, n), O.native_primes(L - 1, 50, n)])
    s1, s2 = np.zeros(L - 1, np.uint64), np.zeros(L - 1, np.uint64)
    assert G.lib().gpufhe_rescale_consts(s1.ctypes.data, s2.ctypes.data, mods.ctypes.data, L - 1) == 0
    r1, r2 = np.zeros(L - 1, np.uint64), np.zeros(L - 1, np.uint64)
    REF.ref_rescale_consts(r1, r2, mods, L, L - 1)
    assert np.array_equal(s1, r1) and np.array_equal(s2, r2)
    Ql = 1
    for q in mods[: L - 1]:
        Ql *= int(q)
    ql = int(mods[L - 1])
    D = Ql * pow(Ql % ql, -1, ql) // ql
    assert [D % int(q) for q in mods[: L - 1]] == [int(x) for x in s2]


def test_library_rescale_consts_reject_non_coprime():
    import gpufhe_b200 as G
    mods = np.array([97, 193, 97], np.uint64)
    s1, s2 = np.zeros(2, np.uint64), np.zeros(2, np.uint64)
    assert G.lib().gpufhe_rescale_consts(s1.ctypes.data, s2.ctypes.data, mods.ctypes.data, 2) == -1
    assert b"coprime" in G.lib().gpufhe_last_error()
