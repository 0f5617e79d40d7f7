"""CPU oracle vs golden digests produced by the reference library itself
(tests/golden/make_golden.py ran the reference's sources rebuilt for sm_100a).
Every array is regenerated from the recorded seeds and compared by SHA-256."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    p = os.path.join(HERE, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated yet")
    with open(p) as f:
        return json.load(f)


def same(a, d):
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.tobytes()).hexdigest() == d["sha256"] and a.size == d["words"]


def message(seed, n, delta_bits=50):
    u = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    return np.rint(u * float(1 << delta_bits)).astype(np.int64)


def test_config1_golden():
    g = load("config1_golden.json")
    p = g["params"]
    n, L, K, sigma = p["n"], p["L"], p["K"], p["sigma"]
    Q, P = np.array(p["Q"], np.uint64), np.array(p["P"], np.uint64)
    assert np.array_equal(Q, np.concatenate([O.native_primes(1, 60, n), O.native_primes(L - 1, 50, n, avoid=[int(Q[0])])]))
    ctx = O.Ctx(n, Q, P, -(-L // p["numPart"]), roots=np.array(p["roots"], np.uint64))
    T = L + K
    s, a, b = ctx.keygen(T, sigma=sigma, seed=101)
    assert same(s, g["s_qp"]) and same(a, g["pkA_qp"]) and same(b, g["pkB_qp"])
    s2 = np.array([(int(v) * int(v)) % int(ctx.QP[i // n]) for i, v in enumerate(s)], np.uint64)
    av, bv = ctx.evalkeygen(s, s2, a, b, sigma=sigma, seed=202)
    assert same(av, g["evk_av"]) and same(bv, g["evk_bv"])
    ctx.set_key(0, av, bv)
    sq, qa, qb = ctx.keygen(L, sigma=sigma, seed=101)
    c0a, c1a = ctx.encrypt(L, message(11, n), qa, qb, sigma=sigma, seed=303)
    c0b, c1b = ctx.encrypt(L, message(12, n), qa, qb, sigma=sigma, seed=304)
    for arr, key in ((c0a, "c0a"), (c1a, "c1a"), (c0b, "c0b"), (c1b, "c1b")):
        assert same(arr, g[key]), key
    o0, o1 = ctx.evalmult_rescale(L, c0a, c1a, c0b, c1b)
    assert same(o0, g["evalmult_rescale_out0"]) and same(o1, g["evalmult_rescale_out1"])
    rng = np.random.default_rng(88)
    ks_in = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    k0, k1 = ctx.keyswitch(L, ks_in)
    assert same(k0, g["keyswitch_ba0"]) and same(k1, g["keyswitch_ba1"])
    sr, _, _ = ctx.keygen(L - 1, sigma=sigma, seed=101)
    assert same(ctx.decrypt(L - 1, o0, o1, sr), g["decrypt_tower0"])
    # decryption matches the exact negacyclic product at scale 2^100 / q_last
    m1, m2 = message(11, n), message(12, n)
    dec = ctx.decrypt_crt(L - 1, o0, o1, sr)
    ql = int(Q[L - 1])
    for k in (0, 1, 777, n - 1):
        exact = 0
        for i in range(n):
            j = k - i
            exact += int(m1[i]) * int(m2[j]) if j >= 0 else -int(m1[i]) * int(m2[j + n])
        assert abs(dec[k] - exact / ql) < 2 ** 20, k


def test_rotation_golden():
    g = load("rotation_golden.json")
    p = g["params"]
    n, L, K, sigma = p["n"], p["L"], p["K"], p["sigma"]
    Q, P = np.array(p["Q"], np.uint64), np.array(p["P"], np.uint64)
    ctx = O.Ctx(n, Q, P, -(-L // p["numPart"]))
    T = L + K
    s, a, b = ctx.keygen(T, sigma=sigma, seed=101)
    rng = np.random.default_rng(505)
    c0 = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    c1 = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    for k in p["galois"]:
        d = g[f"k{k}"]
        sa = ctx.automorph_eval(T, k, s)
        assert same(sa, d["sigma_s"])
        av, bv = ctx.evalkeygen(s, sa, a, b, sigma=sigma, seed=404)
        assert same(av, d["av"]) and same(bv, d["bv"])
        ctx.set_key(k, av, bv)
        r0, r1 = ctx.rotate(L, k, c0, c1, k)
        assert same(r0, d["rot0"]) and same(r1, d["rot1"])


def test_encode_golden():
    """Canonical encode / decode (reference encode.cpp:13-44): the oracle's
    coefficients and decoded doubles equal the reference's, bit for bit."""
    from golden.make_golden import slots
    g = load("encode_golden.json")
    for c in g["cases"]:
        n, d = c["n"], float(2.0 ** c["delta_bits"])
        re, im = slots(c["seed"], n, c["real_only"])
        m = O.encode(re + 1j * im, n, d)
        assert same(m, c["m"]), c
        z = O.decode(m, n, d)
        assert same(np.ascontiguousarray(z.real), c["dec_re"]) and same(np.ascontiguousarray(z.imag), c["dec_im"]), c
