"""Generates tests/golden/*.json from the reference library itself.

Runs the reference's own sources rebuilt for sm_100a (oracle/_ref/
libref_gpu.so, see oracle/build_ref.sh) on a B200 and records SHA-256
digests (plus a few leading words) of every array of seeded
EvalMult+Rescale, keyswitch and rotation runs. tests/test_golden.py then
regenerates the same arrays with the CPU oracle and compares digests, which
pins the oracle to the reference without shipping megabytes of residues.

  python tests/golden/make_golden.py          (needs a CUDA GPU)
  python tests/golden/make_golden.py encode   (canonical encode / decode; host only)

Config-1 parameters: N = 2^15, Q = one 60-bit + three 50-bit primes,
P = two 60-bit primes, dnum = 2, scale 2^50, ternary secret, sigma 3.2,
messages round(u * 2^50) with u ~ U[-1, 1] (numpy default_rng(seed)).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402


def digest(a):
    a = np.ascontiguousarray(a)
    conv = float if a.dtype.kind == "f" else int
    return {"sha256": hashlib.sha256(a.tobytes()).hexdigest(), "head": [conv(x) for x in a.ravel()[:6]],
            "words": int(a.size)}


def message(seed, n, delta_bits=50):
    u = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    return np.rint(u * float(1 << delta_bits)).astype(np.int64)


def chain(n, L, K, bits0=60, bitsQ=50, bitsP=60):
    q0 = O.native_primes(1, bits0, n)
    Q = np.concatenate([q0, O.native_primes(L - 1, bitsQ, n, avoid=list(q0))]) if L > 1 else q0
    P = O.native_primes(K, bitsP, n, avoid=list(Q))
    return Q, P


def config1(R):
    n, L, K, numpart, sigma = 1 << 15, 4, 2, 2, 3.2
    Q, P = chain(n, L, K)
    QP = np.concatenate([Q, P])
    roots = np.array([O.native_root(n, int(q)) for q in QP], np.uint64)
    h = R.refg_create(n, Q, L, P, K, roots)
    T = L + K
    s, a, b = (np.zeros(T * n, np.uint64) for _ in range(3))
    R.refg_keygen(n, QP, T, roots, 1, sigma, 101, s, a, b)
    s2 = np.array([(int(v) * int(v)) % int(QP[i // n]) for i, v in enumerate(s)], np.uint64)
    av, bv = np.zeros(numpart * T * n, np.uint64), np.zeros(numpart * T * n, np.uint64)
    R.refg_evalkeygen(h, numpart, s, s2, a, b, 1, sigma, 202, av, bv)
    R.refg_set_key(h, 0, numpart, av, bv)
    sq, qa, qb = (np.zeros(L * n, np.uint64) for _ in range(3))
    R.refg_keygen(n, Q.copy(), L, roots[:L].copy(), 1, sigma, 101, sq, qa, qb)
    m1, m2 = message(11, n), message(12, n)
    c = [np.zeros(L * n, np.uint64) for _ in range(4)]
    R.refg_encrypt(n, Q.copy(), L, roots[:L].copy(), m1, qa, qb, 1, sigma, 303, c[0], c[1])
    R.refg_encrypt(n, Q.copy(), L, roots[:L].copy(), m2, qa, qb, 1, sigma, 304, c[2], c[3])
    o0, o1 = np.zeros((L - 1) * n, np.uint64), np.zeros((L - 1) * n, np.uint64)
    assert R.refg_evalmult_rescale(h, L, numpart, *c, o0, o1) == 0
    rng = np.random.default_rng(88)
    ks_in = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    k0, k1 = np.zeros(L * n, np.uint64), np.zeros(L * n, np.uint64)
    assert R.refg_keyswitch_resident(h, 0, L, numpart, ks_in, k0, k1) == 0
    sr, _, _ = (np.zeros((L - 1) * n, np.uint64) for _ in range(3))
    ra, rb = np.zeros((L - 1) * n, np.uint64), np.zeros((L - 1) * n, np.uint64)
    R.refg_keygen(n, Q[:L - 1].copy(), L - 1, roots[:L - 1].copy(), 1, sigma, 101, sr, ra, rb)
    dec = np.zeros(n, np.int64)
    R.refg_decrypt(n, Q[:L - 1].copy(), L - 1, roots[:L - 1].copy(), o0, o1, sr, dec)
    R.refg_destroy(h)
    out = {"params": {"n": n, "L": L, "K": K, "numPart": numpart, "sigma": sigma, "Q": [int(x) for x in Q],
                      "P": [int(x) for x in P], "roots": [int(x) for x in roots],
                      "seeds": {"keygen": 101, "evalkey": 202, "enc": [303, 304], "msg": [11, 12], "ks_input": 88}},
           "s_qp": digest(s), "pkA_qp": digest(a), "pkB_qp": digest(b), "evk_av": digest(av), "evk_bv": digest(bv),
           "c0a": digest(c[0]), "c1a": digest(c[1]), "c0b": digest(c[2]), "c1b": digest(c[3]),
           "evalmult_rescale_out0": digest(o0), "evalmult_rescale_out1": digest(o1),
           "keyswitch_ba0": digest(k0), "keyswitch_ba1": digest(k1), "decrypt_tower0": digest(dec)}
    return out


def rotation(R):
    n, L, K, numpart, sigma = 1 << 12, 6, 3, 2, 3.19
    Q, P = chain(n, L, K)
    QP = np.concatenate([Q, P])
    roots = np.array([O.native_root(n, int(q)) for q in QP], np.uint64)
    h = R.refg_create(n, Q, L, P, K, roots)
    T = L + K
    s, a, b = (np.zeros(T * n, np.uint64) for _ in range(3))
    R.refg_keygen(n, QP, T, roots, 1, sigma, 101, s, a, b)
    out = {"params": {"n": n, "L": L, "K": K, "numPart": numpart, "sigma": sigma, "Q": [int(x) for x in Q],
                      "P": [int(x) for x in P], "galois": [5, 2 * n - 1], "seeds": {"keygen": 101, "rotkey": 404,
                                                                                      "ct": 505}}}
    rng = np.random.default_rng(505)
    c0 = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    c1 = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    for key_id, k in enumerate((5, 2 * n - 1), start=1):
        sa = s.copy()
        R.refg_automorph_host(n, T, k, QP.copy(), roots.copy(), sa)
        av, bv = np.zeros(numpart * T * n, np.uint64), np.zeros(numpart * T * n, np.uint64)
        R.refg_evalkeygen(h, numpart, s, sa, a, b, 1, sigma, 404, av, bv)
        R.refg_set_key(h, key_id, numpart, av, bv)
        r0, r1 = c0.copy(), c1.copy()
        assert R.refg_rotate_device(h, key_id, L, numpart, k, r0, r1) == 0
        out[f"k{k}"] = {"sigma_s": digest(sa), "av": digest(av), "bv": digest(bv), "rot0": digest(r0),
                        "rot1": digest(r1)}
    R.refg_destroy(h)
    return out


def slots(seed, n, real_only=False):
    g = np.random.default_rng(seed)
    re = g.uniform(-1.0, 1.0, n // 2)
    im = np.zeros(n // 2) if real_only else g.uniform(-1.0, 1.0, n // 2)
    return re, im


# (n, seed, delta bits, real-only slots): canonical encode / decode cases
ENCODE_CASES = [(1 << 10, 11, 40, False), (1 << 12, 12, 40, False), (1 << 12, 13, 50, True),
                (1 << 13, 14, 30, False)]


def encode_cases(H):
    """The reference's encode_host / decode_host (encode.cpp:13-44, host-only
    code, oracle/_ref/libref_host.so) on seeded slots: digests of the
    coefficients and of the decoded slots."""
    out = {"cases": []}
    for n, seed, dbits, real in ENCODE_CASES:
        re, im = slots(seed, n, real)
        m = np.zeros(n, np.int64)
        H.ref_encode(m, re, im, n, float(2.0 ** dbits))
        zr, zi = np.zeros(n // 2), np.zeros(n // 2)
        H.ref_decode(zr, zi, m, n, float(2.0 ** dbits))
        out["cases"].append({"n": n, "seed": seed, "delta_bits": dbits, "real_only": real, "m": digest(m),
                             "dec_re": digest(zr), "dec_im": digest(zi)})
    return out


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "encode":   # host-only code, no GPU needed
        H = O.load_ref_host()
        if H is None:
            raise SystemExit("oracle/_ref/libref_host.so missing: run oracle/build_ref.sh")
        with open(os.path.join(HERE, "encode_golden.json"), "w") as f:
            json.dump(encode_cases(H), f, indent=1)
        print("encode golden vectors written")
        return
    R = O.load_ref_gpu()
    if R is None:
        raise SystemExit("oracle/_ref/libref_gpu.so missing: run oracle/build_ref.sh")
    with open(os.path.join(HERE, "config1_golden.json"), "w") as f:
        json.dump(config1(R), f, indent=1)
    with open(os.path.join(HERE, "rotation_golden.json"), "w") as f:
        json.dump(rotation(R), f, indent=1)
    out = os.environ.get("GOLDEN_COPY_DIR")      # optional second copy of the GPU-made vectors
    if out and os.path.isdir(out):
        import shutil
        for name in ("config1_golden.json", "rotation_golden.json"):
            shutil.copy(os.path.join(HERE, name), os.path.join(out, name))
    print("golden vectors written")


if __name__ == "__main__":
    main()
