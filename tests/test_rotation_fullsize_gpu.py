"""Rotation at the rotation workload's full size: N = 2^16, 10 towers
(1x60 + 9x50-bit), P = 3x60-bit, alpha = 3, real keys and a real encryption.

* Plain rotations (automorphism + Hybrid keyswitch with the index's own key)
  by steps from {+-1, ..., +-2^14}, and hoisted rotations of the same
  ciphertext (one shared ModUp), all in one batch: each equals the oracle's
  rotate / rotate_hoisted bit for bit (reference src/rotate.cpp:118-132,
  tests/test_rot_resident.cpp:123-210).
* Hoisted and plain rotation differ in the approximate ModUp error, so they
  agree only after decryption: the exact CRT decryptions (on the GPU) differ
  by at most the ModDown rounding bound 2 (K + 1) (1 + ||s||_1), and each
  decrypts to the rotated message m(X^k) within the noise.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from ckks_setup import Setup
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

N, L, K, ALPHA = 1 << 16, 10, 3, 3
STEPS = [1, -1, 1 << 7, -(1 << 3), 1 << 14, -(1 << 14)]   # +-2^14 share one Galois element at 2^15 slots
GALS = sorted({O.galois_element(r, N) for r in STEPS})


@pytest.fixture(scope="module")
def S():
    return Setup(N, L, K=K, alpha=ALPHA, rot_ks=GALS, seed=4242)


def parr(ts):
    return (C.c_void_p * len(ts))(*[ptr(t) for t in ts])


def coeff_automorphism(m, k):
    """m(X) -> m(X^k) in Z[X]/(X^N + 1)."""
    n = len(m)
    out = np.zeros(n, dtype=object)
    for j in range(n):
        e = (j * k) % (2 * n)
        if e < n:
            out[e] += int(m[j])
        else:
            out[e - n] -= int(m[j])
    return out


def test_rotations_fullsize(S):
    import gpufhe_b200 as G
    n = N
    g = S.gpu_context()
    rng = np.random.default_rng(99)
    m = rng.integers(-(1 << 40), 1 << 40, size=n, dtype=np.int64)
    c0, c1 = S.octx.encrypt(L, m, S.pkA[: L * n], S.pkB[: L * n], seed=909)
    d0, d1 = dev(c0), dev(c1)
    specs, plain_out, hoist_out = [], [], []
    for k in GALS:
        o = [empty(L * n), empty(L * n)]
        plain_out.append(o)
        specs.append(dict(level=L, mode=G.ROTATE, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)],
                          out=[ptr(o[0]), ptr(o[1])]))
    for k in GALS:
        o = [empty(L * n), empty(L * n)]
        hoist_out.append(o)
        specs.append(dict(level=L, mode=G.ROTATE_HOISTED, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)],
                          out=[ptr(o[0]), ptr(o[1])]))
    G.run_ops(g, specs)
    sync()
    # bits: plain against the oracle's rotation, hoisted against the oracle's hoisted rotation
    e0s, e1s = S.octx.rotate_hoisted(L, GALS, GALS, c0, c1)
    for i, k in enumerate(GALS):
        f0, f1 = S.octx.rotate(L, k, c0, c1, k)
        assert np.array_equal(host(plain_out[i][0]), f0) and np.array_equal(host(plain_out[i][1]), f1), k
        assert np.array_equal(host(hoist_out[i][0]), e0s[i]) and np.array_equal(host(hoist_out[i][1]), e1s[i]), k
    # decryptions: exact CRT decryption on the GPU of every plain and hoisted result
    ds = dev(S.s[: L * n])
    outs = plain_out + hoist_out
    crt = np.zeros((len(outs), n, 2), np.uint64)
    G.check(G.lib().gpufhe_decrypt_crt_batch(g.h, len(outs), L, parr([o[0] for o in outs]),
                                             parr([o[1] for o in outs]), ptr(ds), crt.ctypes.data, None))
    sync()
    lo, hi = crt[..., 0].astype(object), crt[..., 1].astype(object)
    vals = lo + hi * (1 << 64)
    vals = np.where(vals >= (1 << 127), vals - (1 << 128), vals)
    hw = int(np.count_nonzero(S.s[:n]))
    bound = 2 * (K + 1) * (1 + hw)
    for i, k in enumerate(GALS):
        dp, dh = vals[i], vals[len(GALS) + i]
        diff = max(abs(int(x)) for x in dp - dh)
        assert diff <= bound, (k, diff, bound)
        err = max(abs(int(x)) for x in dp - coeff_automorphism(m, k))
        assert err < 1 << 22, (k, err)
    g.close()
