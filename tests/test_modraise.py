"""ModRaise: a ciphertext at tower q0 alone lifted to L towers
(gpufhe_modraise_batch), the first step of bootstrapping.

* CPU: the oracle's restatement of the reference's host sequence
  (tests/test_modraise.cpp:50-58) passes the reference test's own gate on
  its own parameters (n = 1024, three 40-bit primes, scale 2^25): the raised
  ciphertext's exact CRT decryption is congruent, coefficient by coefficient,
  to the tower-0 decryption mod q0, and differs from it somewhere (the q0*I
  term EvalMod removes).
* GPU: the batched entry equals the oracle bit for bit (several ciphertexts
  per call, an output aliasing its input, the benchmark's N = 2^16 chain),
  and equals the reference library's own decrypt_host + pt_to_eval_host
  composition where that rebuild is present.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from gpu_util import dev, empty, host, ptr, sync

N, L = 1024, 3


def small_chain():
    Q = O.native_primes(L, 40, N)
    P = O.native_primes(1, 60, N, avoid=list(Q))
    return Q, P


def encrypted_sine(octx):
    """The reference test's input: slots 0.4 sin(0.02 i) at scale 2^25,
    encrypted at tower q0 under the secret drawn with seed 101."""
    s1, a1, b1 = octx.keygen(1, seed=101)
    z = (0.4 * np.sin(0.02 * np.arange(N // 2))).astype(np.complex128)
    m = O.encode(z, N, 2.0 ** 25)
    c0, c1 = octx.encrypt(1, m, a1, b1, seed=303)
    return s1, c0, c1


def test_oracle_modraise_meets_the_reference_gate():
    Q, P = small_chain()
    octx = O.Ctx(N, Q, P, L)
    s1, c0, c1 = encrypted_sine(octx)
    sL, _, _ = octx.keygen(L, seed=101)           # same secret over all L towers
    dec1 = octx.decrypt(1, c0, c1, s1)
    r0, r1 = octx.modraise(L, c0, c1)
    assert np.array_equal(r0[:N], c0[:N]) and np.array_equal(r1[:N], c1[:N])   # tower 0 unchanged
    full = octx.decrypt_crt(L, r0, r1, sL)
    q0 = int(Q[0])
    diffs = [full[k] - int(dec1[k]) for k in range(N)]
    assert all(d % q0 == 0 for d in diffs)
    assert any(d != 0 for d in diffs)


def parr(ts):
    return (C.c_void_p * len(ts))(*[ptr(t) for t in ts])


def raise_on_gpu(G, g, towers, ins, outs):
    G.check(G.lib().gpufhe_modraise_batch(g.h, len(ins), towers, parr([a for a, _ in ins]), parr([b for _, b in ins]),
                                          parr([a for a, _ in outs]), parr([b for _, b in outs]), None))
    sync()


@pytest.mark.gpu
def test_modraise_batch_matches_oracle_and_reference():
    import gpufhe_b200 as G
    Q, P = small_chain()
    octx = O.Ctx(N, Q, P, L)
    g = G.Context(N, Q, P, L)
    rng = np.random.default_rng(5)
    s1, c0, c1 = encrypted_sine(octx)
    cts = [(c0[:N], c1[:N])] + [(rng.integers(0, int(Q[0]), N, dtype=np.uint64),
                                 rng.integers(0, int(Q[0]), N, dtype=np.uint64)) for _ in range(4)]
    ins = [(dev(a), dev(b)) for a, b in cts]
    outs = [(empty(L * N), empty(L * N)) for _ in cts]
    raise_on_gpu(G, g, L, ins, outs)
    want = [octx.modraise(L, a, b) for a, b in cts]
    for (o0, o1), (w0, w1) in zip(outs, want):
        assert np.array_equal(host(o0), w0) and np.array_equal(host(o1), w1)

    # in place: the output buffer holds the input in its first tower
    buf = [(dev(np.concatenate([a, np.zeros((L - 1) * N, np.uint64)])),
            dev(np.concatenate([b, np.zeros((L - 1) * N, np.uint64)]))) for a, b in cts[:2]]
    raise_on_gpu(G, g, L, buf, buf)
    for (o0, o1), (w0, w1) in zip(buf, want[:2]):
        assert np.array_equal(host(o0), w0) and np.array_equal(host(o1), w1)

    # fewer towers than the chain holds
    two = [(empty(2 * N), empty(2 * N))]
    raise_on_gpu(G, g, 2, ins[:1], two)
    w0, w1 = octx.modraise(2, *cts[0])
    assert np.array_equal(host(two[0][0]), w0) and np.array_equal(host(two[0][1]), w1)

    with pytest.raises(G.GpuFheError):
        raise_on_gpu(G, g, L + 1, ins[:1], outs[:1])

    refg = O.load_ref_gpu()
    if refg is None:
        return
    zero = np.zeros(N, np.uint64)
    roots = octx.roots
    for (a, b), (w0, w1) in zip(cts, want):
        got = []
        for comp in (a, b):       # test_modraise.cpp:50-58 on the reference library
            coeff = np.zeros(N, np.int64)
            refg.refg_decrypt(N, Q[:1].copy(), 1, roots[:1].copy(), np.ascontiguousarray(comp), zero, zero, coeff)
            out = np.zeros(L * N, np.uint64)
            refg.refg_pt_to_eval(N, L, Q, roots[:L].copy(), coeff, out)
            got.append(out)
        assert np.array_equal(got[0], w0) and np.array_equal(got[1], w1)


@pytest.mark.gpu
def test_modraise_full_size():
    """The benchmark's chain (N = 2^16, one 60-bit and eleven 50-bit primes):
    a batch of 8 ciphertexts raised to all 12 towers, two checked against the
    oracle and the rest against a batch of one."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench as B
    import gpufhe_b200 as G
    n = 1 << B.N_LOG
    Q, P = B.chain(G.native_primes, n)
    g = G.Context(n, Q, P, B.ALPHA)
    octx = O.Ctx(n, Q, P, B.ALPHA)
    rng = np.random.default_rng(17)
    cts = [(rng.integers(0, int(Q[0]), n, dtype=np.uint64), rng.integers(0, int(Q[0]), n, dtype=np.uint64))
           for _ in range(8)]
    ins = [(dev(a), dev(b)) for a, b in cts]
    Lf = B.FULLQ
    outs = [(empty(Lf * n), empty(Lf * n)) for _ in cts]
    raise_on_gpu(G, g, Lf, ins, outs)
    for i in range(2):
        w0, w1 = octx.modraise(Lf, *cts[i])
        assert np.array_equal(host(outs[i][0]), w0) and np.array_equal(host(outs[i][1]), w1)
    for i in range(2, 8):
        one = [(empty(Lf * n), empty(Lf * n))]
        raise_on_gpu(G, g, Lf, ins[i:i + 1], one)
        assert np.array_equal(host(one[0][0]), host(outs[i][0]))
        assert np.array_equal(host(one[0][1]), host(outs[i][1]))
