"""The GPU pipeline against the golden digests the reference library produced
(tests/golden/*.json): config-1 EvalMult+Rescale and keyswitch, and rotations,
computed by the batched C ABI on the B200 and compared by SHA-256. Inputs
and keys are regenerated from the recorded seeds by the oracle's harness
(itself pinned to the same digests on the CPU)."""
import numpy as np
import pytest

import oracle as O
from gpu_util import dev, empty, host, ptr, sync
from test_golden import load, message, same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gpufhe_b200
    return gpufhe_b200


def test_config1_golden_on_gpu(G):
    g = load("config1_golden.json")
    p = g["params"]
    n, L, K, sigma = p["n"], p["L"], p["K"], p["sigma"]
    Q, P = np.array(p["Q"], np.uint64), np.array(p["P"], np.uint64)
    roots = np.array(p["roots"], np.uint64)
    alpha = -(-L // p["numPart"])
    octx = O.Ctx(n, Q, P, alpha, roots=roots)
    s, a, b = octx.keygen(L + K, sigma=sigma, seed=101)
    s2 = np.array([(int(v) * int(v)) % int(octx.QP[i // n]) for i, v in enumerate(s)], np.uint64)
    av, bv = octx.evalkeygen(s, s2, a, b, sigma=sigma, seed=202)
    assert same(av, g["evk_av"]) and same(bv, g["evk_bv"])
    _, qa, qb = octx.keygen(L, sigma=sigma, seed=101)
    c0a, c1a = octx.encrypt(L, message(11, n), qa, qb, sigma=sigma, seed=303)
    c0b, c1b = octx.encrypt(L, message(12, n), qa, qb, sigma=sigma, seed=304)
    gctx = G.Context(n, Q, P, alpha, roots=roots)
    gctx.set_key(0, av, bv)
    ins = [dev(x) for x in (c0a, c1a, c0b, c1b)]
    o0, o1 = empty((L - 1) * n), empty((L - 1) * n)
    rng = np.random.default_rng(88)
    ks_in = dev(np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q]))
    k0, k1 = empty(L * n), empty(L * n)
    G.run_ops(gctx, [dict(level=L, inp=[ptr(x) for x in ins], out=[ptr(o0), ptr(o1)]),
                     dict(level=L, mode=G.KEYSWITCH, inp=[ptr(ks_in)], out=[ptr(k0), ptr(k1)])])
    sync()
    assert same(host(o0), g["evalmult_rescale_out0"]) and same(host(o1), g["evalmult_rescale_out1"])
    assert same(host(k0), g["keyswitch_ba0"]) and same(host(k1), g["keyswitch_ba1"])


def test_rotation_golden_on_gpu(G):
    g = load("rotation_golden.json")
    p = g["params"]
    n, L, K, sigma = p["n"], p["L"], p["K"], p["sigma"]
    Q, P = np.array(p["Q"], np.uint64), np.array(p["P"], np.uint64)
    alpha = -(-L // p["numPart"])
    octx = O.Ctx(n, Q, P, alpha)
    s, a, b = octx.keygen(L + K, sigma=sigma, seed=101)
    rng = np.random.default_rng(505)
    c0 = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    c1 = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q])
    gctx = G.Context(n, Q, P, alpha)
    d0, d1 = dev(c0), dev(c1)
    specs, outs = [], []
    for k in p["galois"]:
        av, bv = octx.evalkeygen(s, octx.automorph_eval(L + K, k, s), a, b, sigma=sigma, seed=404)
        gctx.set_key(k, av, bv)
        r0, r1 = empty(L * n), empty(L * n)
        outs.append((k, r0, r1))
        specs.append(dict(level=L, mode=G.ROTATE, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)],
                          out=[ptr(r0), ptr(r1)]))
    G.run_ops(gctx, specs)
    sync()
    for k, r0, r1 in outs:
        assert same(host(r0), g[f"k{k}"]["rot0"]) and same(host(r1), g[f"k{k}"]["rot1"]), k
