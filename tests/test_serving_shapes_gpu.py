"""The serving workload's own contexts, bit for bit against the oracle.

bench.py serves requests over three contexts (N = 2^14, 2^15, 2^16; Q = 1x60 +
23x50-bit, P = 8x60-bit, alpha = 8 so dnum = 3: a P5 key tile of 3 digits x 8
special rows and conversions 8 wide). This test builds those contexts with
the bench's own functions (same chains, same key material), serves a short
mixed trace through gpufhe_server_* (requests at the full 24 towers and at
low levels, with rotations, at every ring size, batched together), and
compares every result with the oracle's chain of EvalMult+Rescale and
rotations, and with the same request served alone (the plain form).
"""
import os
import sys

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402

EMR, ROT = 0, 2


@pytest.fixture(scope="module")
def shapes():
    """(gpu context, oracle context, n, Q, rotation Galois elements) per ring size."""
    import gpufhe_b200 as G
    out = []
    for lg in bench.SERVE_LOGNS:
        n, Q, P = bench.serving_chain(G.native_primes, lg)
        g = G.Context(n, Q, P, bench.SERVE_ALPHA)
        o = O.Ctx(n, Q, P, bench.SERVE_ALPHA)
        gals = []
        for k, av, bv in bench.serving_keys(lg):
            g.set_key(k, av, bv)
            o.set_key(k, av, bv)
            if k:
                gals.append(k)
        out.append((g, o, n, Q, gals))
    yield out
    for g, *_ in out:
        g.close()


def trace(shapes, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for c, (_, _, n, Q, gals) in enumerate(shapes):
        for L, depth, nrot in ((24, 2, 2), (int(rng.integers(5, 20)), 2, 1), (4, 3, 1)):
            ops = [(EMR, 0)] * depth + [(ROT, int(k)) for k in rng.choice(gals, nrot, replace=False)]
            ops = [ops[j] for j in rng.permutation(len(ops))]
            h_in = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q[:L]] * 2)
            reqs.append(dict(ctx=c, level=L, ops=ops, h_in=h_in))
    return reqs


def serve(G, shapes, reqs, plain):
    ctxs = [s[0] for s in shapes]
    resident = sum(g.resident_bytes() for g in ctxs)
    srv = G.Server(ctxs, resident + (8 << 30), plain=plain)
    outs = []
    for i, r in enumerate(reqs):
        n = shapes[r["ctx"]][2]
        fin = r["level"] - sum(1 for m, _ in r["ops"] if m == EMR)
        out = np.zeros(2 * fin * n, np.uint64)
        srv.submit(r["ctx"], r["level"], r["ops"], arrival_s=0.0, seed=7 + i, h_in=r["h_in"], h_out=out)
        outs.append(out)
    srv.start()
    srv.drain(600.0)
    st = srv.stats()
    srv.close()
    return outs, st


def oracle_chain(octx, n, r):
    L = r["level"]
    c0, c1 = r["h_in"][: L * n].copy(), r["h_in"][L * n:].copy()
    for m, k in r["ops"]:
        if m == EMR:
            c0, c1 = octx.evalmult_rescale(L, c0, c1, c0, c1)
            L -= 1
        else:
            c0, c1 = octx.rotate(L, k, c0, c1, k)
    return np.concatenate([c0[: L * n], c1[: L * n]])


def test_serving_contexts_bit_exact(shapes):
    import gpufhe_b200 as G
    reqs = trace(shapes, seed=2027)
    served, st = serve(G, shapes, reqs, plain=False)
    assert st["completed"] == len(reqs)
    assert st["max_batch"] > 1                 # requests of one ring size were batched together
    alone, st1 = serve(G, shapes, reqs, plain=True)
    assert st1["max_batch"] == 1
    for i, r in enumerate(reqs):
        _, octx, n, _, _ = shapes[r["ctx"]]
        want = oracle_chain(octx, n, r)
        assert np.array_equal(served[i], want), (i, n, r["level"], r["ops"])
        assert np.array_equal(alone[i], want), (i, n, r["level"])
