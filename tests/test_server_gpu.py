"""Continuous-batching server (gpufhe_server_* C ABI).

Every request's result is the same, bit for bit, served in the mix (uneven
ring sizes, levels and chains batched together) and alone (the plain
one-request-at-a-time form), and equals the oracle's chain of
EvalMult+Rescale (the ciphertext times itself) and rotations. Admission under
a small HBM budget, seeded device inputs and error returns are covered too.
"""
import numpy as np
import pytest

import oracle as O
from ckks_setup import Setup

pytestmark = pytest.mark.gpu

EMR, ROT = 0, 2


@pytest.fixture(scope="module")
def G():
    import gpufhe_b200
    return gpufhe_b200


@pytest.fixture(scope="module")
def setups():
    a = Setup(4096, 10, K=3, alpha=3, rot_ks=(5, O.galois_element(-2, 4096)))
    b = Setup(2048, 8, K=2, alpha=4, rot_ks=(O.galois_element(1, 2048),), seed=77)
    return [a, b]


@pytest.fixture(scope="module")
def gctxs(setups):
    return [s.gpu_context() for s in setups]


def make_trace(setups, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        c = int(rng.integers(0, len(setups)))
        S = setups[c]
        L = int(rng.integers(3, S.fullQ + 1))
        depth = int(rng.integers(1, min(4, L - 1) + 1))
        rots = [int(k) for k in rng.choice(list(S.rot), size=int(rng.integers(0, 4)))]
        ops = [(EMR, 0)] * depth + [(ROT, k) for k in rots]
        order = rng.permutation(len(ops))
        ops = [ops[j] for j in order]
        c0, c1 = S.rand_ct(rng, L)
        reqs.append(dict(ctx=c, level=L, ops=ops, h_in=np.concatenate([c0, c1]), arrival=i * 2e-4))
    return reqs


def final_level(r):
    return r["level"] - sum(1 for m, _ in r["ops"] if m == EMR)


def run(G, gctxs, setups, reqs, plain=False, budget=None, seeded=False, tune=0, max_active=0):
    resident = sum(g.resident_bytes() for g in gctxs)
    srv = G.Server(gctxs, budget or resident + (1 << 30), max_active=max_active, plain=plain)
    if tune:
        assert srv.tune(tune) > 0
    outs = []
    for i, r in enumerate(reqs):
        n = setups[r["ctx"]].n
        out = np.zeros(2 * final_level(r) * n, np.uint64)
        srv.submit(r["ctx"], r["level"], r["ops"], arrival_s=r["arrival"], seed=1000 + i,
                   h_in=None if seeded else r["h_in"], h_out=out)
        outs.append(out)
    srv.start()
    srv.drain(300.0)
    st, rec = srv.stats(), srv.records()
    srv.close()
    return outs, st, rec


def oracle_chain(S, r):
    n, L = S.n, r["level"]
    c0, c1 = r["h_in"][: L * n].copy(), r["h_in"][L * n:].copy()
    for m, k in r["ops"]:
        if m == EMR:
            c0, c1 = S.octx.evalmult_rescale(L, c0, c1, c0, c1)
            L -= 1
        else:
            c0, c1 = S.octx.rotate(L, k, c0, c1, k)
    return np.concatenate([c0[: L * n], c1[: L * n]])


def test_served_equals_alone_and_oracle(G, setups, gctxs):
    reqs = make_trace(setups, 24, seed=5)
    served, st, rec = run(G, gctxs, setups, reqs)
    alone, st1, _ = run(G, gctxs, setups, reqs, plain=True)
    nops = sum(len(r["ops"]) for r in reqs)
    assert st["completed"] == len(reqs) and st["ops"] == nops
    assert st["emr_ops"] == sum(1 for r in reqs for m, _ in r["ops"] if m == EMR)
    assert st["max_batch"] > 1          # requests really were batched together
    assert st1["max_batch"] == 1 and st1["peak_active"] == 1
    for i, r in enumerate(reqs):
        assert np.array_equal(served[i], alone[i]), i
    for i, r in enumerate(reqs[:8]):
        assert np.array_equal(served[i], oracle_chain(setups[r["ctx"]], r)), i
    for x in rec:
        assert x["t_admit"] >= x["t_arrival"] - 1e-9
        assert x["t_finish"] >= x["t_admit"] - 1e-3


def test_budget_admission(G, setups, gctxs):
    reqs = make_trace(setups, 10, seed=9)
    for r in reqs:
        r["arrival"] = 0.0
    resident = sum(g.resident_bytes() for g in gctxs)
    srv = G.Server(gctxs, resident + (1 << 30))
    sizes = [srv.request_bytes(r["ctx"], r["level"]) for r in reqs]
    srv.close()
    budget = resident + 2 * max(sizes) + 4096
    assert sum(sizes) > budget - resident        # the whole trace does not fit at once
    small, st, _ = run(G, gctxs, setups, reqs, budget=budget)
    big, _, _ = run(G, gctxs, setups, reqs)
    assert st["completed"] == len(reqs)
    assert st["peak_bytes"] <= st["arena_bytes"] <= budget - resident
    assert st["peak_active"] < len(reqs)         # admission waited for memory
    for i in range(len(reqs)):
        assert np.array_equal(small[i], big[i]), i


def test_active_cap(G, setups, gctxs):
    """max_active bounds the requests admitted at once (an option beside the
    HBM budget); the results are the same bits as uncapped."""
    reqs = make_trace(setups, 12, seed=21)
    for r in reqs:
        r["arrival"] = 0.0
    capped, st, rec = run(G, gctxs, setups, reqs, max_active=3)
    free, _, _ = run(G, gctxs, setups, reqs)
    assert st["completed"] == len(reqs) and st["peak_active"] == 3 and st["max_batch"] > 1
    for i in range(len(reqs)):
        assert np.array_equal(capped[i], free[i]), i
    admits = sorted(x["t_admit"] for x in rec)
    finishes = sorted(x["t_finish"] for x in rec)
    assert admits[3] >= finishes[0] - 1e-3     # the fourth admission waited for a finish


def test_seeded_inputs_same_alone_and_mixed(G, setups, gctxs):
    reqs = make_trace(setups, 12, seed=13)
    served, _, _ = run(G, gctxs, setups, reqs, seeded=True)
    alone, _, _ = run(G, gctxs, setups, reqs, plain=True, seeded=True)
    for i in range(len(reqs)):
        assert np.array_equal(served[i], alone[i]), i
        assert served[i].any()


def test_submit_errors(G, setups, gctxs):
    resident = sum(g.resident_bytes() for g in gctxs)
    srv = G.Server(gctxs, resident + (64 << 20))
    with pytest.raises(G.GpuFheError):
        srv.submit(0, 2, [(EMR, 0), (EMR, 0)])          # second EvalMult+Rescale at level 1
    with pytest.raises(G.GpuFheError):
        srv.submit(0, 4, [(ROT, 7)])                    # no key for Galois element 7
    with pytest.raises(G.GpuFheError):
        srv.submit(0, 10, [(EMR, 0)] * 2 + [(ROT, 4)])  # even Galois element
    srv.close()
    with pytest.raises(G.GpuFheError):
        G.Server(gctxs, resident // 2)                  # budget below the resident tables


def test_tuned_server_same_bits(G, setups, gctxs):
    """Schedules picked by the server's autotuner give the same outputs."""
    reqs = make_trace(setups, 10, seed=21)
    base, _, _ = run(G, gctxs, setups, reqs)
    tuned, st, _ = run(G, gctxs, setups, reqs, tune=16)
    assert st["completed"] == len(reqs)
    for i in range(len(reqs)):
        assert np.array_equal(base[i], tuned[i]), i
