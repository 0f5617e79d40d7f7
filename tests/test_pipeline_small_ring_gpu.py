"""The batched pipeline at the smallest ring it supports, n = 2^10 (the
reference's own test ring, tests/test_c2s_engine.cpp:36): a mixed batch of
EvalMult+Rescale at uneven levels, keyswitch, rotation and hoisted rotation
equals the oracle in every P5 and P3 form."""
import numpy as np
import pytest

import oracle as O
from ckks_setup import Setup
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

N = 1024


@pytest.fixture(scope="module")
def S():
    return Setup(N, 6, K=2, alpha=2, rot_ks=(5, O.galois_element(3, N)))


@pytest.mark.parametrize("schedule", [0, 1, 2, 3, 8, 16, 7, 64, 67, 71, 192, 64 | 1 << 17, 64 | 1 << 18,
                                      64 | 1 << 17 | 1 << 18, 192 | 1 << 18])
def test_mixed_batch_small_ring(S, schedule):
    import gpufhe_b200 as G
    g = S.gpu_context()
    rng = np.random.default_rng(70 + schedule)
    keep, specs, want = [], [], []
    for L in (2, 4, 6):
        c0a, c1a = S.rand_ct(rng, L)
        c0b, c1b = S.rand_ct(rng, L)
        ins = [dev(x) for x in (c0a, c1a, c0b, c1b)]
        outs = [empty((L - 1) * N), empty((L - 1) * N)]
        keep += ins + outs
        specs.append(dict(level=L, inp=[ptr(x) for x in ins], out=[ptr(x) for x in outs]))
        want.append((outs, S.octx.evalmult_rescale(L, c0a, c1a, c0b, c1b)))
    c0, c1 = S.rand_ct(rng, 5)
    d0, d1 = dev(c0), dev(c1)
    keep += [d0, d1]
    k5, k3 = 5, O.galois_element(3, N)
    for mode, k in ((G.ROTATE, k5), (G.ROTATE_HOISTED, k5), (G.ROTATE_HOISTED, k3)):
        o0, o1 = empty(5 * N), empty(5 * N)
        keep += [o0, o1]
        specs.append(dict(level=5, mode=mode, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)], out=[ptr(o0), ptr(o1)]))
        want.append(([o0, o1], S.octx.rotate(5, k, c0, c1, k) if mode == G.ROTATE else None))
    e_h = S.octx.rotate_hoisted(5, [k5, k3], [k5, k3], c0, c1)
    want[-2] = (want[-2][0], (e_h[0][0], e_h[1][0]))
    want[-1] = (want[-1][0], (e_h[0][1], e_h[1][1]))
    k0, k1 = empty(5 * N), empty(5 * N)
    keep += [k0, k1]
    specs.append(dict(level=5, mode=G.KEYSWITCH, inp=[ptr(d0)], out=[ptr(k0), ptr(k1)]))
    want.append(([k0, k1], S.octx.keyswitch(5, c0)))
    plan = G.Plan(g, specs)
    plan.set_schedule(schedule)
    plan.launch()
    sync()
    assert g.device_status() == 0
    for j, (outs, (e0, e1)) in enumerate(want):
        assert np.array_equal(host(outs[0]), e0) and np.array_equal(host(outs[1]), e1), j


def test_context_destroyed_before_plan(S):
    """gpufhe_ctx_destroy while a plan built on the context lives: the plan
    keeps the context's device state until it is destroyed itself, and still
    computes the oracle's bits."""
    import gpufhe_b200 as G
    g = S.gpu_context()
    rng = np.random.default_rng(5)
    c0a, c1a = S.rand_ct(rng, 4)
    c0b, c1b = S.rand_ct(rng, 4)
    ins = [dev(x) for x in (c0a, c1a, c0b, c1b)]
    outs = [empty(3 * N), empty(3 * N)]
    plan = G.Plan(g, [dict(level=4, inp=[ptr(x) for x in ins], out=[ptr(x) for x in outs])])
    g.close()                                 # the handle ends; the plan holds the context
    plan.launch()
    sync()
    e0, e1 = S.octx.evalmult_rescale(4, c0a, c1a, c0b, c1b)
    assert np.array_equal(host(outs[0]), e0) and np.array_equal(host(outs[1]), e1)
    plan.close()                              # frees the context too


def test_forms_after_a_larger_dnum():
    """Every P5 form still launches on a context with fewer digits than one
    used before it in the same process (kernel shared-memory limits are set
    for the largest digit count, not the first one seen), with equal bits."""
    import gpufhe_b200 as G
    rng = np.random.default_rng(8)
    q0 = O.native_primes(1, 60, N)
    Q = np.concatenate([q0, O.native_primes(13, 50, N, avoid=list(q0))])
    P = O.native_primes(2, 60, N, avoid=list(Q))
    for tw, alpha in ((14, 2), (5, 2), (3, 2)):            # dnum 7, then 3 and 2
        g = G.Context(N, Q[:tw], P, alpha)
        QP = np.concatenate([Q[:tw], P])
        rows = -(-tw // alpha) * len(QP)
        key = [np.concatenate([rng.integers(0, int(QP[r % len(QP)]), N, dtype=np.uint64) for r in range(rows)])
               for _ in range(2)]
        g.set_key(0, key[0], key[1])
        x = [dev(np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in Q[:tw]])) for _ in range(4)]
        got = []
        for sched in (0, 1, 2, 3, 64, 67, 192):
            o0, o1 = empty((tw - 1) * N), empty((tw - 1) * N)
            plan = G.Plan(g, [dict(level=tw, inp=[ptr(t) for t in x], out=[ptr(o0), ptr(o1)])])
            plan.set_schedule(sched)
            plan.launch()
            sync()
            got.append((host(o0), host(o1)))
        for k in range(1, len(got)):
            assert np.array_equal(got[k][0], got[0][0]) and np.array_equal(got[k][1], got[0][1]), (tw, k)


@pytest.mark.parametrize("schedule", [64, 192, 0, 64 | 1 << 17, 64 | 1 << 18, 192 | 1 << 18])
def test_many_digits_fp64_key_product(schedule):
    """Twelve digits (alpha = 1): the FP64 key inner product normalises its
    accumulators after every eighth digit; EvalMult+Rescale and keyswitch at
    every digit count up to twelve equal the oracle in the FP64 forms (the
    TMA ring's among them) and in the integer form."""
    import gpufhe_b200 as G
    S = Setup(N, 12, K=2, alpha=1, seed=33)
    g = S.gpu_context()
    rng = np.random.default_rng(77 + schedule)
    keep, specs, want = [], [], []
    for L in (2, 9, 12):
        c0a, c1a = S.rand_ct(rng, L)
        c0b, c1b = S.rand_ct(rng, L)
        ins = [dev(x) for x in (c0a, c1a, c0b, c1b)]
        outs = [empty((L - 1) * N), empty((L - 1) * N)]
        keep += ins + outs
        specs.append(dict(level=L, inp=[ptr(x) for x in ins], out=[ptr(x) for x in outs]))
        want.append((outs, S.octx.evalmult_rescale(L, c0a, c1a, c0b, c1b)))
        k0, k1 = empty(L * N), empty(L * N)
        keep += [k0, k1]
        specs.append(dict(level=L, mode=G.KEYSWITCH, inp=[ptr(ins[0])], out=[ptr(k0), ptr(k1)]))
        want.append(([k0, k1], S.octx.keyswitch(L, c0a)))
    plan = G.Plan(g, specs)
    plan.set_schedule(schedule)
    plan.launch()
    sync()
    assert plan.schedule()["p5_fp64_rows"] == bool(schedule & 64)
    for j, (outs, (e0, e1)) in enumerate(want):
        assert np.array_equal(host(outs[0]), e0) and np.array_equal(host(outs[1]), e1), j
