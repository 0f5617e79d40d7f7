"""Rotation-key residency under a device budget: keys beyond the budget live in
pinned host copies, come back when a plan needs them (evicting the least
recently used key no plan holds), and rotations stay bit-exact against the
oracle. A batch whose keys cannot all be resident at once is refused with
GPUFHE_ENOMEM; a live plan keeps its keys from being evicted."""
import numpy as np
import pytest

import oracle as O
from ckks_setup import Setup
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

N = 4096


@pytest.fixture(scope="module")
def G():
    import gpufhe_b200
    return gpufhe_b200


@pytest.fixture(scope="module")
def S():
    ks = tuple(O.galois_element(r, N) for r in (1, 2, 3, -1))
    return Setup(N, 8, K=3, alpha=3, rot_ks=ks)


def rotation(G, S, rng, L, k, keep):
    c0, c1 = S.rand_ct(rng, L)
    d0, d1, o0, o1 = dev(c0), dev(c1), empty(L * N), empty(L * N)
    keep.append((k, L, c0, c1, o0, o1, d0, d1))
    return dict(level=L, mode=G.ROTATE, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)], out=[ptr(o0), ptr(o1)])


def check_all(S, keep):
    for k, L, c0, c1, o0, o1, _, _ in keep:
        e0, e1 = S.octx.rotate(L, k, c0, c1, k)
        assert np.array_equal(host(o0), e0) and np.array_equal(host(o1), e1), k


def test_budget_evicts_and_reuploads(G, S):
    g = S.gpu_context()
    kb = g.key_bytes()
    st = g.key_stats()
    assert st["known"] == 5 and st["resident"] == 5 and st["resident_bytes"] == 5 * kb
    g.set_key_budget(2 * kb)
    st = g.key_stats()
    assert st["resident"] == 2 and st["resident_bytes"] == 2 * kb and st["evictions"] == 3
    rng = np.random.default_rng(7)
    keep = []
    for rep in range(2):
        for k in S.rot:
            G.run_ops(g, [rotation(G, S, rng, 6, k, keep)])
            sync()
            assert g.key_stats()["resident_bytes"] <= 2 * kb
    check_all(S, keep)
    st = g.key_stats()
    assert st["uploads"] >= 4 and st["evictions"] >= 7


def test_batch_over_budget_is_refused(G, S):
    g = S.gpu_context()
    kb = g.key_bytes()
    g.set_key_budget(2 * kb)
    rng = np.random.default_rng(8)
    ks = list(S.rot)[:3]
    keep = []
    with pytest.raises(G.GpuFheError, match="status -3"):
        G.run_ops(g, [rotation(G, S, rng, 5, k, keep) for k in ks])
    # the refused batch held nothing: a two-key batch still fits
    keep = []
    G.run_ops(g, [rotation(G, S, rng, 5, k, keep) for k in ks[:2]])
    sync()
    check_all(S, keep)
    # no cap: the three-key batch runs
    g.set_key_budget(0)
    keep = []
    G.run_ops(g, [rotation(G, S, rng, 5, k, keep) for k in ks])
    sync()
    check_all(S, keep)


def test_live_plan_pins_its_keys(G, S):
    g = S.gpu_context()
    kb = g.key_bytes()
    g.set_key_budget(2 * kb)
    rng = np.random.default_rng(9)
    ks = list(S.rot)
    keep = []
    plan = G.Plan(g, [rotation(G, S, rng, 4, k, keep) for k in ks[:2]])
    other = []
    with pytest.raises(G.GpuFheError, match="status -3"):
        G.run_ops(g, [rotation(G, S, rng, 4, ks[2], other)])
    plan.launch()
    sync()
    check_all(S, keep)
    del plan
    other = []
    G.run_ops(g, [rotation(G, S, rng, 4, ks[2], other)])
    sync()
    check_all(S, other)


def test_budget_below_one_key(G, S):
    g = S.gpu_context()
    with pytest.raises(G.GpuFheError, match="status -1"):
        g.set_key_budget(g.key_bytes() - 8)
