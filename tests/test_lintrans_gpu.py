"""Baby-step giant-step linear transform (gpufhe_lintrans_bsgs) against the
oracle's restatement of the reference's BSGS sequence, per-rotation and
hoisted baby steps, with zero diagonals in the mix."""
import numpy as np
import pytest

import oracle as O
from ckks_setup import Setup
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu

N, FULLQ, N1, N2 = 4096, 8, 4, 3


@pytest.fixture(scope="module")
def G():
    import gpufhe_b200
    return gpufhe_b200


@pytest.fixture(scope="module")
def S():
    rots = sorted({O.galois_element(r, N) for r in (1, 2, 3, 4, 8)})
    return Setup(N, FULLQ, K=3, alpha=3, rot_ks=tuple(rots))


@pytest.fixture(scope="module")
def gctx(S):
    return S.gpu_context()


@pytest.mark.parametrize("L,hoisted", [(FULLQ, False), (5, False), (FULLQ, True)])
def test_lintrans_bsgs(G, S, gctx, L, hoisted):
    rng = np.random.default_rng(10 * L + hoisted)
    c0, c1 = S.rand_ct(rng, L)
    diags = []
    for g in range(N2):
        for b in range(N1):
            if (g, b) in ((0, 2), (2, 1)):
                diags.append(None)
            else:
                diags.append(np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in S.Q[:L]]))
    want0, want1 = S.octx.lintrans_bsgs(L, N1, N2, c0, c1, diags, hoisted=hoisted)
    d0, d1 = dev(c0), dev(c1)
    ddiag = [None if d is None else dev(d) for d in diags]
    o0, o1 = empty(L * N), empty(L * N)
    G.lintrans_bsgs(gctx, L, ptr(d0), ptr(d1), N1, N2, [None if d is None else ptr(d) for d in ddiag],
                    ptr(o0), ptr(o1), hoisted=hoisted)
    sync()
    assert np.array_equal(host(o0), want0) and np.array_equal(host(o1), want1)


def test_lintrans_missing_key(G, gctx):
    d = empty(4 * N)
    with pytest.raises(G.GpuFheError):
        G.lintrans_bsgs(gctx, 4, ptr(d), ptr(d), 6, 1, [None] * 6, ptr(d), ptr(d))   # rot 5 has no key


@pytest.mark.parametrize("hoisted", [False, True])
def test_lintrans_plan_graph_replay(G, S, gctx, hoisted):
    """Plan form: built once, captured in a CUDA graph, replayed on fresh
    ciphertexts written into the same input buffers; every replay equals the
    oracle's BSGS sequence."""
    import ctypes as C
    import torch
    L = 6
    rng = np.random.default_rng(500 + hoisted)
    diags = [np.concatenate([rng.integers(0, int(q), N, dtype=np.uint64) for q in S.Q[:L]])
             for _ in range(N1 * N2)]
    diags[3] = None
    ddiag = [None if d is None else dev(d) for d in diags]
    d0, d1, o0, o1 = empty(L * N), empty(L * N), empty(L * N), empty(L * N)
    arr = (C.c_void_p * len(ddiag))(*[None if d is None else ptr(d) for d in ddiag])
    h = C.c_void_p()
    G.check(G.lib().gpufhe_lintrans_plan_create(gctx.h, L, ptr(d0), ptr(d1), N1, N2, arr, int(hoisted),
                                                ptr(o0), ptr(o1), C.byref(h)))
    st = torch.cuda.Stream()
    G.check(G.lib().gpufhe_lintrans_plan_launch(h, st.cuda_stream))   # outside capture first
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=st):
        G.check(G.lib().gpufhe_lintrans_plan_launch(h, torch.cuda.current_stream().cuda_stream))
    for rep in range(2):
        c0, c1 = S.rand_ct(rng, L)
        d0.copy_(torch.from_numpy(c0.view(np.int64)))
        d1.copy_(torch.from_numpy(c1.view(np.int64)))
        graph.replay()
        sync()
        want0, want1 = S.octx.lintrans_bsgs(L, N1, N2, c0, c1, diags, hoisted=hoisted)
        assert np.array_equal(host(o0), want0) and np.array_equal(host(o1), want1), rep
    del graph
    G.lib().gpufhe_lintrans_plan_destroy(h)
