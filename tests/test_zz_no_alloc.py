"""gpufhe_rescale_noalloc: the rescale that calls no cudaMalloc / cudaFree.

Hosts that own the device-memory budget through their own pool (and forbid a
library from allocating) and serving threads that must not block on an
allocation call this entry point instead of the workspace-based ones. Its
scratch is a static device array, so it must give exactly the bits of the
existing rescale entry point (GPUFHE_RESCALE through gpufhe_run_ops), on
consecutive calls that reuse the same array, and it must refuse sizes that do
not fit the array. This file is collected last on purpose.
"""
import numpy as np
import pytest

from ckks_setup import chain
from gpu_util import dev, host, ptr, sync

pytestmark = pytest.mark.gpu


def test_noalloc_rescale_matches_existing_entry_point():
    import gpufhe_b200 as G
    n, L = 1 << 16, 12
    Q, P = chain(n, L, 3)
    ctx = G.Context(n, Q, P, 3)
    for call in range(2):   # two calls in a row share the static scratch
        rng = np.random.default_rng(4242 + call)
        comp = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q[:L]])
        a, b = dev(comp), dev(comp)
        G.run_ops(ctx, [dict(level=L, mode=G.RESCALE, inp=[ptr(a)], out=[ptr(a)])])
        G.check(G.lib().gpufhe_rescale_noalloc(ctx.h, L, ptr(b), None))
        sync()
        assert np.array_equal(host(b)[: (L - 1) * n], host(a)[: (L - 1) * n]), call


def test_noalloc_rescale_rejects_oversize():
    import gpufhe_b200 as G
    n = 1 << 16
    max_words = int(G.lib().gpufhe_rescale_noalloc_max_words())
    L = max_words // n + 1
    Q, P = chain(n, L, 2)
    ctx = G.Context(n, Q, P, 4)
    buf = dev(np.zeros(L * n, np.uint64))
    rc = G.lib().gpufhe_rescale_noalloc(ctx.h, L, ptr(buf), None)
    assert rc == -3   # GPUFHE_ENOMEM
    assert b"exceeds the static scratch" in G.lib().gpufhe_last_error()
    assert G.lib().gpufhe_rescale_noalloc(ctx.h, 1, ptr(buf), None) == -1
