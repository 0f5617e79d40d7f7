"""gpufhe_rescale_noalloc: the rescale that calls no cudaMalloc / cudaFree.

Hosts that own the device-memory budget through their own pool (and forbid a
library from allocating) and serving threads that must not block on an
allocation call this entry point instead of the workspace-based ones. Its
scratch is a static device array, so it must give exactly the bits of the
existing rescale entry point (GPUFHE_RESCALE through gpufhe_run_ops), on
consecutive calls that reuse the same array, at every level (the per-level
constants and twiddle offsets differ), on the default stream and on a created
one, and it must refuse sizes that do not fit the array. This file is
collected last on purpose.
"""
import numpy as np
import pytest

from ckks_setup import chain
from gpu_util import dev, host, ptr, sync

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [2, 7, 12])
def test_noalloc_rescale_matches_existing_entry_point(L):
    import torch

    import gpufhe_b200 as G
    n, fullQ = 1 << 16, 12
    Q, P = chain(n, fullQ, 3)
    ctx = G.Context(n, Q, P, 3)
    stream = torch.cuda.Stream()
    for call in range(3):   # calls in a row share the static scratch
        rng = np.random.default_rng(4242 + 31 * L + call)
        comp = np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in Q[:L]])
        a, b = dev(comp), dev(comp)
        G.run_ops(ctx, [dict(level=L, mode=G.RESCALE, inp=[ptr(a)], out=[ptr(a)])])
        sync()
        s = stream.cuda_stream if call == 2 else None   # the third call on a created stream
        G.check(G.lib().gpufhe_rescale_noalloc(ctx.h, L, ptr(b), s))
        sync()
        assert np.array_equal(host(b)[: (L - 1) * n], host(a)[: (L - 1) * n]), (L, call)


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
