"""gpufhe_pointwise_batch, every kind, against the formulas the reference's
host loops use (src/ptops.cpp:13-26 and the add / subtract / scale loops of
its tests): add s = a + b, minus q when s >= q; subtract a >= b ? a - b :
a + q - b; products (a * b) mod q over the full 64-bit operand range. One
batch mixes kinds and levels over a 60-bit tower (integer products) and
50-bit towers (exact FP64 products for canonical operands); the product
kinds also take operands and scalars at or above q, which go through the
reducing integer form. Bit for bit."""
import numpy as np
import pytest

from gpu_util import chain, dev, host, ptr, sync

pytestmark = pytest.mark.gpu


def expect(kind, a0, a1, b0, b1, q, scalar, G):
    qo = int(q)
    f = np.frompyfunc
    add = f(lambda x, y: (int(x) + int(y)) - qo if int(x) + int(y) >= qo else int(x) + int(y), 2, 1)
    sub = f(lambda x, y: int(x) - int(y) if int(x) >= int(y) else int(x) + qo - int(y), 2, 1)
    mul = f(lambda x, y: (int(x) * int(y)) % qo, 2, 1)
    u = lambda z: np.array(z, dtype=object).astype(np.uint64)
    if kind == G.PW_ADD:
        return u(add(a0, b0)), u(add(a1, b1))
    if kind == G.PW_SUB:
        return u(sub(a0, b0)), u(sub(a1, b1))
    if kind == G.PW_MUL_PT:
        return u(mul(a0, b0)), u(mul(a1, b0))
    if kind == G.PW_ADD_PT:
        return u(add(a0, b0)), a1.copy()
    if kind == G.PW_SUB_PT:
        return u(sub(a0, b0)), a1.copy()
    return u(mul(a0, np.full_like(a0, scalar))), u(mul(a1, np.full_like(a1, scalar)))


@pytest.mark.parametrize("wide", [False, True])
def test_pointwise_kinds_bit_exact(wide):
    import gpufhe_b200 as G
    n, L = 4096, 4
    Q, P = chain(n, L, K=1, alpha=2)
    ctx = G.Context(n, Q, P, 2)
    rng = np.random.default_rng(12 + wide)
    keep, ops, want = [], [], []
    kinds = [G.PW_ADD, G.PW_SUB, G.PW_MUL_PT, G.PW_ADD_PT, G.PW_SUB_PT, G.PW_MUL_INT]
    if wide:   # operands and scalars over the whole 64-bit range: the product kinds only
        kinds = [G.PW_MUL_PT, G.PW_MUL_INT, G.PW_MUL_PT]
    for i, kind in enumerate(kinds):
        tw = 1 + i % L
        def draw():
            if wide:
                return rng.integers(0, 2**63, size=(tw, n), dtype=np.uint64) * np.uint64(2) + \
                    rng.integers(0, 2, size=(tw, n), dtype=np.uint64)
            return np.stack([rng.integers(0, int(Q[t]), n, dtype=np.uint64) for t in range(tw)])
        a0, a1, b0, b1 = draw(), draw(), draw(), draw()
        scalar = int(rng.integers(0, 2**63)) * 2 + 1 if wide else int(rng.integers(0, 1 << 20))
        bufs = [dev(x.ravel()) for x in (a0, a1, b0, b1)]
        o0, o1 = dev(np.zeros(tw * n, np.uint64)), dev(np.zeros(tw * n, np.uint64))
        keep += bufs + [o0, o1]
        b = () if kind == G.PW_MUL_INT else ((ptr(bufs[2]), ptr(bufs[3])) if kind in (G.PW_ADD, G.PW_SUB) else (ptr(bufs[2]),))
        ops.append(dict(kind=kind, towers=tw, a=(ptr(bufs[0]), ptr(bufs[1])), b=b, o=(ptr(o0), ptr(o1)), scalar=scalar))
        e0 = np.empty((tw, n), np.uint64)
        e1 = np.empty((tw, n), np.uint64)
        for t in range(tw):
            e0[t], e1[t] = expect(kind, a0[t], a1[t], b0[t], b1[t], Q[t], scalar, G)
        want.append((o0, o1, e0.ravel(), e1.ravel()))
    G.pointwise(ctx, ops)
    sync()
    for j, (o0, o1, e0, e1) in enumerate(want):
        assert np.array_equal(host(o0), e0), (j, kinds[j])
        assert np.array_equal(host(o1), e1), (j, kinds[j])
    ctx.close()
