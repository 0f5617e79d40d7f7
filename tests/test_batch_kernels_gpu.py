"""Batched kernels of the kernel-isolation workload (forward / inverse RNS NTT
and RNS multiply over [poly][tower][n]) bit-exact against the CPU oracle."""
import numpy as np
import pytest

import oracle as O
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gpufhe_b200
    return gpufhe_b200


def make_ctx(G, n, towers):
    Q = O.native_primes(towers, 50, n)
    P = O.native_primes(1, 60, n, avoid=list(Q))
    return G.Context(n, Q, P, 1), Q


@pytest.mark.parametrize("n,npolys,towers", [(4096, 3, 4), (65536, 2, 3)])
def test_ntt_batch(G, n, npolys, towers):
    ctx, Q = make_ctx(G, n, towers)
    roots = ctx.roots()
    rng = np.random.default_rng(n + npolys)
    x = np.concatenate([rng.integers(0, int(Q[t]), n, dtype=np.uint64)
                        for _ in range(npolys) for t in range(towers)])
    dx = dev(x)
    jb = int(G.lib().gpufhe_ntt_job_bytes())
    jobs = empty(npolys * towers * jb // 8)
    G.check(G.lib().gpufhe_ntt_batch(ctx.h, ptr(dx), npolys, towers, 0, 0, ptr(jobs), None))
    sync()
    y = host(dx)
    for p in range(npolys):
        for t in range(towers):
            q = int(Q[t])
            fr, fp, ir, ip, ni, nip = O.root_tables(n, q, int(roots[t]))
            seg = slice((p * towers + t) * n, (p * towers + t + 1) * n)
            assert np.array_equal(y[seg], O.ntt(x[seg], n, q, fr, fp)), (p, t)
    # inverse brings every tower back; a replay of the prepared job list does the same
    G.check(G.lib().gpufhe_ntt_batch(ctx.h, ptr(dx), npolys, towers, 0, 1, ptr(jobs), None))
    sync()
    assert np.array_equal(host(dx), x)
    G.check(G.lib().gpufhe_ntt_batch(ctx.h, ptr(dx), npolys, towers, 0, 0, ptr(jobs), None))
    G.check(G.lib().gpufhe_ntt_run_jobs(ctx.h, ptr(jobs), npolys * towers, 0, None))
    G.check(G.lib().gpufhe_ntt_batch(ctx.h, ptr(dx), npolys, towers, 0, 1, ptr(jobs), None))
    G.check(G.lib().gpufhe_ntt_run_jobs(ctx.h, ptr(jobs), npolys * towers, 1, None))
    sync()
    assert np.array_equal(host(dx), x)


@pytest.mark.parametrize("n,npolys,q_towers", [(65536, 26, 3), (32768, 41, 4)])
def test_ntt_batch_large(G, n, npolys, q_towers):
    """A batch larger than 48 MiB that mixes 50-bit (FP64 path, signed twiddle
    tables) and 60-bit (integer path) towers, transformed once and three times
    in a row from a prepared job list."""
    ctx, Q = make_ctx(G, n, q_towers)
    mods = [int(q) for q in Q] + [int(ctx._P[0])]
    towers = len(mods)
    assert npolys * towers * n * 8 > 48 << 20
    roots = ctx.roots()
    rng = np.random.default_rng(n + npolys)
    x = np.concatenate([rng.integers(0, int(mods[t]), n, dtype=np.uint64)
                        for _ in range(npolys) for t in range(towers)])
    dx = dev(x)
    jb = int(G.lib().gpufhe_ntt_job_bytes())
    jf = empty(npolys * towers * jb // 8)
    ji = empty(npolys * towers * jb // 8)
    G.check(G.lib().gpufhe_ntt_batch(ctx.h, ptr(dx), npolys, towers, 0, 0, ptr(jf), None))
    sync()
    y = host(dx)
    for p in range(npolys):
        for t in range(towers):
            q = int(mods[t])
            fr, fp, ir, ip, ni, nip = O.root_tables(n, q, int(roots[t]))
            seg = slice((p * towers + t) * n, (p * towers + t + 1) * n)
            assert np.array_equal(y[seg], O.ntt(x[seg], n, q, fr, fp)), (p, t)
    G.check(G.lib().gpufhe_ntt_batch(ctx.h, ptr(dx), npolys, towers, 0, 1, ptr(ji), None))
    sync()
    assert np.array_equal(host(dx), x)
    for _ in range(3):
        G.check(G.lib().gpufhe_ntt_run_jobs(ctx.h, ptr(jf), npolys * towers, 0, None))
    sync()
    y3 = host(dx)
    for p, t in ((0, 0), (npolys - 1, towers - 1)):   # an FP64 tower and the 60-bit tower
        q = int(mods[t])
        fr, fp = O.root_tables(n, q, int(roots[t]))[:2]
        seg = slice((p * towers + t) * n, (p * towers + t + 1) * n)
        want = x[seg]
        for _ in range(3):
            want = O.ntt(want, n, q, fr, fp)
        assert np.array_equal(y3[seg], want), (p, t)
    for _ in range(3):
        G.check(G.lib().gpufhe_ntt_run_jobs(ctx.h, ptr(ji), npolys * towers, 1, None))
    sync()
    assert np.array_equal(host(dx), x)


@pytest.mark.parametrize("n,npolys,towers", [(2048, 2, 3), (65536, 3, 4)])
def test_rns_mult_batch(G, n, npolys, towers):
    ctx, Q = make_ctx(G, n, towers)
    rng = np.random.default_rng(7 * n + towers)
    a = np.concatenate([rng.integers(0, int(Q[t]), n, dtype=np.uint64)
                        for _ in range(npolys) for t in range(towers)])
    b = np.concatenate([rng.integers(0, int(Q[t]), n, dtype=np.uint64)
                        for _ in range(npolys) for t in range(towers)])
    a[:4] = Q[0] - 1
    b[:4] = Q[0] - 1
    da, db, do = dev(a), dev(b), empty(a.size)
    G.check(G.lib().gpufhe_rns_mult_batch(ctx.h, ptr(da), ptr(db), ptr(do), npolys, towers, 0, None))
    sync()
    got = host(do)
    for p in range(npolys):
        for t in range(towers):
            seg = slice((p * towers + t) * n, (p * towers + t + 1) * n)
            want = np.zeros(n, np.uint64)
            O.lib().orc_rns_mult(a[seg].copy(), b[seg].copy(), want, int(Q[t]), n)
            assert np.array_equal(got[seg], want), (p, t)
    # in place (out aliases a)
    G.check(G.lib().gpufhe_rns_mult_batch(ctx.h, ptr(da), ptr(db), ptr(da), npolys, towers, 0, None))
    sync()
    assert np.array_equal(host(da), got)
