"""Parity at the benchmark's full size: N = 2^16, Q = one 60-bit + eleven
50-bit primes, P = three 60-bit primes, alpha = 3 (dnum = 4), levels drawn
from 4..12 as in bench.py.

* A mixed-level batch with a relinearisation key made on the GPU equals the
  oracle's EvalMult+Rescale pair by pair, bit for bit.
* The whole 128-pair workload in one batched plan equals each pair run alone
  (a plan of one operation), bit for bit: batching changes no output at the
  size the benchmark times.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import oracle as O
from gpu_util import empty, host, ptr, sync

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench as B  # noqa: E402   (workload constants and chain)

N = 1 << B.N_LOG


@pytest.fixture(scope="module")
def env():
    import torch
    import gpufhe_b200 as G
    Q, P = B.chain(G.native_primes, N)
    g = G.Context(N, Q, P, B.ALPHA)
    T = B.FULLQ + B.K_SPECIAL
    ds, da, db = (torch.empty(T * N, dtype=torch.int64, device="cuda") for _ in range(3))
    G.check(G.lib().gpufhe_keygen(g.h, T, 0, 1, 3.19, 101, ptr(ds), ptr(da), ptr(db), None))
    dnum = -(-B.FULLQ // B.ALPHA)
    av, bv = empty(dnum * T * N), empty(dnum * T * N)
    one = C.c_uint64 * 1
    pa = (C.c_void_p * 1)(ptr(av))
    pb = (C.c_void_p * 1)(ptr(bv))
    G.check(G.lib().gpufhe_evalkeygen(g.h, 1, one(0), one(0), one(202), ptr(ds), ptr(da), ptr(db), 1, 3.19,
                                      pa, pb, None))
    return dict(G=G, Q=Q, P=P, g=g, av=host(av), bv=host(bv))


def rand_ct(torch, gen, Q, L):
    t = torch.empty((2, L, N), dtype=torch.int64, device="cuda")
    for i in range(L):
        t[:, i].random_(0, int(Q[i]), generator=gen)
    return t


def test_mixed_levels_match_oracle(env):
    import torch
    G, Q, g = env["G"], env["Q"], env["g"]
    octx = O.Ctx(N, Q, env["P"], B.ALPHA)
    octx.set_key(0, env["av"], env["bv"])
    gen = torch.Generator(device="cuda")
    gen.manual_seed(31)
    levels = [12, 4, 9, 7, 12, 5]
    ins = [[rand_ct(torch, gen, Q, L) for _ in range(2)] for L in levels]
    outs = [torch.empty((2, L - 1, N), dtype=torch.int64, device="cuda") for L in levels]
    specs = [dict(level=L, mode=G.EVALMULT_RESCALE,
                  inp=[ins[j][0][0].data_ptr(), ins[j][0][1].data_ptr(), ins[j][1][0].data_ptr(),
                       ins[j][1][1].data_ptr()],
                  out=[outs[j][0].data_ptr(), outs[j][1].data_ptr()]) for j, L in enumerate(levels)]
    G.run_ops(g, specs)
    sync()
    for j, L in enumerate(levels):
        a, b = ins[j]
        want = octx.evalmult_rescale(L, host(a[0].reshape(-1)), host(a[1].reshape(-1)),
                                     host(b[0].reshape(-1)), host(b[1].reshape(-1)))
        assert np.array_equal(host(outs[j][0].reshape(-1)), want[0]), L
        assert np.array_equal(host(outs[j][1].reshape(-1)), want[1]), L


def test_full_batch_equals_single_pairs(env):
    import torch
    G, Q, g = env["G"], env["Q"], env["g"]
    levels = B.workload_levels(B.SEED)
    assert len(levels) == B.PAIRS
    gen = torch.Generator(device="cuda")
    gen.manual_seed(B.SEED)
    specs, ins, outs, alone = [], [], [], []
    for L in levels:
        x = [rand_ct(torch, gen, Q, L) for _ in range(2)]
        o = torch.empty((2, L - 1, N), dtype=torch.int64, device="cuda")
        ins.append(x)
        outs.append(o)
        specs.append(dict(level=L, mode=G.EVALMULT_RESCALE,
                          inp=[x[0][0].data_ptr(), x[0][1].data_ptr(), x[1][0].data_ptr(), x[1][1].data_ptr()],
                          out=[o[0].data_ptr(), o[1].data_ptr()]))
    G.run_ops(g, specs)                      # one batched plan over all 128 pairs
    sync()
    batched = [host(o.reshape(-1)) for o in outs]
    for j, sp in enumerate(specs):           # each pair alone
        G.run_ops(g, [sp])
    sync()
    for j in range(len(levels)):
        assert np.array_equal(host(outs[j].reshape(-1)), batched[j]), (j, levels[j])
