"""Batched pipeline (gpufhe_plan_* C ABI) bit-exact against the CPU oracle:
EvalMult+Rescale over uneven levels, keyswitch, rotation and rescale."""
import numpy as np
import pytest

import oracle as O
from ckks_setup import Setup
from gpu_util import dev, empty, host, ptr, sync

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gpufhe_b200
    return gpufhe_b200


@pytest.fixture(scope="module")
def S():
    return Setup(4096, 12, K=3, alpha=3, rot_ks=(5, O.galois_element(-2, 4096)))


@pytest.fixture(scope="module")
def gctx(S):
    return S.gpu_context()


def test_evalmult_rescale_uneven_batch(G, S, gctx):
    rng = np.random.default_rng(2024)
    levels = [2, 3, 4, 5, 7, 9, 12, 12, 6]
    n = S.n
    keep, specs, want = [], [], []
    for L in levels:
        c0a, c1a = S.rand_ct(rng, L)
        c0b, c1b = S.rand_ct(rng, L)
        ins = [dev(x) for x in (c0a, c1a, c0b, c1b)]
        outs = [empty((L - 1) * n), empty((L - 1) * n)]
        keep += ins + outs
        specs.append(dict(level=L, mode=G.EVALMULT_RESCALE, inp=[ptr(x) for x in ins], out=[ptr(x) for x in outs]))
        want.append(S.octx.evalmult_rescale(L, c0a, c1a, c0b, c1b))
    plan = G.Plan(gctx, specs)
    for rep in range(2):   # replay: same bits every time, outputs cleared in between
        for x in keep[4::6] + keep[5::6]:
            x.zero_()
        plan.launch()
        sync()
        for j, L in enumerate(levels):
            o0, o1 = host(keep[6 * j + 4]), host(keep[6 * j + 5])
            assert np.array_equal(o0, want[j][0]), (rep, L)
            assert np.array_equal(o1, want[j][1]), (rep, L)


@pytest.mark.parametrize("L", [1, 3, 8, 12])
def test_keyswitch(G, S, gctx, L):
    rng = np.random.default_rng(L)
    a = S.rand_ct(rng, L)[0]
    da, b0, b1 = dev(a), empty(L * S.n), empty(L * S.n)
    G.run_ops(gctx, [dict(level=L, mode=G.KEYSWITCH, inp=[ptr(da)], out=[ptr(b0), ptr(b1)])])
    e0, e1 = S.octx.keyswitch(L, a)
    assert np.array_equal(host(b0), e0) and np.array_equal(host(b1), e1)


@pytest.mark.parametrize("L", [2, 5, 12])
def test_rescale(G, S, gctx, L):
    rng = np.random.default_rng(100 + L)
    c = S.rand_ct(rng, L)[0]
    dc = dev(c)
    G.run_ops(gctx, [dict(level=L, mode=G.RESCALE, inp=[ptr(dc)], out=[ptr(dc)])])
    assert np.array_equal(host(dc)[: (L - 1) * S.n], S.octx.rescale(L, c))


@pytest.mark.parametrize("L", [4, 12])
def test_rotate(G, S, gctx, L):
    rng = np.random.default_rng(200 + L)
    for k in S.rot:
        c0, c1 = S.rand_ct(rng, L)
        d0, d1, o0, o1 = dev(c0), dev(c1), empty(L * S.n), empty(L * S.n)
        G.run_ops(gctx, [dict(level=L, mode=G.ROTATE, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)],
                              out=[ptr(o0), ptr(o1)])])
        e0, e1 = S.octx.rotate(L, k, c0, c1, k)
        assert np.array_equal(host(o0), e0) and np.array_equal(host(o1), e1), k


def test_evalmult_rescale_decrypts(G, S, gctx):
    """Known-answer product (test_evalmult_rescale.cpp:82-93 at scale 2^40)."""
    n, L = S.n, 12
    sQ, pkA, pkB = S.octx.keygen(L, seed=101)
    D = 1 << 40
    m1 = np.zeros(n, np.int64); m1[0], m1[1] = 3 * D, -2 * D
    m2 = np.zeros(n, np.int64); m2[0], m2[2] = 4 * D, 5 * D
    c0a, c1a = S.octx.encrypt(L, m1, pkA, pkB, seed=303)
    c0b, c1b = S.octx.encrypt(L, m2, pkA, pkB, seed=304)
    ins = [dev(x) for x in (c0a, c1a, c0b, c1b)]
    o0, o1 = empty((L - 1) * n), empty((L - 1) * n)
    G.run_ops(gctx, [dict(level=L, inp=[ptr(x) for x in ins], out=[ptr(o0), ptr(o1)])])
    sR, _, _ = S.octx.keygen(L - 1, seed=101)
    dec = S.octx.decrypt_crt(L - 1, host(o0), host(o1), sR)
    ql = int(S.Q[L - 1])
    got = [round(v * ql / (D * D)) for v in dec[:6]]
    assert got == [12, -8, 15, -10, 0, 0]


def test_rotate_hoisted_groups(G, S, gctx):
    """Hoisted rotations (one shared ModUp per c1 buffer and level) next to a
    plain rotation of the same ciphertext, in one batch."""
    rng = np.random.default_rng(300)
    ks = list(S.rot)
    n = S.n
    cases = [(8, ks), (4, ks[:1])]
    keep, specs, want = [], [], []
    for L, group in cases:
        c0, c1 = S.rand_ct(rng, L)
        d0, d1 = dev(c0), dev(c1)
        keep += [d0, d1]
        e0, e1 = S.octx.rotate_hoisted(L, group, group, c0, c1)
        for r, k in enumerate(group):
            o0, o1 = empty(L * n), empty(L * n)
            keep += [o0, o1]
            specs.append(dict(level=L, mode=G.ROTATE_HOISTED, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)],
                              out=[ptr(o0), ptr(o1)]))
            want.append((o0, o1, e0[r], e1[r]))
        # a plain rotation of the same buffers is not part of the hoisted group
        p0, p1 = empty(L * n), empty(L * n)
        keep += [p0, p1]
        specs.append(dict(level=L, mode=G.ROTATE, key_id=group[0], galois=group[0], inp=[ptr(d0), ptr(d1)],
                          out=[ptr(p0), ptr(p1)]))
        f0, f1 = S.octx.rotate(L, group[0], c0, c1, group[0])
        want.append((p0, p1, f0, f1))
    plan = G.Plan(gctx, specs)
    for rep in range(2):
        plan.launch()
        sync()
        for j, (o0, o1, e0, e1) in enumerate(want):
            assert np.array_equal(host(o0), e0) and np.array_equal(host(o1), e1), (rep, j)
    for form in (1, 3):                       # the staged P5 forms gather hoisted digits themselves
        for o0, o1, _, _ in want:
            o0.zero_()
            o1.zero_()
        plan.set_schedule(form | 4)
        plan.launch()
        sync()
        assert gctx.device_status() == 0
        for j, (o0, o1, e0, e1) in enumerate(want):
            assert np.array_equal(host(o0), e0) and np.array_equal(host(o1), e1), (form, j)


@pytest.mark.parametrize("schedule", [0, 1, 2, 3, 4, 5, 6, 7, 8, 11, 12, 13, 16, 19, 20, 64, 65, 66, 67, 68, 72, 84, 192, 195, 196, 64 | 1 << 17, 195 | 1 << 17,
                                      64 | 1 << 18, 67 | 1 << 17 | 1 << 18, 196 | 1 << 18, 192 | 1 << 18, 195 | 1 << 17 | 1 << 18])
def test_every_schedule_same_bits(G, S, gctx, schedule):
    """Each launch schedule the autotuner can pick (P5 form, P5 50-bit Q rows
    on the FP64 pipe or not and in which of its three forms, P3 form, interleaved or separate integer / FP64
    transform launches) gives the oracle's bits on a mixed batch
    (EvalMult+Rescale at uneven levels, keyswitch, rotation)."""
    rng = np.random.default_rng(900 + schedule)
    n, k = S.n, list(S.rot)[0]
    keep, specs, want = [], [], []
    for L in (3, 7, 12):
        c0a, c1a = S.rand_ct(rng, L)
        c0b, c1b = S.rand_ct(rng, L)
        ins = [dev(x) for x in (c0a, c1a, c0b, c1b)]
        outs = [empty((L - 1) * n), empty((L - 1) * n)]
        keep += ins + outs
        specs.append(dict(level=L, inp=[ptr(x) for x in ins], out=[ptr(x) for x in outs]))
        want.append((outs, S.octx.evalmult_rescale(L, c0a, c1a, c0b, c1b)))
    c0, c1 = S.rand_ct(rng, 9)
    d0, d1, o0, o1, k0, k1 = dev(c0), dev(c1), empty(9 * n), empty(9 * n), empty(9 * n), empty(9 * n)
    keep += [d0, d1, o0, o1, k0, k1]
    specs.append(dict(level=9, mode=G.ROTATE, key_id=k, galois=k, inp=[ptr(d0), ptr(d1)], out=[ptr(o0), ptr(o1)]))
    want.append(([o0, o1], S.octx.rotate(9, k, c0, c1, k)))
    specs.append(dict(level=9, mode=G.KEYSWITCH, inp=[ptr(d0)], out=[ptr(k0), ptr(k1)]))
    want.append(([k0, k1], S.octx.keyswitch(9, c0)))
    plan = G.Plan(gctx, specs)
    plan.set_schedule(schedule)
    plan.launch()
    sync()
    got = plan.schedule()
    assert gctx.device_status() == 0          # no bounded wait expired (TMA form)
    assert got["p5"] == ("register-128x4", "cp.async", "register-256x2", "tma")[schedule & 3]
    assert got["tuned"] and got["mixed_paths"] == bool(schedule & 4)
    assert got["p3"] == ("plain", "warp-specialised-128x2", "warp-specialised-256x1")[(schedule >> 3) & 3]
    assert got["p5_fp64_rows"] == bool(schedule & 64)
    assert got["p5_fp64_form"] == (2 if schedule >> 18 & 1 else 0) + ((schedule >> 7) & 1)
    assert got["p5_split"] == bool(schedule >> 17 & 1)
    for outs, (e0, e1) in want:
        assert np.array_equal(host(outs[0]), e0) and np.array_equal(host(outs[1]), e1)


def test_launch_host_sync_and_async(G, S, gctx):
    """Host-buffer entry points: inputs copied in, the batch, outputs copied
    out; the async form on pinned buffers after a stream synchronisation."""
    import torch
    rng = np.random.default_rng(77)
    n, levels = S.n, [5, 9]
    specs, keep, h_in, want, pins = [], [], [], [], []
    for L in levels:
        cts = [*S.rand_ct(rng, L), *S.rand_ct(rng, L)]
        ins = [empty(L * n) for _ in range(4)]
        outs = [empty((L - 1) * n), empty((L - 1) * n)]
        keep += ins + outs
        specs.append(dict(level=L, inp=[ptr(x) for x in ins], out=[ptr(x) for x in outs]))
        for c in cts:
            t = torch.from_numpy(c.view(np.int64).copy()).pin_memory()
            pins.append(t)
            h_in.append(t.data_ptr())
        want.append(S.octx.evalmult_rescale(L, *cts))
    plan = G.Plan(gctx, specs)
    for sync in (True, False):
        outs_h = [torch.zeros((L - 1) * n, dtype=torch.int64).pin_memory() for L in levels for _ in range(2)]
        plan.launch_host(h_in, [t.data_ptr() for t in outs_h], None, sync=sync)
        torch.cuda.synchronize()
        for j, (e0, e1) in enumerate(want):
            assert np.array_equal(outs_h[2 * j].numpy().view(np.uint64), e0), (sync, j)
            assert np.array_equal(outs_h[2 * j + 1].numpy().view(np.uint64), e1), (sync, j)


def test_launch_host_contiguous_batch(G, S, gctx):
    """gpufhe_plan_launch_host_batch_async: one host buffer per direction,
    every op's inputs / outputs back to back in op order. With device buffers
    in the same layout inside one allocation the copies merge (one transfer
    each way); with separate device allocations they stay piecewise. Both give
    the oracle's results."""
    import torch
    rng = np.random.default_rng(78)
    n, levels = S.n, [4, 7, 6]
    cts = [[*S.rand_ct(rng, L), *S.rand_ct(rng, L)] for L in levels]
    want = [S.octx.evalmult_rescale(L, *c) for L, c in zip(levels, cts)]
    in_words = [L * n for L in levels for _ in range(4)]
    out_words = [(L - 1) * n for L in levels for _ in range(2)]
    offs = lambda ws: [int(o) for o in np.cumsum([0] + ws[:-1])]
    h_in_buf = torch.from_numpy(np.concatenate([x for c in cts for x in c]).view(np.int64).copy()).pin_memory()
    h_out_buf = torch.zeros(sum(out_words), dtype=torch.int64).pin_memory()
    for contiguous in (True, False):
        if contiguous:
            d_in, d_out = empty(sum(in_words)), empty(sum(out_words))
            keep = [d_in, d_out]
            ip = [ptr(d_in) + 8 * o for o in offs(in_words)]
            op = [ptr(d_out) + 8 * o for o in offs(out_words)]
        else:
            keep = [empty(w) for w in in_words] + [empty(w) for w in out_words]
            ip = [ptr(t) for t in keep[:len(in_words)]]
            op = [ptr(t) for t in keep[len(in_words):]]
        specs = [dict(level=L, inp=ip[4 * j:4 * j + 4], out=op[2 * j:2 * j + 2]) for j, L in enumerate(levels)]
        plan = G.Plan(gctx, specs)
        h_out_buf.zero_()
        plan.launch_host_batch(h_in_buf.data_ptr(), h_out_buf.data_ptr(), None, sync=True)
        got = h_out_buf.numpy().view(np.uint64)
        o = offs(out_words)
        for j, (e0, e1) in enumerate(want):
            assert np.array_equal(got[o[2 * j]:o[2 * j] + out_words[2 * j]], e0), (contiguous, j)
            assert np.array_equal(got[o[2 * j + 1]:o[2 * j + 1] + out_words[2 * j + 1]], e1), (contiguous, j)
        plan.close()
        del keep
