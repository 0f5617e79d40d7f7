"""ApproxSwitchCRTBasis on the integer tensor cores (gpufhe_approx_switch:
tcgen05.mma kind::i8 with tensor-memory sums, and the warp-level mma.sync
form) against the integer-pipe form (form 2), the reference ABI entry
LaunchApproxSwitchCRTBasis (which takes the tcgen05 form where it can) and
the oracle's restatement of
kernels/basis_convert.cu:14-114, bit for bit, at the widths the workloads use
(ModUp alpha = 3 into 12 targets, alpha = 8 into 24, ModDown K = 8 into 24)
and at ragged and maximal ones; two calls in a row; the bounded-wait status
word stays clear."""
import numpy as np
import pytest

import oracle as O
from gpu_util import dev, empty, host, ptr, rand_res, sync

pytestmark = pytest.mark.gpu


def constants(Qm, Pm):
    prod = 1
    for q in Qm:
        prod *= int(q)
    qhi = np.array([pow((prod // int(q)) % int(q), -1, int(q)) for q in Qm], np.uint64)
    qhip = np.array([(int(h) << 64) // int(q) for h, q in zip(qhi, Qm)], np.uint64)
    qmp = np.array([[(prod // int(q)) % int(p) for p in Pm] for q in Qm], np.uint64).ravel()
    mu = [((1 << 128) - 1) // int(p) for p in Pm]
    mulo = np.array([m & (2**64 - 1) for m in mu], np.uint64)
    muhi = np.array([m >> 64 for m in mu], np.uint64)
    return qhi, qhip, qmp, mulo, muhi


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("sizeQ,sizeP,bitsQ,bitsP", [(3, 12, 50, 50), (8, 24, 50, 60), (8, 24, 60, 50),
                                                     (1, 1, 60, 60), (5, 13, 55, 58), (12, 64, 60, 60),
                                                     (4, 9, 50, 60)])
def test_tensor_conversion_bit_exact(form, sizeQ, sizeP, bitsQ, bitsP):
    import gpufhe_b200 as G
    n = 4096
    Qm = O.native_primes(sizeQ, bitsQ, n)
    Pm = O.native_primes(sizeP, bitsP, n, avoid=list(Qm))
    rng = np.random.default_rng(sizeQ * 97 + sizeP)
    src = rand_res(rng, Qm, n)
    qhi, qhip, qmp, mulo, muhi = constants(Qm, Pm)
    bufs = [dev(x) for x in (src, qhi, qhip, Qm, qmp, Pm, mulo, muhi)]
    d_int, d_mma = empty(sizeP * n), empty(sizeP * n)
    G.check(G.lib().gpufhe_approx_switch(ptr(bufs[0]), ptr(d_int), *[ptr(x) for x in bufs[1:]], sizeQ, sizeP, n,
                                         2, None))   # the integer form
    d_abi = empty(sizeP * n)   # the reference ABI entry (tcgen05 where the shape allows)
    G.lib().LaunchApproxSwitchCRTBasis(ptr(bufs[0]), ptr(d_abi), *[ptr(x) for x in bufs[1:]], sizeQ, sizeP, n, None)
    sync()
    assert np.array_equal(host(d_abi), host(d_int))
    for rep in range(2):   # the second call reuses nothing from the first
        d_mma.fill_(-1)
        G.check(G.lib().gpufhe_approx_switch(ptr(bufs[0]), ptr(d_mma), *[ptr(x) for x in bufs[1:]], sizeQ,
                                                    sizeP, n, form, None))
        sync()
        st = np.zeros(1, np.uint32)
        G.check(G.lib().gpufhe_approx_switch_status(st.ctypes.data))
        assert st[0] == 0
        assert np.array_equal(host(d_mma), host(d_int)), rep
    want = np.zeros(sizeP * n, np.uint64)
    O.lib().orc_approx_switch(src, want, qhi, qhip, Qm, qmp, Pm, mulo, muhi, sizeQ, sizeP, n)
    assert np.array_equal(host(d_mma), want)


def test_tensor_conversion_rejects_unsupported():
    import gpufhe_b200 as G
    x = empty(64)
    p = ptr(x)
    f = G.lib().gpufhe_approx_switch
    assert f(p, p, p, p, p, p, p, p, p, 13, 4, 128, 0, None) == -1    # sizeQ > 12
    assert f(p, p, p, p, p, p, p, p, p, 4, 65, 128, 0, None) == -1    # sizeP > 64
    assert f(p, p, p, p, p, p, p, p, p, 4, 4, 64, 0, None) == -1      # tcgen05 form needs n % 128 == 0
    assert f(p, p, p, p, p, p, p, p, p, 4, 4, 24, 1, None) == -1      # mma.sync form needs n % 16 == 0
    assert f(p, p, p, p, p, p, p, p, p, 4, 4, 128, 3, None) == -1     # unknown form
