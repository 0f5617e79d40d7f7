"""The plain per-chain form (drivers/plain_chain: the reference's
bench_evalmult_resident driver on this library's drop-in API, one CUDA graph
of LaunchTensor -> keyswitch_resident -> LaunchCombine ->
rescale_resident_raw x2 per chain, one DeviceKSContext per level sharing the
full-QP key) gives the oracle's EvalMult+Rescale bits at every level,
including levels whose digit partition the reference would derive differently
(L = 4 with alpha = 3). This also checks that keyswitch_resident and
rescale_resident_raw are capturable in a CUDA graph."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from ckks_setup import chain, square_mod

pytestmark = pytest.mark.gpu


def test_plain_chain_driver(tmp_path):
    from gpufhe_b200 import build as B
    exe = B.build_driver()
    n, fullQ, K, alpha = 4096, 6, 3, 3
    levels = [4, 6, 5, 2]
    dump = tmp_path / "plain.bin"
    r = subprocess.run([exe, str(n), str(fullQ), str(K), str(alpha), "2", str(dump), *map(str, levels)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert '"chains": 4' in r.stdout
    Q, P = chain(n, fullQ, K)
    octx = O.Ctx(n, Q, P, alpha)
    T = fullQ + K
    s, a, b = octx.keygen(T, seed=101)
    av, bv = octx.evalkeygen(s, square_mod(s, octx.QP, n), a, b, seed=202)
    octx.set_key(0, av, bv)
    data = np.fromfile(dump, dtype=np.uint64)
    off = 0
    for L in levels:
        ins = []
        for _ in range(4):
            ins.append(data[off:off + L * n])
            off += L * n
        outs = []
        for _ in range(2):
            outs.append(data[off:off + (L - 1) * n])
            off += (L - 1) * n
        want = octx.evalmult_rescale(L, *ins)
        assert np.array_equal(outs[0], want[0]) and np.array_equal(outs[1], want[1]), L
    assert off == data.size
