"""Host-side pieces of the composed bootstrap (tests/test_bootstrap_gpu.py)
checked on the CPU in plain floating point: the merged FFT-stage diagonals
derived as the reference derives them (test_boot.cpp:222-239, 465-488),
applied as sums of diagonal (.) rotation, turn the slots of a coefficient
vector a into (a_k + i a_{k+n/2}) / scale in bit-reversed order
(CoeffsToSlots), and SlotsToCoeffs of the real and imaginary parts brings the
slots back (the round trip the reference gates at 9.6e-16).
"""
import numpy as np

import oracle as O
import test_bootstrap_gpu as B


def apply(v, offs, dg):
    return sum(d * np.roll(v, -o) for o, d in zip(offs, dg))


def test_stage_diagonals_round_trip():
    N, S = B.N, B.S
    rng = np.random.default_rng(7)
    a = rng.integers(-(1 << 40), 1 << 40, N).astype(np.int64)
    scale = float(1 << 59)
    y = O.decode(a, N, scale)
    c2s = [B.stage_diagonals(g, False) for g in range(B.LST)]
    s2c = [B.stage_diagonals(g, True) for g in range(B.LST)]
    assert [len(o) for o, _ in c2s] == [16, 31, 31] and [len(o) for o, _ in s2c] == [16, 31, 31]
    v = y
    for offs, dg in c2s:
        v = apply(v, offs, dg)
    perm = np.array([B.brev(k) for k in range(S)])
    want = (a[:S] + 1j * a[S:]) / scale
    assert np.max(np.abs(v[perm] - want)) < 1e-12 * np.max(np.abs(want))
    w = apply(v.real, *s2c[B.LST - 1]) + apply(1j * v.imag, *s2c[B.LST - 1])
    for g in range(B.LST - 2, -1, -1):
        w = apply(w, *s2c[g])
    assert np.max(np.abs(w - y)) < 1e-12 * np.max(np.abs(y))
