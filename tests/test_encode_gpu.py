"""Canonical encode / decode on the GPU (gpufhe_encode_batch /
gpufhe_decode_batch) against the oracle's restatement of the reference's
encode_host / decode_host (encode.cpp:13-44), which the CPU tests pin to the
reference's own code and golden digests: coefficients and decoded doubles
are bit-identical, for single messages and batches whose size is not a
multiple of the per-thread message count."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def slots(rng, n, count):
    return rng.uniform(-1, 1, (count, n // 2)) + 1j * rng.uniform(-1, 1, (count, n // 2))


@pytest.mark.parametrize("n,count,dbits", [(16, 1, 20), (1024, 5, 40), (4096, 3, 50), (8192, 1, 30)])
def test_encode_decode_bit_exact(n, count, dbits):
    import gpufhe_b200 as G
    E = G.Encoder(n)
    rng = np.random.default_rng(n + count)
    z = slots(rng, n, count)
    z[0, :3] = [0.0, 1e-300, -1.0 + 0.5j]
    d = float(2.0 ** dbits)
    m = E.encode(z, d)
    for b in range(count):
        assert np.array_equal(m[b], O.encode(z[b], n, d)), b
    zd = E.decode(m, d)
    for b in range(count):
        want = O.decode(m[b], n, d)
        assert np.array_equal(zd[b].real, want.real) and np.array_equal(zd[b].imag, want.imag), b
    # each coefficient rounds by at most 1/2, and a slot sums n of them
    assert np.abs(zd - z).max() <= n / (2 * d)


def test_encode_full_ring_round_trip():
    """N = 2^16, a batch of 6: bit-exact for one message against the oracle,
    and decode(encode(z)) within the scale's rounding for all."""
    import gpufhe_b200 as G
    n = 1 << 16
    E = G.Encoder(n)
    z = slots(np.random.default_rng(3), n, 6)
    d = float(2.0 ** 40)
    m = E.encode(z, d)
    assert np.array_equal(m[5], O.encode(z[5], n, d))
    zd = E.decode(m, d)
    want = O.decode(m[2], n, d)
    assert np.array_equal(zd[2].real, want.real) and np.array_equal(zd[2].imag, want.imag)
    assert np.abs(zd - z).max() <= n / (2 * d)


@pytest.mark.parametrize("n,count,dbits", [(4, 3, 10), (1024, 5, 40), (16384, 2, 40), (65536, 3, 40)])
def test_fast_encode_decode(n, count, dbits):
    """O(n log n) form: coefficients equal the reference's sums or differ by
    one (rounding of a value within floating-point error of a half-integer);
    decoded slots agree with the reference's decode to n * 2^-52 relative."""
    import gpufhe_b200 as G
    E = G.Encoder(n)
    z = slots(np.random.default_rng(7 * n + count), n, count)
    d = float(2.0 ** dbits)
    mf = E.encode(z, d, fast=True)
    me = E.encode(z, d)   # the exact form (bit-identical to the reference, checked above)
    diff = np.abs(mf - me)
    assert diff.max() <= 1, diff.max()
    assert (diff != 0).mean() < 0.2
    zf = E.decode(me, d, fast=True)
    ze = E.decode(me, d)
    scale = max(1.0, float(np.abs(ze).max()))
    assert np.abs(zf - ze).max() <= n * 2.0 ** -52 * scale * 64
    if n <= 1024:
        assert np.array_equal(me[0], O.encode(z[0], n, d))
