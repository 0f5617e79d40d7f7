"""The reference-style C++ API (include/*.h, namespace gpufhe) driven by a C++
program exactly as the reference's own tests drive it; its outputs are then
checked bit-for-bit against the CPU oracle on the same seeds."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from ckks_setup import square_mod

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_cpp_api.cpp")
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "test_cpp_api")
LIBDIR = os.path.join(ROOT, "gpu-resident-library_b200", "gpufhe_b200")


def _build():
    if os.path.exists(BIN) and os.path.getmtime(BIN) >= os.path.getmtime(SRC):
        return
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-ccbin", "/usr/bin/g++",
                    f"-I{ROOT}/include", SRC, "-o", BIN, f"-L{LIBDIR}", "-lgpufhe_b200",
                    "-Xlinker", "-rpath", "-Xlinker", LIBDIR, "-Wno-deprecated-gpu-targets"], check=True)


def test_cpp_api(tmp_path):
    _build()
    out = tmp_path / "cpp_api.bin"
    r = subprocess.run([BIN, str(out)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    n, L, K, alpha = 4096, 6, 3, 3
    Q = np.concatenate([O.native_primes(1, 60, n), O.native_primes(L - 1, 50, n, avoid=list(O.native_primes(1, 60, n)))])
    P = O.native_primes(K, 60, n, avoid=list(Q))
    octx = O.Ctx(n, Q, P, alpha)
    s, pkA, pkB = octx.keygen(L + K, seed=101)
    av, bv = octx.evalkeygen(s, square_mod(s, octx.QP, n), pkA, pkB, seed=202)
    octx.set_key(0, av, bv)
    sQ, qA, qB = octx.keygen(L, seed=101)
    D = 1 << 40
    m1 = np.zeros(n, np.int64); m1[0], m1[1] = 3 * D, -2 * D
    m2 = np.zeros(n, np.int64); m2[0], m2[2] = 4 * D, 5 * D
    c0a, c1a = octx.encrypt(L, m1, qA, qB, seed=303)
    c0b, c1b = octx.encrypt(L, m2, qA, qB, seed=304)
    data = np.fromfile(out, dtype=np.uint64)
    T1, T = (L - 1) * n, L * n
    r0, r1, k0, k1 = data[:T1], data[T1:2 * T1], data[2 * T1:2 * T1 + T], data[2 * T1 + T:2 * T1 + 2 * T]
    rest = data[2 * T1 + 2 * T:]
    ez = rest[:n].view(np.float64).view(np.complex128)
    em = rest[n:2 * n].view(np.int64)
    dz = rest[2 * n:3 * n].view(np.float64).view(np.complex128)
    assert np.array_equal(em, O.encode(ez, n, 2.0 ** 40))         # the reference's encode_host, bit for bit
    want = O.decode(em, n, 2.0 ** 40)
    assert np.array_equal(dz.real, want.real) and np.array_equal(dz.imag, want.imag)
    e0, e1 = octx.evalmult_rescale(L, c0a, c1a, c0b, c1b)
    assert np.array_equal(r0, e0) and np.array_equal(r1, e1)
    t2 = np.zeros(T, np.uint64)
    t0, t1 = np.zeros(T, np.uint64), np.zeros(T, np.uint64)
    O.lib().orc_tensor(c0a, c1a, c0b, c1b, t0, t1, t2, Q, L, n)
    f0, f1 = octx.keyswitch(L, t2)
    assert np.array_equal(k0, f0) and np.array_equal(k1, f1)
