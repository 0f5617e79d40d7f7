"""CPU oracle for the resident leveled-CKKS path (test infrastructure only).

Loads ``oracle/_build/libckks_oracle.so`` (built by ``oracle/Makefile``) and
wraps it for numpy. Only tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may use this package; the product library never
does. ``load_ref_host`` / ``load_ref_gpu`` give the reference library rebuilt
from its own sources (``oracle/build_ref.sh``) for parity pins.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "_build", "libckks_oracle.so")
_REF_HOST = os.path.join(HERE, "_ref", "libref_host.so")
_REF_GPU = os.path.join(HERE, "_ref", "libref_gpu.so")

u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
VP = C.c_void_p
U32, U64, I32, DBL = C.c_uint32, C.c_uint64, C.c_int, C.c_double

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "ckks_oracle.cpp")
        if not os.path.exists(_LIB) or (os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(_LIB)):
            build()
        L = C.CDLL(_LIB)
        sig = {
            "orc_native_primes": (I32, [u64p, U32, U32, U32, VP, U32]),
            "orc_native_root": (U64, [U32, U64]),
            "orc_rescale_consts": (None, [u64p, u64p, u64p, U32]),
            "orc_root_tables": (None, [U32, U64, U64, u64p, u64p, u64p, u64p, u64p]),
            "orc_ntt": (None, [u64p, u64p, u64p, U32, U64]),
            "orc_intt": (None, [u64p, u64p, u64p, U32, U64, U64, U64]),
            "orc_rns_mult": (None, [u64p, u64p, u64p, U64, U32]),
            "orc_tensor": (None, [u64p, u64p, u64p, u64p, u64p, u64p, u64p, u64p, U32, U32]),
            "orc_combine": (None, [u64p, u64p, u64p, u64p, u64p, u64p, u64p, U32, U32]),
            "orc_switch_modulus": (None, [u64p, U64, U64, U32]),
            "orc_rescale_fuse": (None, [u64p, u64p, U64, U64, U64, U32]),
            "orc_barrett_u128": (U64, [U64, U64, U64, U64, U64]),
            "orc_approx_switch": (None, [u64p, u64p, u64p, u64p, u64p, u64p, u64p, u64p, u64p, U32, U32, U32]),
            "orc_ks_macc": (None, [u64p, u64p, u64p, u64p, u64p, U64, U32]),
            "orc_moddown_combine": (None, [u64p, u64p, u64p, U64, U64, U32]),
            "orc_automorph": (None, [u64p, u64p, U32, U64, U64]),
            "orc_add_into": (None, [u64p, u64p, U64, U32]),
            "orc_ptmulacc": (None, [u64p, u64p, u64p, u64p, u64p, U64, U32]),
            "orc_lintrans_bsgs": (None, [VP, U32, U32, U32, u64p, u64p, VP, I32, u64p, u64p]),
            "orc_ks_constants_size": (U64, [U32, U32, U32]),
            "orc_ks_constants": (None, [u64p, u64p, U32, u64p, U32, U32]),
            "orc_ctx_create": (VP, [U32, u64p, U32, u64p, U32, U32, VP]),
            "orc_ctx_destroy": (None, [VP]),
            "orc_ctx_roots": (None, [VP, u64p]),
            "orc_ctx_set_key": (I32, [VP, U32, u64p, u64p]),
            "orc_set_hamming_weight": (None, [U32]),
            "orc_keygen": (None, [VP, U32, U64, DBL, U64, u64p, u64p, u64p]),
            "orc_evalkeygen": (None, [VP, u64p, u64p, u64p, u64p, U64, DBL, U64, u64p, u64p]),
            "orc_encrypt": (None, [VP, U32, i64p, u64p, u64p, U64, DBL, U64, u64p, u64p]),
            "orc_decrypt": (None, [VP, U32, u64p, u64p, u64p, i64p]),
            "orc_modraise": (None, [VP, U32, u64p, u64p, u64p, u64p]),
            "orc_phase_coeff": (None, [VP, U32, u64p, u64p, u64p, u64p]),
            "orc_keyswitch": (None, [VP, U32, U32, u64p, u64p, u64p]),
            "orc_rescale": (None, [VP, U32, u64p]),
            "orc_evalmult_rescale": (None, [VP, U32, u64p, u64p, u64p, u64p, u64p, u64p]),
            "orc_evalmult_rescale_batch": (None, [VP, U32, u32p, VP, VP, VP, VP, VP, VP, I32]),
            "orc_automorph_eval": (None, [VP, U32, U32, u64p, I32]),
            "orc_rotate": (None, [VP, U32, U32, U32, u64p, u64p]),
            "orc_rotate_hoisted": (None, [VP, U32, U32, u32p, u32p, u64p, u64p, VP, VP]),
            "orc_num_threads": (I32, []),
            "orc_encode": (None, [i64p, f64p, f64p, U32, DBL]),
            "orc_decode": (None, [f64p, f64p, i64p, U32, DBL]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


# ---------------------------------------------------------------- params
def native_primes(count, bits, n, avoid=()):
    out = np.zeros(count, dtype=np.uint64)
    av = _u64(list(avoid)) if len(avoid) else None
    rc = lib().orc_native_primes(out, count, bits, n, av.ctypes.data if av is not None else None, len(avoid))
    if rc != 0:
        raise RuntimeError("prime search exhausted")
    return out


def native_root(n, q):
    return int(lib().orc_native_root(n, int(q)))


def rescale_consts(mods, last):
    s1 = np.zeros(last, dtype=np.uint64)
    s2 = np.zeros(last, dtype=np.uint64)
    lib().orc_rescale_consts(s1, s2, _u64(mods), last)
    return s1, s2


def root_tables(n, q, root):
    fr, fp, ir, ip = (np.zeros(n, np.uint64) for _ in range(4))
    ni = np.zeros(2, np.uint64)
    lib().orc_root_tables(n, int(q), int(root), fr, fp, ir, ip, ni)
    return fr, fp, ir, ip, int(ni[0]), int(ni[1])


def ks_constants(Q, P, alpha):
    Q, P = _u64(Q), _u64(P)
    out = np.zeros(lib().orc_ks_constants_size(len(Q), len(P), alpha), dtype=np.uint64)
    lib().orc_ks_constants(out, Q, len(Q), P, len(P), alpha)
    return out


# ---------------------------------------------------------------- primitives
def ntt(x, n, q, fr, fp):
    x = _u64(x).copy()
    lib().orc_ntt(x, _u64(fr), _u64(fp), n, int(q))
    return x


def intt(x, n, q, ir, ip, ninv, ninvp):
    x = _u64(x).copy()
    lib().orc_intt(x, _u64(ir), _u64(ip), n, int(q), int(ninv), int(ninvp))
    return x


class Ctx:
    """Chain Q (fullQ towers), special primes P, digit width alpha, tables, keys."""

    def __init__(self, n, Q, P, alpha, roots=None):
        self.n, self.Q, self.P, self.alpha = n, _u64(Q), _u64(P), alpha
        self.fullQ, self.K = len(self.Q), len(self.P)
        self.dnum = -(-self.fullQ // alpha)
        r = _u64(roots) if roots is not None else None
        self.h = lib().orc_ctx_create(n, self.Q, self.fullQ, self.P, self.K, alpha,
                                      r.ctypes.data if r is not None else None)
        self._keep = r
        self.roots = np.zeros(self.fullQ + self.K, np.uint64)
        lib().orc_ctx_roots(self.h, self.roots)
        self.QP = np.concatenate([self.Q, self.P])

    def __del__(self):
        try:
            lib().orc_ctx_destroy(self.h)
        except Exception:
            pass

    def set_key(self, key_id, av, bv):
        lib().orc_ctx_set_key(self.h, key_id, _u64(av), _u64(bv))

    def keygen(self, towers, ns=1, sigma=3.19, seed=101):
        shape = towers * self.n
        s, a, b = (np.zeros(shape, np.uint64) for _ in range(3))
        lib().orc_keygen(self.h, towers, ns, sigma, seed, s, a, b)
        return s, a, b

    def evalkeygen(self, sQP, sOld, pkA, pkB, ns=1, sigma=3.19, seed=202):
        W = self.dnum * (self.fullQ + self.K) * self.n
        av, bv = np.zeros(W, np.uint64), np.zeros(W, np.uint64)
        lib().orc_evalkeygen(self.h, _u64(sQP), _u64(sOld), _u64(pkA), _u64(pkB), ns, sigma, seed, av, bv)
        return av, bv

    def encrypt(self, towers, m, pkA, pkB, ns=1, sigma=3.19, seed=303):
        c0, c1 = np.zeros(towers * self.n, np.uint64), np.zeros(towers * self.n, np.uint64)
        lib().orc_encrypt(self.h, towers, np.ascontiguousarray(m, np.int64), _u64(pkA), _u64(pkB),
                          ns, sigma, seed, c0, c1)
        return c0, c1

    def decrypt(self, towers, c0, c1, s):
        m = np.zeros(self.n, np.int64)
        lib().orc_decrypt(self.h, towers, _u64(c0), _u64(c1), _u64(s), m)
        return m

    def phase_coeff(self, towers, c0, c1, s):
        ph = np.zeros(towers * self.n, np.uint64)
        lib().orc_phase_coeff(self.h, towers, _u64(c0), _u64(c1), _u64(s), ph)
        return ph

    def modraise(self, towers, c0, c1):
        """Tower-0 ciphertext raised to `towers` towers (test_modraise.cpp:50-58)."""
        o0, o1 = np.zeros(towers * self.n, np.uint64), np.zeros(towers * self.n, np.uint64)
        lib().orc_modraise(self.h, towers, _u64(c0[:self.n]), _u64(c1[:self.n]), o0, o1)
        return o0, o1

    def decrypt_crt(self, towers, c0, c1, s):
        """Full-CRT decryption: centered integer coefficients over Q_towers."""
        ph = self.phase_coeff(towers, c0, c1, s).reshape(towers, self.n)
        qs = [int(q) for q in self.Q[:towers]]
        Qt = 1
        for q in qs:
            Qt *= q
        basis = []
        for q in qs:
            Mi = Qt // q
            basis.append(Mi * pow(Mi % q, -1, q))
        out = []
        for k in range(self.n):
            v = sum(int(ph[t, k]) * basis[t] for t in range(towers)) % Qt
            out.append(v - Qt if v > Qt // 2 else v)
        return out

    def keyswitch(self, L, a, key_id=0):
        ba0, ba1 = np.zeros(L * self.n, np.uint64), np.zeros(L * self.n, np.uint64)
        lib().orc_keyswitch(self.h, key_id, L, _u64(a), ba0, ba1)
        return ba0, ba1

    def rescale(self, L, comp):
        c = _u64(comp).copy()
        lib().orc_rescale(self.h, L, c)
        return c[: (L - 1) * self.n]

    def evalmult_rescale(self, L, c0a, c1a, c0b, c1b):
        o0, o1 = np.zeros((L - 1) * self.n, np.uint64), np.zeros((L - 1) * self.n, np.uint64)
        lib().orc_evalmult_rescale(self.h, L, _u64(c0a), _u64(c1a), _u64(c0b), _u64(c1b), o0, o1)
        return o0, o1

    def evalmult_rescale_batch(self, Ls, c0a, c1a, c0b, c1b, nthreads=0):
        """Lists of per-pair arrays; OpenMP over pairs."""
        npairs = len(Ls)
        outs0 = [np.zeros((L - 1) * self.n, np.uint64) for L in Ls]
        outs1 = [np.zeros((L - 1) * self.n, np.uint64) for L in Ls]
        arr = lambda lst: (C.c_void_p * npairs)(*[x.ctypes.data for x in lst])
        ins = [[_u64(x) for x in lst] for lst in (c0a, c1a, c0b, c1b)]
        lib().orc_evalmult_rescale_batch(self.h, npairs, np.ascontiguousarray(Ls, np.uint32),
                                         arr(ins[0]), arr(ins[1]), arr(ins[2]), arr(ins[3]),
                                         arr(outs0), arr(outs1), nthreads)
        return outs0, outs1

    def automorph_eval(self, towers, k, v):
        v = _u64(v).copy()
        lib().orc_automorph_eval(self.h, towers, k, v, 1)
        return v

    def rotate(self, L, k, c0, c1, key_id):
        a, b = _u64(c0).copy(), _u64(c1).copy()
        lib().orc_rotate(self.h, key_id, L, k, a, b)
        return a, b

    def lintrans_bsgs(self, L, n1, n2, c0, c1, diags, hoisted=False):
        """diags: list of n2*n1 arrays ([L*n] eval form) or None, index g*n1+b."""
        keep = [None if d is None else _u64(d) for d in diags]
        arr = (C.c_void_p * len(keep))(*[None if d is None else d.ctypes.data for d in keep])
        o0, o1 = np.zeros(L * self.n, np.uint64), np.zeros(L * self.n, np.uint64)
        lib().orc_lintrans_bsgs(self.h, L, n1, n2, _u64(c0), _u64(c1), arr, 1 if hoisted else 0, o0, o1)
        return o0, o1

    def rotate_hoisted(self, L, ks, key_ids, c0, c1):
        nr = len(ks)
        o0 = [np.zeros(L * self.n, np.uint64) for _ in range(nr)]
        o1 = [np.zeros(L * self.n, np.uint64) for _ in range(nr)]
        arr = lambda lst: (C.c_void_p * nr)(*[x.ctypes.data for x in lst])
        lib().orc_rotate_hoisted(self.h, L, nr, np.ascontiguousarray(ks, np.uint32),
                                 np.ascontiguousarray(key_ids, np.uint32), _u64(c0), _u64(c1),
                                 arr(o0), arr(o1))
        return o0, o1


def set_hamming_weight(h):
    lib().orc_set_hamming_weight(h)


def num_threads():
    return int(lib().orc_num_threads())


def encode(z, n, delta):
    """Canonical encode of n/2 complex slots (reference encode.cpp:13-28)."""
    z = np.asarray(z, dtype=np.complex128)
    m = np.zeros(n, np.int64)
    lib().orc_encode(m, np.ascontiguousarray(z.real), np.ascontiguousarray(z.imag), n, float(delta))
    return m


def decode(m, n, delta):
    """Canonical decode of n integer coefficients (reference encode.cpp:30-44)."""
    zr, zi = np.zeros(n // 2), np.zeros(n // 2)
    lib().orc_decode(zr, zi, np.ascontiguousarray(m, np.int64), n, float(delta))
    return zr + 1j * zi


def galois_element(r, n):
    """k = 5^r mod 2n; negative r uses the inverse (5^-r), conjugation is 2n-1."""
    M = 2 * n
    return pow(5, r, M) if r >= 0 else pow(pow(5, -r, M), -1, M)


# ---------------------------------------------------------------- reference builds
def load_ref_host():
    if not os.path.exists(_REF_HOST):
        return None
    L = C.CDLL(_REF_HOST)
    L.ref_native_primes.restype = I32
    L.ref_native_primes.argtypes = [u64p, U32, U32, U32, VP, U32]
    L.ref_native_root.restype = U64
    L.ref_native_root.argtypes = [U32, U64]
    L.ref_rescale_consts.restype = None
    L.ref_rescale_consts.argtypes = [u64p, u64p, u64p, U32, U32]
    L.ref_ks_constants.restype = U32
    L.ref_ks_constants.argtypes = [u64p, u64p, U32, u64p, U32, U32]
    L.ref_encode.restype = None
    L.ref_encode.argtypes = [i64p, f64p, f64p, U32, DBL]
    L.ref_decode.restype = None
    L.ref_decode.argtypes = [f64p, f64p, i64p, U32, DBL]
    return L


def load_ref_gpu():
    if not os.path.exists(_REF_GPU):
        return None
    L = C.CDLL(_REF_GPU)
    sig = {
        "refg_create": (VP, [U32, u64p, U32, u64p, U32, u64p]),
        "refg_destroy": (None, [VP]),
        "refg_set_hw": (None, [U32]),
        "refg_keygen": (None, [U32, u64p, U32, u64p, U64, DBL, U64, u64p, u64p, u64p]),
        "refg_evalkeygen": (None, [VP, U32, u64p, u64p, u64p, u64p, U64, DBL, U64, u64p, u64p]),
        "refg_set_key": (None, [VP, U32, U32, u64p, u64p]),
        "refg_encrypt": (None, [U32, u64p, U32, u64p, i64p, u64p, u64p, U64, DBL, U64, u64p, u64p]),
        "refg_decrypt": (None, [U32, u64p, U32, u64p, u64p, u64p, u64p, i64p]),
        "refg_automorph_host": (None, [U32, U32, U32, u64p, u64p, u64p]),
        "refg_keyswitch_resident": (I32, [VP, U32, U32, U32, u64p, u64p, u64p]),
        "refg_keyswitch_core": (I32, [VP, U32, U32, U32, u64p, u64p, u64p]),
        "refg_rescale": (I32, [VP, U32, U32, u64p]),
        "refg_evalmult_rescale": (I32, [VP, U32, U32, u64p, u64p, u64p, u64p, u64p, u64p]),
        "refg_rotate_device": (I32, [VP, U32, U32, U32, U32, u64p, u64p]),
        "refg_ntt": (I32, [u64p, U32, U64, u64p, u64p, I32, U64, U64]),
        "refg_pt_to_eval": (None, [U32, U32, u64p, u64p, i64p, u64p]),
        "refg_ptops": (None, [U32, U32, u64p, I32, u64p, u64p, u64p, u64p]),
        "refg_rotate_host": (I32, [VP, U32, U32, U32, U32, u64p, u64p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L
