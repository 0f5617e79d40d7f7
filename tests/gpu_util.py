"""Device-buffer helpers for the GPU tests (torch is only the allocator)."""
import numpy as np


def torch():
    import torch as t
    return t


def dev(a):
    """numpy uint64 -> CUDA int64 tensor with the same bits."""
    t = torch()
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return t.from_numpy(a.view(np.int64).copy()).cuda()


def empty(n):
    t = torch()
    return t.zeros(int(n), dtype=t.int64, device="cuda")


def host(x):
    return x.cpu().numpy().view(np.uint64).copy()


def ptr(x):
    return x.data_ptr()


def sync():
    torch().cuda.synchronize()


def chain(n, L, K=2, alpha=2, bitsQ=50, bits0=60):
    import oracle as O
    Q = np.concatenate([O.native_primes(1, bits0, n), O.native_primes(L - 1, bitsQ, n)]) if L > 1 else O.native_primes(1, bits0, n)
    P = O.native_primes(K, 60, n, avoid=list(Q))
    return Q, P


def rand_res(rng, mods, n):
    return np.concatenate([rng.integers(0, int(q), n, dtype=np.uint64) for q in mods])
