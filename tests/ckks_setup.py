"""Seeded CKKS setup shared by the GPU tests: chain, oracle context, keys."""
import numpy as np

import oracle as O


def chain(n, L, K=3, bitsQ=50, bits0=60, bitsP=60):
    Q = O.native_primes(1, bits0, n)
    if L > 1:
        Q = np.concatenate([Q, O.native_primes(L - 1, bitsQ, n, avoid=list(Q))])
    P = O.native_primes(K, bitsP, n, avoid=list(Q))
    return Q, P


def square_mod(s, QP, n):
    out = np.empty_like(s)
    for t, q in enumerate(QP):
        seg = s[t * n:(t + 1) * n].astype(object)
        out[t * n:(t + 1) * n] = np.array([(int(x) * int(x)) % int(q) for x in seg], dtype=np.uint64)
    return out


class Setup:
    """Oracle context + secret/public/relin keys (+ optional rotation keys)."""

    def __init__(self, n, fullQ, K=3, alpha=3, bitsQ=50, rot_ks=(), seed=101):
        self.n, self.fullQ, self.K, self.alpha = n, fullQ, K, alpha
        self.Q, self.P = chain(n, fullQ, K, bitsQ)
        self.octx = O.Ctx(n, self.Q, self.P, alpha)
        T = fullQ + K
        self.s, self.pkA, self.pkB = self.octx.keygen(T, seed=seed)
        s2 = square_mod(self.s, self.octx.QP, n)
        self.av, self.bv = self.octx.evalkeygen(self.s, s2, self.pkA, self.pkB, seed=202)
        self.octx.set_key(0, self.av, self.bv)
        self.rot = {}
        for k in rot_ks:
            sa = self.octx.automorph_eval(T, k, self.s)
            av, bv = self.octx.evalkeygen(self.s, sa, self.pkA, self.pkB, seed=400 + k)
            self.octx.set_key(k, av, bv)
            self.rot[k] = (av, bv)

    def gpu_context(self):
        import gpufhe_b200 as G
        g = G.Context(self.n, self.Q, self.P, self.alpha)
        g.set_key(0, self.av, self.bv)
        for k, (av, bv) in self.rot.items():
            g.set_key(k, av, bv)
        return g

    def rand_ct(self, rng, L):
        return [np.concatenate([rng.integers(0, int(q), self.n, dtype=np.uint64) for q in self.Q[:L]])
                for _ in range(2)]
