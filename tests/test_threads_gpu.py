"""Two host threads, two contexts, one device, in a fresh process.

Kernel attributes (the dynamic shared-memory limits of the P5 and transform
forms) are set once per device on first use. Here two threads build contexts
with different digit counts at the same moment and launch their first plans
together, so the autotuner of each tries every P5 form (the TMA form asks for
200 KiB) while the other thread is setting up: both results must still equal
the oracle bit for bit. A fresh process makes this the first use.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, threading
import numpy as np
sys.path[:0] = [{root!r}, {pkg!r}, {tests!r}]
from ckks_setup import Setup
from gpu_util import dev, empty, host, ptr
import torch
import gpufhe_b200 as G

setups = [Setup(4096, 6, K=3, alpha=3), Setup(4096, 8, K=2, alpha=2, seed=77)]
start = threading.Barrier(2)
errors = []

def work(i):
    try:
        S = setups[i]
        L = S.fullQ
        rng = np.random.default_rng(10 + i)
        ins = S.rand_ct(rng, L) + S.rand_ct(rng, L)
        want = S.octx.evalmult_rescale(L, *ins)
        d = [dev(x) for x in ins]
        out = [empty((L - 1) * S.n) for _ in range(2)]
        torch.cuda.synchronize()
        start.wait()
        g = S.gpu_context()
        for rep in range(3):
            G.run_ops(g, [dict(level=L, mode=G.EVALMULT_RESCALE, inp=[ptr(x) for x in d],
                               out=[ptr(x) for x in out])])
            torch.cuda.synchronize()
            for got, exp in zip(out, want):
                if not np.array_equal(host(got), exp):
                    errors.append((i, rep))
    except Exception as e:
        errors.append((i, repr(e)))

ts = [threading.Thread(target=work, args=(i,)) for i in range(2)]
for t in ts: t.start()
for t in ts: t.join()
print("errors", errors)
sys.exit(1 if errors else 0)
"""


def test_two_threads_two_contexts_first_use():
    code = SCRIPT.format(root=ROOT, pkg=os.path.join(ROOT, "gpu-resident-library_b200"),
                         tests=os.path.join(ROOT, "tests"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
