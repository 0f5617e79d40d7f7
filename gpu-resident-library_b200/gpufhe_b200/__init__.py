"""Python bindings for libgpufhe_b200.so (B200-native resident CKKS path).

The shared library is the product; this module only loads it with ctypes and
declares the C-ABI signatures from include/*.h. There is no CPU fallback: if
the library is missing or no CUDA device is present, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpufhe_b200.so")

VP, U32, U64, I32, DBL = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double

_lib = None

# reference ABI: include/{ntt,intt,rns_arith,switch_modulus,rescale,basis_convert,
# ks_fastcore,moddown,tensor,automorph,stage_acc}.h
_REF_ABI = {
    "LaunchNTT_CT": [VP, VP, VP, U32, U64, VP],
    "LaunchINTT_GS": [VP, VP, VP, U32, U64, U64, U64, VP],
    "LaunchRNSMultTower": [VP, VP, VP, U64, U32, VP],
    "LaunchSwitchModulus": [VP, U64, U64, U32, VP],
    "LaunchRescaleFuse": [VP, VP, U64, U64, U64, U32, VP],
    "LaunchApproxSwitchCRTBasis": [VP, VP, VP, VP, VP, VP, VP, VP, VP, U32, U32, U32, VP],
    "LaunchKSMultAcc": [VP, VP, VP, VP, VP, U64, U32, VP],
    "LaunchKSMultAccBatched": [VP, VP, VP, VP, VP, VP, VP, U32, U32, VP],
    "LaunchModDownCombine": [VP, VP, VP, U64, U64, U32, VP],
    "LaunchTensor": [VP, VP, VP, VP, VP, VP, VP, VP, U32, U32, VP],
    "LaunchCombine": [VP, VP, VP, VP, VP, VP, VP, U32, U32, VP],
    "LaunchAutomorphPermute": [VP, VP, U32, U64, U64, VP],
    "LaunchPtMulAcc": [VP, VP, VP, VP, VP, U64, U32, VP],
    "LaunchAddInto": [VP, VP, U64, U32, VP],
}

CP = C.c_char_p
_API: dict = {
    "gpufhe_last_error": (CP, []),
    "gpufhe_ctx_create": (I32, [U32, VP, U32, VP, U32, U32, VP, I32, C.POINTER(VP)]),
    "gpufhe_ctx_destroy": (None, [VP]),
    "gpufhe_ctx_roots": (I32, [VP, VP]),
    "gpufhe_ctx_set_key": (I32, [VP, U64, VP, VP]),
    "gpufhe_ctx_resident_bytes": (U64, [VP]),
    "gpufhe_ctx_set_key_budget": (I32, [VP, U64]),
    "gpufhe_ctx_key_stats": (I32, [VP, VP]),
    "gpufhe_ctx_device_status": (I32, [VP, VP]),
    "gpufhe_keygen": (I32, [VP, U32, U32, U64, C.c_double, U64, VP, VP, VP, VP]),
    "gpufhe_evalkeygen": (I32, [VP, U32, VP, VP, VP, VP, VP, VP, U64, C.c_double, VP, VP, VP]),
    "gpufhe_ctx_set_key_device": (I32, [VP, U64, VP, VP]),
    "gpufhe_encrypt_batch": (I32, [VP, U32, U32, VP, VP, VP, VP, U64, C.c_double, VP, VP, VP]),
    "gpufhe_decrypt_batch": (I32, [VP, U32, VP, VP, VP, VP, VP]),
    "gpufhe_decrypt_crt_batch": (I32, [VP, U32, U32, VP, VP, VP, VP, VP]),
    "gpufhe_modraise_batch": (I32, [VP, U32, U32, VP, VP, VP, VP, VP]),
    "gpufhe_pt_to_eval_batch": (I32, [VP, U32, U32, VP, VP, VP]),
    "gpufhe_pointwise_batch": (I32, [VP, U32, VP, VP]),
    "gpufhe_encoder_create": (I32, [U32, I32, C.POINTER(VP)]),
    "gpufhe_encoder_destroy": (None, [VP]),
    "gpufhe_encode_batch": (I32, [VP, U32, VP, C.c_double, VP, VP]),
    "gpufhe_decode_batch": (I32, [VP, U32, VP, C.c_double, VP, VP]),
    "gpufhe_encode_batch_fast": (I32, [VP, U32, VP, C.c_double, VP, VP]),
    "gpufhe_decode_batch_fast": (I32, [VP, U32, VP, C.c_double, VP, VP]),
    "gpufhe_ntt_batch": (I32, [VP, VP, U32, U32, U32, I32, VP, VP]),
    "gpufhe_ntt_job_bytes": (U64, []),
    "gpufhe_ntt_run_jobs": (I32, [VP, VP, U32, I32, VP]),
    "gpufhe_approx_switch": (I32, [VP, VP, VP, VP, VP, VP, VP, VP, VP, U32, U32, U32, I32, VP]),
    "gpufhe_approx_switch_status": (I32, [VP]),
    "gpufhe_rns_mult_batch": (I32, [VP, VP, VP, VP, U32, U32, U32, VP]),
    "gpufhe_op_workspace_bytes": (U64, [VP, U32]),
    "gpufhe_plan_create": (I32, [VP, U32, VP, VP, U64, C.POINTER(VP)]),
    "gpufhe_plan_launch": (I32, [VP, VP]),
    "gpufhe_plan_destroy": (None, [VP]),
    "gpufhe_run_ops": (I32, [VP, U32, VP, VP]),
    "gpufhe_plan_launch_host_batch_async": (I32, [VP, VP, VP, VP]),
    "gpufhe_plan_launch_phase": (I32, [VP, U32, VP]),
    "gpufhe_plan_kernel_count": (U32, [VP]),
    "gpufhe_plan_schedule": (U32, [VP]),
    "gpufhe_plan_set_schedule": (I32, [VP, U32]),
    "gpufhe_plan_launch_host": (I32, [VP, VP, VP, VP]),
    "gpufhe_plan_launch_host_async": (I32, [VP, VP, VP, VP]),
    "gpufhe_native_primes": (I32, [VP, U32, U32, U32, VP, U32]),
    "gpufhe_native_root": (U64, [U32, U64]),
    "gpufhe_rescale_consts": (I32, [VP, VP, VP, U32]),
    "gpufhe_rescale_noalloc": (I32, [VP, U32, VP, VP]),
    "gpufhe_lintrans_bsgs": (I32, [VP, U32, VP, VP, U32, U32, VP, I32, VP, VP, VP]),
    "gpufhe_lintrans_plan_create": (I32, [VP, U32, VP, VP, U32, U32, VP, I32, VP, VP, C.POINTER(VP)]),
    "gpufhe_lintrans_plan_launch": (I32, [VP, VP]),
    "gpufhe_lintrans_plan_destroy": (None, [VP]),
    "gpufhe_rescale_noalloc_max_words": (U64, []),
    "gpufhe_server_create": (I32, [VP, U32, U64, U32, U32, I32, C.POINTER(VP)]),
    "gpufhe_server_destroy": (None, [VP]),
    "gpufhe_server_request_bytes": (U64, [VP, U32, U32]),
    "gpufhe_server_submit": (I32, [VP, U32, U32, VP, U32, DBL, U64, VP, VP, C.POINTER(U64)]),
    "gpufhe_server_start": (I32, [VP]),
    "gpufhe_server_tune": (I32, [VP, U32, C.POINTER(U32)]),
    "gpufhe_server_step": (I32, [VP, C.POINTER(U32)]),
    "gpufhe_server_drain": (I32, [VP, DBL]),
    "gpufhe_server_pending": (U64, [VP]),
    "gpufhe_server_get_stats": (I32, [VP, VP]),
    "gpufhe_server_records": (I32, [VP, VP, U32, C.POINTER(U32)]),
}

EVALMULT_RESCALE, KEYSWITCH, ROTATE, RESCALE, ROTATE_HOISTED = 0, 1, 2, 3, 4


class Op(C.Structure):
    """struct gpufhe_op (include/gpufhe_b200.h)."""
    _fields_ = [("level", U32), ("mode", U32), ("key_id", U64), ("galois", U64),
                ("inp", VP * 4), ("out", VP * 2)]



def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m gpufhe_b200.build` "
                               "(or __graft_entry__.build()) first")
        L = C.CDLL(LIB_PATH)
        for name, args in _REF_ABI.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None
        for name, (res, args) in _API.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def ref_abi_symbols():
    return list(_REF_ABI)


class GpuFheError(RuntimeError):
    pass


def check(rc):
    if rc != 0:
        raise GpuFheError(f"gpufhe status {rc}: {lib().gpufhe_last_error().decode()}")
    return rc


def api_symbols():
    return list(_API)


def _np_u64(a):
    import numpy as np
    return np.ascontiguousarray(a, dtype=np.uint64)


class Encoder:
    """Canonical encode / decode (the reference's encode_host / decode_host)
    on the device, numpy in and out."""

    def __init__(self, n, device=0):
        h = VP()
        check(lib().gpufhe_encoder_create(n, device, C.byref(h)))
        self.h, self.n = h, n

    def close(self):
        if getattr(self, "h", None):
            lib().gpufhe_encoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def encode(self, z, delta, fast=False):
        """z: [count][n/2] or [n/2] complex -> int64 [count][n] (or [n]).
        fast: the O(n log n) form (coefficients within one of the reference's)."""
        import numpy as np
        z = np.asarray(z, dtype=np.complex128)
        one = z.ndim == 1
        z = np.ascontiguousarray(z.reshape(-1, self.n // 2))
        m = np.zeros((z.shape[0], self.n), np.int64)
        f = lib().gpufhe_encode_batch_fast if fast else lib().gpufhe_encode_batch
        check(f(self.h, z.shape[0], z.ctypes.data, float(delta), m.ctypes.data, None))
        return m[0] if one else m

    def decode(self, m, delta, fast=False):
        import numpy as np
        m = np.asarray(m, dtype=np.int64)
        one = m.ndim == 1
        m = np.ascontiguousarray(m.reshape(-1, self.n))
        z = np.zeros((m.shape[0], self.n // 2), np.complex128)
        f = lib().gpufhe_decode_batch_fast if fast else lib().gpufhe_decode_batch
        check(f(self.h, m.shape[0], m.ctypes.data, float(delta), z.ctypes.data, None))
        return z[0] if one else z


class Context:
    """Owns a gpufhe_ctx handle (chain, tables, constants, resident keys)."""

    def __init__(self, n, Q, P, alpha, roots=None, device=0):
        self._Q, self._P = _np_u64(Q), _np_u64(P)
        r = _np_u64(roots) if roots is not None else None
        h = VP()
        check(lib().gpufhe_ctx_create(n, self._Q.ctypes.data, len(self._Q), self._P.ctypes.data, len(self._P),
                                      alpha, r.ctypes.data if r is not None else None, device, C.byref(h)))
        self.h, self.n, self.alpha = h, n, alpha
        self.fullQ, self.K = len(self._Q), len(self._P)

    def close(self):
        if getattr(self, "h", None):
            lib().gpufhe_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_key(self, key_id, av, bv):
        av, bv = _np_u64(av), _np_u64(bv)
        check(lib().gpufhe_ctx_set_key(self.h, key_id, av.ctypes.data, bv.ctypes.data))

    def roots(self):
        import numpy as np
        r = np.zeros(self.fullQ + self.K, np.uint64)
        check(lib().gpufhe_ctx_roots(self.h, r.ctypes.data))
        return r

    def workspace_bytes(self, level):
        return int(lib().gpufhe_op_workspace_bytes(self.h, level))

    def resident_bytes(self):
        return int(lib().gpufhe_ctx_resident_bytes(self.h))

    def set_key_budget(self, nbytes):
        """Caps the device bytes of resident keys (0 = no cap); evicted keys
        live in pinned host copies and come back when a plan needs them."""
        check(lib().gpufhe_ctx_set_key_budget(self.h, int(nbytes)))

    def key_stats(self):
        out = (C.c_uint64 * 6)()
        check(lib().gpufhe_ctx_key_stats(self.h, out))
        return dict(zip(("known", "resident", "resident_bytes", "uploads", "evictions", "budget"), map(int, out)))

    def device_status(self):
        """Synchronises and returns (then clears) the device status word:
        0 unless a bounded wait inside a kernel expired."""
        out = (C.c_uint32 * 1)()
        check(lib().gpufhe_ctx_device_status(self.h, out))
        return int(out[0])

    def key_bytes(self):
        """Device bytes of one key: 2 * dnum * (fullQ + K) * n words."""
        dnum = -(-self.fullQ // self.alpha)
        return 2 * dnum * (self.fullQ + self.K) * self.n * 8


def make_ops(specs):
    """specs: iterable of dicts {level, mode, key_id, galois, inp: [ptrs], out: [ptrs]}."""
    specs = list(specs)
    arr = (Op * max(1, len(specs)))()
    for i, s in enumerate(specs):
        o = arr[i]
        o.level, o.mode = s["level"], s.get("mode", EVALMULT_RESCALE)
        o.key_id, o.galois = s.get("key_id", 0), s.get("galois", 0)
        for k, p in enumerate(s.get("inp", [])):
            o.inp[k] = p
        for k, p in enumerate(s.get("out", [])):
            o.out[k] = p
    return arr, len(specs)


class Plan:
    """A built batch (job tables + workspace); launch() only enqueues kernels."""

    def __init__(self, ctx, specs, d_ws=None, ws_bytes=0):
        self.ops, self.nops = make_ops(specs)
        h = VP()
        check(lib().gpufhe_plan_create(ctx.h, self.nops, C.cast(self.ops, VP), d_ws, ws_bytes, C.byref(h)))
        self.h = h
        self._ctx = ctx                  # the context object outlives the plan

    def launch(self, stream=None):
        check(lib().gpufhe_plan_launch(self.h, stream))

    def set_schedule(self, bits):
        """Fix the launch schedule (bits 0-1 P5 form, bit 2 interleaved paths, bits 3-4 P3 form)."""
        check(lib().gpufhe_plan_set_schedule(self.h, bits))

    def launch_phase(self, phase, stream=None):
        check(lib().gpufhe_plan_launch_phase(self.h, phase, stream))

    def kernel_count(self):
        return int(lib().gpufhe_plan_kernel_count(self.h))

    def schedule(self):
        """Autotuner choice: {'p5': form, 'mixed_paths': bool, 'tuned': bool}."""
        b = int(lib().gpufhe_plan_schedule(self.h))
        form = {0: "register-128x4", 1: "cp.async", 2: "register-256x2", 3: "tma"}.get(b & 3, "?")
        p3 = {0: "plain", 1: "warp-specialised-128x2", 2: "warp-specialised-256x1"}.get((b >> 3) & 3, "?")
        mixed = [k + 1 for k in range(9) if b >> (8 + k) & 1]
        return {"p5": form, "p5_fp64_rows": bool(b & 64), "p5_fp64_form": (2 if b >> 18 & 1 else 0) + ((b >> 7) & 1), "p5_split": bool(b >> 17 & 1), "mixed_paths": bool(b & 4), "mixed_phases": mixed,
                "p3": p3, "tuned": bool(b & 32)}

    def launch_host(self, h_in, h_out, stream=None, sync=True):
        """h_in: list of 4 host pointers per op (0 for unused); h_out: 2 per op.
        sync=False queues the copies and kernels only (pinned host buffers)."""
        ai = (VP * len(h_in))(*h_in)
        ao = (VP * len(h_out))(*h_out)
        f = lib().gpufhe_plan_launch_host if sync else lib().gpufhe_plan_launch_host_async
        check(f(self.h, ai, ao, stream))

    def launch_host_batch(self, h_in, h_out, stream=None, sync=True):
        """h_in / h_out: one pinned host buffer each, all ops' inputs / outputs
        back to back in op order (gpufhe_plan_launch_host_batch_async)."""
        check(lib().gpufhe_plan_launch_host_batch_async(self.h, h_in, h_out, stream))
        if sync:
            import torch
            torch.cuda.synchronize()

    def close(self):
        if getattr(self, "h", None):
            lib().gpufhe_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ReqOp(C.Structure):
    """struct gpufhe_req_op (include/gpufhe_b200.h)."""
    _fields_ = [("mode", U32), ("reserved", U32), ("galois", U64)]


class ServerStats(C.Structure):
    """struct gpufhe_server_stats."""
    _fields_ = [("steps", U64), ("ops", U64), ("emr_ops", U64), ("completed", U64), ("peak_active", U64),
                ("max_batch", U64), ("peak_bytes", U64), ("arena_bytes", U64), ("resident_bytes", U64),
                ("busy_s", DBL), ("host_build_s", DBL), ("host_wait_s", DBL)]


class RequestRecord(C.Structure):
    """struct gpufhe_request_record."""
    _fields_ = [("id", U64), ("ctx", U32), ("start_level", U32), ("final_level", U32), ("nops", U32),
                ("t_arrival", DBL), ("t_admit", DBL), ("t_finish", DBL)]


class Server:
    """Continuous-batching server over contexts of one device (gpufhe_server_*)."""

    def __init__(self, ctxs, budget_bytes, max_active=0, batch_cap=0, plain=False):
        self._ctxs = list(ctxs)          # keep the contexts alive
        arr = (VP * len(self._ctxs))(*[c.h.value for c in self._ctxs])
        h = VP()
        check(lib().gpufhe_server_create(arr, len(self._ctxs), int(budget_bytes), max_active, batch_cap,
                                         1 if plain else 0, C.byref(h)))
        self.h = h
        self._keep = []                  # host buffers referenced by queued requests

    def request_bytes(self, ctx, level):
        return int(lib().gpufhe_server_request_bytes(self.h, ctx, level))

    def submit(self, ctx, level, ops, arrival_s=0.0, seed=0, h_in=None, h_out=None):
        """ops: list of (mode, galois). h_in / h_out: host numpy uint64 arrays or None."""
        arr = (ReqOp * max(1, len(ops)))()
        for i, (m, g) in enumerate(ops):
            arr[i].mode, arr[i].galois = m, g
        if h_in is not None:
            self._keep.append(h_in)
        if h_out is not None:
            self._keep.append(h_out)
        rid = U64()
        check(lib().gpufhe_server_submit(self.h, ctx, level, C.cast(arr, VP), len(ops), float(arrival_s), seed,
                                         None if h_in is None else h_in.ctypes.data,
                                         None if h_out is None else h_out.ctypes.data, C.byref(rid)))
        return rid.value

    def start(self):
        check(lib().gpufhe_server_start(self.h))

    def tune(self, max_batch=256):
        """Autotune every context's schedule on batches of 1..max_batch EvalMult+Rescale operations."""
        t = U32()
        check(lib().gpufhe_server_tune(self.h, max_batch, C.byref(t)))
        return t.value

    def step(self):
        q = U32()
        check(lib().gpufhe_server_step(self.h, C.byref(q)))
        return q.value

    def drain(self, max_seconds=600.0):
        check(lib().gpufhe_server_drain(self.h, float(max_seconds)))

    def pending(self):
        return int(lib().gpufhe_server_pending(self.h))

    def stats(self):
        st = ServerStats()
        check(lib().gpufhe_server_get_stats(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def records(self):
        cnt = U32()
        check(lib().gpufhe_server_records(self.h, None, 0, C.byref(cnt)))
        arr = (RequestRecord * max(1, cnt.value))()
        check(lib().gpufhe_server_records(self.h, C.cast(arr, VP), cnt.value, C.byref(cnt)))
        return [{k: getattr(arr[i], k) for k, _ in RequestRecord._fields_} for i in range(cnt.value)]

    def close(self):
        if getattr(self, "h", None):
            lib().gpufhe_server_destroy(self.h)
            self.h = None
        self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PW_ADD, PW_SUB, PW_MUL_PT, PW_ADD_PT, PW_SUB_PT, PW_MUL_INT = range(6)


class PwOp(C.Structure):
    """struct gpufhe_pw_op."""
    _fields_ = [("kind", U32), ("towers", U32), ("a0", VP), ("a1", VP), ("b0", VP), ("b1", VP),
                ("o0", VP), ("o1", VP), ("scalar", U64)]


def pointwise(ctx, ops, stream=None):
    """ops: dicts {kind, towers, a: (a0, a1), b: (b0, b1) or (pt,), o: (o0, o1), scalar}
    of device pointers; one launch for the whole list."""
    arr = (PwOp * len(ops))()
    for i, o in enumerate(ops):
        b = tuple(o.get("b", ())) + (None, None)
        arr[i] = PwOp(o["kind"], o["towers"], o["a"][0], o["a"][1], b[0], b[1], o["o"][0], o["o"][1],
                      int(o.get("scalar", 0)))
    check(lib().gpufhe_pointwise_batch(ctx.h, len(ops), C.cast(arr, VP), stream))


def lintrans_bsgs(ctx, level, c0, c1, n1, n2, diags, out0, out1, hoisted=False, stream=None):
    """Baby-step giant-step linear transform; diags: n1*n2 device pointers (or None), index g*n1+b."""
    arr = (VP * len(diags))(*[d if d else None for d in diags])
    check(lib().gpufhe_lintrans_bsgs(ctx.h, level, c0, c1, n1, n2, C.cast(arr, VP), 1 if hoisted else 0,
                                     out0, out1, stream))


def run_ops(ctx, specs, stream=None):
    ops, n = make_ops(specs)
    check(lib().gpufhe_run_ops(ctx.h, n, C.cast(ops, VP), stream))


def native_primes(count, bits, n, avoid=()):
    import numpy as np
    out = np.zeros(count, np.uint64)
    av = np.ascontiguousarray(list(avoid), np.uint64)
    check(lib().gpufhe_native_primes(out.ctypes.data, count, bits, n, av.ctypes.data if len(av) else None, len(av)))
    return out


def native_root(n, q):
    return int(lib().gpufhe_native_root(n, int(q)))
