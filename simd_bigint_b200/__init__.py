"""simd_bigint_b200 -- B200 (sm_100a) large-operand multiplication for
mpn-style little-endian uint64 limb arrays.

The product is the native library ``_lib/libsimd_bigint_b200.so`` (C ABI,
``include/simd_bigint_b200.h``).  This module is a thin ctypes host layer
over it for Python callers, tests and the benchmark: it mirrors the
reference's entry points (``nt_mul``, ``nt_sqr``; include/ntmul.h:71-80) with
the same argument order and meaning, and exposes the context (stream +
workspace) API for device-resident operands held in torch tensors.

There is no CPU fallback: if the library or a CUDA device is missing, the
calls raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

__all__ = [
    "SbgError", "lib", "Context", "nt_mul", "nt_sqr", "mpn_mulmid", "STATUS",
]

STATUS = {
    0: "SBG_OK", 1: "SBG_EINVAL", 2: "SBG_EBAND", 3: "SBG_EALLOC", 4: "SBG_ECUDA",
    5: "SBG_ETIMEOUT", 6: "SBG_ESPILL", 7: "SBG_EADMIT", 8: "SBG_ENODEV", 9: "SBG_ECANCELED",
}

_lib = None
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p
_i64 = C.c_int64


class SbgError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")


def lib_path() -> Path:
    return _build.lib_path()


def lib(build_if_missing: bool = False):
    """Load the native library (raises if it is not built)."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not path.exists():
            if not build_if_missing:
                raise FileNotFoundError(f"native library missing: {path} (run python -m simd_bigint_b200.build)")
            _build.build()
        L = C.CDLL(str(path))
        L.sbg_ctx_create.argtypes = [C.c_int, C.POINTER(_vp)]
        L.sbg_ctx_create.restype = C.c_int
        L.sbg_ctx_destroy.argtypes = [_vp]
        L.sbg_ctx_destroy.restype = None
        L.sbg_ctx_set_stream.argtypes = [_vp, _vp]
        L.sbg_ctx_set_stream.restype = C.c_int
        L.sbg_ctx_get_stream.argtypes = [_vp]
        L.sbg_ctx_get_stream.restype = _vp
        L.sbg_ctx_sync.argtypes = [_vp]
        L.sbg_ctx_sync.restype = C.c_int
        L.sbg_ctx_reserve.argtypes = [_vp, _i64]
        L.sbg_ctx_reserve.restype = C.c_int
        L.sbg_ctx_set_timing.argtypes = [_vp, C.c_int]
        L.sbg_ctx_set_timing.restype = C.c_int
        L.sbg_ctx_kernel_times.argtypes = [_vp, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int]
        L.sbg_ctx_kernel_times.restype = C.c_int
        L.sbg_strerror.argtypes = [C.c_int]
        L.sbg_strerror.restype = C.c_char_p
        L.sbg_max_total_limbs.argtypes = []
        L.sbg_max_total_limbs.restype = _i64
        for name in ("sbg_mul", "sbg_mulmid"):
            getattr(L, name).argtypes = [_vp, _vp, _vp, _i64, _vp, _i64]
            getattr(L, name).restype = C.c_int
        L.sbg_sqr.argtypes = [_vp, _vp, _vp, _i64]
        L.sbg_sqr.restype = C.c_int
        L.sbg_mul_host.argtypes = [_vp, _vp, _vp, _i64, _vp, _i64]
        L.sbg_mul_host.restype = C.c_int
        L.sbg_sqr_host.argtypes = [_vp, _vp, _vp, _i64]
        L.sbg_sqr_host.restype = C.c_int
        L.sbg_nt_mul.argtypes = [_vp, _vp, C.c_ssize_t, _vp, C.c_ssize_t]
        L.sbg_nt_mul.restype = C.c_int
        L.sbg_nt_sqr.argtypes = [_vp, _vp, C.c_ssize_t]
        L.sbg_nt_sqr.restype = C.c_int
        L.sbg_probe_bfly_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
        L.sbg_probe_bfly_peak.restype = C.c_int
        L.sbg_batch_create.argtypes = [_vp, _vp, _i64, C.POINTER(_vp)]
        L.sbg_batch_create.restype = C.c_int
        L.sbg_batch_capture.argtypes = [_vp]
        L.sbg_batch_capture.restype = C.c_int
        L.sbg_batch_run.argtypes = [_vp]
        L.sbg_batch_run.restype = C.c_int
        L.sbg_batch_destroy.argtypes = [_vp]
        L.sbg_batch_destroy.restype = None
        L.sbg_mul_batch.argtypes = [_vp, _vp, _i64]
        L.sbg_mul_batch.restype = C.c_int
        L.sbg_recip.argtypes = [_vp, _vp, _vp, _i64]
        L.sbg_recip.restype = C.c_int
        L.sbg_divrem.argtypes = [_vp, _vp, _vp, _vp, _i64, _vp, _i64]
        L.sbg_divrem.restype = C.c_int
        L.sbg_divrem_batch.argtypes = [_vp, _vp, _i64]
        L.sbg_divrem_batch.restype = C.c_int
        L.sbg_divrem_batch_async.argtypes = [_vp, _vp, _i64]
        L.sbg_divrem_batch_async.restype = C.c_int
        L.sbg_divrem_wait.argtypes = [_vp]
        L.sbg_divrem_wait.restype = C.c_int
        L.sbg_divrem_u64.argtypes = [_vp, _vp, _vp, C.c_uint64, _vp, C.c_uint64,
                                     C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.sbg_divrem_u64.restype = C.c_int
        L.sbg_server_create.argtypes = [_vp, _vp, C.POINTER(_vp)]
        L.sbg_server_create.restype = C.c_int
        L.sbg_server_submit.argtypes = [_vp, _vp, C.POINTER(C.c_uint64)]
        L.sbg_server_submit.restype = C.c_int
        L.sbg_server_submit_many.argtypes = [_vp, _vp, _i64, _vp, C.POINTER(_i64)]
        L.sbg_server_submit_many.restype = C.c_int
        L.sbg_server_poll.argtypes = [_vp, _vp, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.sbg_server_poll.restype = C.c_int
        L.sbg_server_release.argtypes = [_vp, C.c_uint64]
        L.sbg_server_release.restype = C.c_int
        L.sbg_server_cancel.argtypes = [_vp, C.c_uint64]
        L.sbg_server_cancel.restype = C.c_int
        L.sbg_debug_inject.argtypes = [C.c_uint32]
        L.sbg_debug_inject.restype = C.c_int
        L.sbg_debug_fail_allocs.argtypes = [C.c_int]
        L.sbg_debug_fail_allocs.restype = None
        L.sbg_noalloc_status.argtypes = [_vp]
        L.sbg_noalloc_status.restype = C.c_int
        L.sbg_mul_noalloc.argtypes = [_vp, _vp, _i64, _vp, _i64, _vp]
        L.sbg_mul_noalloc.restype = C.c_int
        L.sbg_batch_set_engine.argtypes = [_vp, C.c_int, _i64]
        L.sbg_batch_set_engine.restype = C.c_int
        L.sbg_batch_autotune.argtypes = [_vp, C.POINTER(C.c_double)]
        L.sbg_batch_autotune.restype = C.c_int
        L.sbg_u52_from_u64.argtypes = [_vp, _vp, _i64, _vp, _i64]
        L.sbg_u52_from_u64.restype = C.c_int
        L.sbg_u64_from_u52.argtypes = [_vp, _vp, _i64, _vp, _i64, C.c_int]
        L.sbg_u64_from_u52.restype = C.c_int
        L.sbg_mul_u52.argtypes = [_vp, _vp, _vp, _i64, _vp, _i64]
        L.sbg_mul_u52.restype = C.c_int
        L.sbg_server_stats.argtypes = [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64), C.POINTER(C.c_size_t)]
        L.sbg_server_stats.restype = C.c_int
        L.sbg_server_launches.argtypes = [_vp]
        L.sbg_server_launches.restype = _i64
        L.sbg_ctx_launches.argtypes = [_vp]
        L.sbg_ctx_launches.restype = _i64
        L.sbg_ctx_autotune.argtypes = [_vp, C.POINTER(C.c_double)]
        L.sbg_ctx_autotune.restype = C.c_int
        L.sbg_ctx_set_len3_mask.argtypes = [_vp, C.c_uint32]
        L.sbg_ctx_set_len3_mask.restype = C.c_int
        L.sbg_ctx_get_len3_mask.argtypes = [_vp]
        L.sbg_ctx_get_len3_mask.restype = C.c_uint32
        L.sbg_server_destroy.argtypes = [_vp]
        L.sbg_server_destroy.restype = None
        _lib = L
    return _lib


def _check(st: int, what: str):
    if st != 0:
        raise SbgError(st, what)


def _dptr(t) -> int:
    """Device address of a torch tensor (int64/uint64 limbs) or a raw int."""
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise ValueError("device entry points need CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("limb tensors must be contiguous")
    return t.data_ptr()


class Context:
    """One CUDA stream + twiddle plans + device workspace (the reference's
    scratch* argument, include/ntmul.h:47).  Device entry points queue work on
    the context's stream and return immediately; sync() waits and raises any
    sticky device-side error."""

    def __init__(self, device: int = 0, stream=None):
        self._L = lib()
        h = _vp()
        _check(self._L.sbg_ctx_create(device, C.byref(h)), "sbg_ctx_create")
        self.handle = h
        self.device = device
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if getattr(self, "handle", None):
            self._L.sbg_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream):
        """stream: a torch.cuda.Stream, a raw cudaStream_t int, or None."""
        raw = getattr(stream, "cuda_stream", stream)
        _check(self._L.sbg_ctx_set_stream(self.handle, raw), "sbg_ctx_set_stream")

    @property
    def stream(self) -> int:
        return self._L.sbg_ctx_get_stream(self.handle) or 0

    def sync(self):
        _check(self._L.sbg_ctx_sync(self.handle), "sbg_ctx_sync")

    KERNEL_NAMES = ("k_small", "k_col_fwd", "k_row", "k_col_inv", "k_crt_carry", "k_batch",
                    "k_div", "k_other")

    def set_timing(self, on: bool):
        _check(self._L.sbg_ctx_set_timing(self.handle, int(bool(on))), "sbg_ctx_set_timing")

    def kernel_times(self) -> dict:
        """{kernel name: (total ms, launches)} since the previous call."""
        ms = (C.c_double * 8)()
        cnt = (C.c_int64 * 8)()
        _check(self._L.sbg_ctx_kernel_times(self.handle, ms, cnt, 8), "sbg_ctx_kernel_times")
        return {self.KERNEL_NAMES[i]: (ms[i], cnt[i]) for i in range(8) if cnt[i]}

    def reserve(self, total_limbs: int):
        _check(self._L.sbg_ctx_reserve(self.handle, int(total_limbs)), "sbg_ctx_reserve")

    # device entries (torch CUDA tensors of 64-bit limbs, or raw addresses)
    def mul(self, r, a, b, an: int | None = None, bn: int | None = None):
        an = a.numel() if an is None else an
        bn = b.numel() if bn is None else bn
        _check(self._L.sbg_mul(self.handle, _dptr(r), _dptr(a), an, _dptr(b), bn), "sbg_mul")

    def sqr(self, r, a, an: int | None = None):
        an = a.numel() if an is None else an
        _check(self._L.sbg_sqr(self.handle, _dptr(r), _dptr(a), an), "sbg_sqr")

    def mul_host(self, r: np.ndarray, a: np.ndarray, b: np.ndarray):
        """Queue r = a * b on HOST uint64 arrays (sbg_mul_host); r is valid
        after sync().  Page-locked arrays overlap consecutive products."""
        _check(self._L.sbg_mul_host(self.handle, r.ctypes.data, a.ctypes.data, len(a), b.ctypes.data, len(b)),
               "sbg_mul_host")

    def sqr_host(self, r: np.ndarray, a: np.ndarray):
        _check(self._L.sbg_sqr_host(self.handle, r.ctypes.data, a.ctypes.data, len(a)), "sbg_sqr_host")

    def launches(self) -> int:
        """Kernel launches this context has queued so far."""
        return int(self._L.sbg_ctx_launches(self.handle))

    def autotune(self) -> dict:
        """sbg_ctx_autotune: {k: (ms at 2^(k+2), ms at 3*2^k)} and the chosen mask."""
        t = (C.c_double * 16)()
        _check(self._L.sbg_ctx_autotune(self.handle, t), "sbg_ctx_autotune")
        return {"times": {16 + i: (t[2 * i], t[2 * i + 1]) for i in range(8)},
                "len3_mask": int(self._L.sbg_ctx_get_len3_mask(self.handle))}

    def set_len3_mask(self, mask: int):
        _check(self._L.sbg_ctx_set_len3_mask(self.handle, mask), "sbg_ctx_set_len3_mask")

    @property
    def len3_mask(self) -> int:
        return int(self._L.sbg_ctx_get_len3_mask(self.handle))

    def recip(self, i, d, n: int | None = None):
        """i[0..n) = floor((B^2n - 1) / D) - B^n for a normalised n-limb D."""
        n = d.numel() if n is None else n
        _check(self._L.sbg_recip(self.handle, _dptr(i), _dptr(d), n), "sbg_recip")

    def divrem(self, q, r, n_, d, nn: int | None = None, dn: int | None = None):
        """q = N // D (nn-dn+1 limbs), r = N % D (dn limbs); D normalised,
        dn <= nn <= 2 dn."""
        nn = n_.numel() if nn is None else nn
        dn = d.numel() if dn is None else dn
        _check(self._L.sbg_divrem(self.handle, _dptr(q), _dptr(r), _dptr(n_), nn, _dptr(d), dn),
               "sbg_divrem")

    @staticmethod
    def _div_jobs(jobs: list[tuple]):
        arr = (DivJob * max(1, len(jobs)))()
        for i, (q, r, n_, d, nn, dn) in enumerate(jobs):
            arr[i].qp, arr[i].rp, arr[i].np, arr[i].dp, arr[i].nn, arr[i].dn = q, r, n_, d, nn, dn
        return arr

    def divrem_batch(self, jobs: list[tuple]):
        """jobs: (q_ptr, r_ptr, n_ptr, d_ptr, nn, dn) raw device addresses."""
        arr = self._div_jobs(jobs)
        _check(self._L.sbg_divrem_batch(self.handle, C.cast(arr, _vp), len(jobs)), "sbg_divrem_batch")

    def divrem_batch_async(self, jobs: list[tuple]):
        """sbg_divrem_batch_async: queue the batch and return; results are
        ready, and device errors reported, after divrem_wait()."""
        arr = self._div_jobs(jobs)
        _check(self._L.sbg_divrem_batch_async(self.handle, C.cast(arr, _vp), len(jobs)),
               "sbg_divrem_batch_async")

    def divrem_wait(self):
        _check(self._L.sbg_divrem_wait(self.handle), "sbg_divrem_wait")

    def mulmid(self, r, a, b, an: int | None = None, bn: int | None = None):
        an = a.numel() if an is None else an
        bn = b.numel() if bn is None else bn
        _check(self._L.sbg_mulmid(self.handle, _dptr(r), _dptr(a), an, _dptr(b), bn), "sbg_mulmid")

    # ---- u52 redundant-digit boundary (device tensors of 64-bit lanes) ----
    def u52_from_u64(self, d, a):
        """d[i] = bits [52 i, 52 i + 52) of a, for i < d.numel()."""
        _check(self._L.sbg_u52_from_u64(self.handle, _dptr(d), d.numel(), _dptr(a), a.numel()),
               "sbg_u52_from_u64")

    def u64_from_u52(self, r, d, signed: bool = False):
        """r = sum_i d[i] 2^(52 i) mod 2^(64 r.numel()), lanes unsigned or signed."""
        _check(self._L.sbg_u64_from_u52(self.handle, _dptr(r), r.numel(), _dptr(d), d.numel(), int(signed)),
               "sbg_u64_from_u52")

    def mul_u52(self, r, a, b):
        """r (a.numel() + b.numel() digits) = the canonical digits of a * b."""
        _check(self._L.sbg_mul_u52(self.handle, _dptr(r), _dptr(a), a.numel(), _dptr(b), b.numel()),
               "sbg_mul_u52")


JOB_MUL, JOB_SQR, JOB_MULMID = 0, 1, 2


class DivJob(C.Structure):
    """sbg_div_job (include/simd_bigint_b200.h)."""
    _fields_ = [("qp", C.c_void_p), ("rp", C.c_void_p), ("np", C.c_void_p), ("dp", C.c_void_p),
                ("nn", C.c_int64), ("dn", C.c_int64)]


class Job(C.Structure):
    """sbg_job (include/simd_bigint_b200.h)."""
    _fields_ = [("rp", C.c_void_p), ("ap", C.c_void_p), ("bp", C.c_void_p),
                ("an", C.c_int64), ("bn", C.c_int64), ("kind", C.c_int32), ("reserved", C.c_int32)]


def out_limbs(kind: int, an: int, bn: int) -> int:
    return an + bn if kind == JOB_MUL else (2 * an if kind == JOB_SQR else an - bn + 3)


class Batch:
    """A planned batch of independent products on device pointers (raw
    addresses), run in a few launches per size class; optionally captured
    into a CUDA graph (capture()) and replayed by run()."""

    def __init__(self, ctx: Context, jobs: list[tuple]):
        """jobs: (kind, r_ptr, a_ptr, b_ptr, an, bn) with raw device addresses."""
        self._L = lib()
        self.ctx = ctx
        arr = (Job * max(1, len(jobs)))()
        for i, (kind, r, a, b, an, bn) in enumerate(jobs):
            arr[i].kind, arr[i].rp, arr[i].ap, arr[i].bp = kind, r, a, b
            arr[i].an, arr[i].bn = an, bn
        self._jobs = arr
        h = _vp()
        _check(self._L.sbg_batch_create(ctx.handle, C.cast(arr, _vp), len(jobs), C.byref(h)),
               "sbg_batch_create")
        self.handle = h

    def capture(self):
        _check(self._L.sbg_batch_capture(self.handle), "sbg_batch_capture")

    def set_engine(self, engine: int, wave_bytes: int = 0):
        """0: the persistent kernel over a device work-item queue, 1: one
        launch per stage per length class (default), 2: the queue with one
        CTA per item.  wave_bytes: the queue's L2 blocking (0: keep).  Drops a
        captured graph (capture again)."""
        _check(self._L.sbg_batch_set_engine(self.handle, engine, wave_bytes), "sbg_batch_set_engine")

    def autotune(self) -> list[float]:
        """Times each engine on this batch and keeps the fastest; returns the
        per-run milliseconds of engines 0, 1, 2."""
        ms = (C.c_double * 3)()
        _check(self._L.sbg_batch_autotune(self.handle, ms), "sbg_batch_autotune")
        return list(ms)

    def run(self):
        _check(self._L.sbg_batch_run(self.handle), "sbg_batch_run")

    def close(self):
        if getattr(self, "handle", None):
            self._L.sbg_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


REQ_MUL, REQ_SQR, REQ_RECIP = 0, 1, 2
# test hooks of the CRT kernel (sbg_debug_inject)
INJECT_WITHHOLD, INJECT_TOP, INJECT_MID = 1, 2, 4


class Request(C.Structure):
    """sbg_request."""
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("ap", C.c_void_p), ("an", C.c_int64),
                ("bp", C.c_void_p), ("bn", C.c_int64)]


class Completion(C.Structure):
    """sbg_completion."""
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("reserved", C.c_int32),
                ("rp", C.c_void_p), ("rn", C.c_int64), ("latency_s", C.c_double), ("queue_s", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("arena_bytes", C.c_size_t), ("slots", C.c_int32), ("max_batch", C.c_int32),
                ("recip_workers", C.c_int32), ("batch_lg_points", C.c_int32)]


class Server:
    """The serving loop (sbg_server_*): submit device-operand requests from
    any thread, poll completions (device result pointer + latency), release."""

    def __init__(self, ctx: Context, arena_bytes: int = 8 << 30, slots: int = 4, max_batch: int = 512,
                 recip_workers: int = 2, batch_lg_points: int = 0):
        self._L = lib()
        self.ctx = ctx
        cfg = ServerConfig(arena_bytes, slots, max_batch, recip_workers, batch_lg_points)
        h = _vp()
        _check(self._L.sbg_server_create(ctx.handle, C.byref(cfg), C.byref(h)), "sbg_server_create")
        self.handle = h
        self._buf = (Completion * 4096)()

    def submit(self, kind: int, ap: int, an: int, bp: int = 0, bn: int = 0) -> int:
        req = Request(kind, 0, ap, an, bp, bn)
        t = C.c_uint64(0)
        _check(self._L.sbg_server_submit(self.handle, C.byref(req), C.byref(t)), "sbg_server_submit")
        return t.value

    def try_submit(self, kind: int, ap: int, an: int, bp: int = 0, bn: int = 0) -> tuple[int, int]:
        req = Request(kind, 0, ap, an, bp, bn)
        t = C.c_uint64(0)
        st = self._L.sbg_server_submit(self.handle, C.byref(req), C.byref(t))
        return st, t.value

    def submit_many(self, reqs: list[tuple]) -> list[int]:
        """reqs: (kind, ap, an, bp, bn) tuples, queued under one lock; returns tickets."""
        n = len(reqs)
        arr = (Request * max(1, n))()
        for i, (kind, ap, an, bp, bn) in enumerate(reqs):
            arr[i].kind, arr[i].ap, arr[i].an, arr[i].bp, arr[i].bn = kind, ap, an, bp or None, bn
        t = (C.c_uint64 * max(1, n))()
        acc = _i64(0)
        _check(self._L.sbg_server_submit_many(self.handle, C.cast(arr, _vp), n, C.cast(t, _vp), C.byref(acc)),
               "sbg_server_submit_many")
        return list(t[: acc.value])

    def poll(self, wait_ms: int = 0) -> list[tuple[int, int, int, int, float]]:
        """[(ticket, status, result device pointer, result limbs, latency_s)];
        poll_detail() adds the queueing part of each latency."""
        n = C.c_int(0)
        _check(self._L.sbg_server_poll(self.handle, C.cast(self._buf, _vp), 4096, C.byref(n), wait_ms),
               "sbg_server_poll")
        return [(c.ticket, c.status, c.rp or 0, c.rn, c.latency_s) for c in self._buf[: n.value]]

    def poll_detail(self, wait_ms: int = 0) -> list[tuple[int, int, int, int, float, float]]:
        """[(ticket, status, result pointer, result limbs, latency_s, queue_s)]"""
        n = C.c_int(0)
        _check(self._L.sbg_server_poll(self.handle, C.cast(self._buf, _vp), 4096, C.byref(n), wait_ms),
               "sbg_server_poll")
        return [(c.ticket, c.status, c.rp or 0, c.rn, c.latency_s, c.queue_s) for c in self._buf[: n.value]]

    def result(self, rp: int, rn: int):
        """torch.int64 view of a completed result in the server's arena; valid
        until the ticket is released."""
        return device_limbs(rp, rn)

    def release(self, ticket: int):
        _check(self._L.sbg_server_release(self.handle, ticket), "sbg_server_release")

    def cancel(self, ticket: int) -> bool:
        """Cancels a still-queued request (it completes with SBG_ECANCELED);
        False when it was already launched or completed."""
        return self._L.sbg_server_cancel(self.handle, ticket) == 0

    def launches(self) -> int:
        """Kernel launches the server has queued so far."""
        return int(self._L.sbg_server_launches(self.handle))

    def stats(self) -> dict:
        p, c, b, u = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_size_t(0)
        _check(self._L.sbg_server_stats(self.handle, C.byref(p), C.byref(c), C.byref(b), C.byref(u)),
               "sbg_server_stats")
        return {"pending": p.value, "completed": c.value, "batches": b.value, "arena_used": u.value}

    def close(self):
        if getattr(self, "handle", None):
            self._L.sbg_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _DevArray:
    """Minimal __cuda_array_interface__ holder for a raw device pointer."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_limbs(ptr: int, n: int):
    """torch.int64 CUDA tensor viewing n limbs at device address ptr (no copy)."""
    import torch
    return torch.as_tensor(_DevArray(ptr, n), device="cuda")


def _np_u64(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.uint64)


def nt_mul(rp: np.ndarray, ap: np.ndarray, an: int, bp: np.ndarray, bn: int) -> int:
    """Reference-signature multiply (include/ntmul.h:71): rp[0..an+bn) =
    {ap,an} * {bp,bn} on host arrays; returns 1 on success, 0 on failure."""
    for arr in (rp, ap, bp):
        if not (isinstance(arr, np.ndarray) and arr.dtype == np.uint64 and arr.flags.c_contiguous):
            raise TypeError("nt_mul wants contiguous uint64 numpy arrays")
    if len(rp) < an + bn:
        raise ValueError("rp too short")
    return lib().sbg_nt_mul(rp.ctypes.data, ap.ctypes.data, an, bp.ctypes.data, bn)


def nt_sqr(rp: np.ndarray, ap: np.ndarray, an: int) -> int:
    """Reference-signature square (include/ntmul.h:77)."""
    for arr in (rp, ap):
        if not (isinstance(arr, np.ndarray) and arr.dtype == np.uint64 and arr.flags.c_contiguous):
            raise TypeError("nt_sqr wants contiguous uint64 numpy arrays")
    if len(rp) < 2 * an:
        raise ValueError("rp too short")
    return lib().sbg_nt_sqr(rp.ctypes.data, ap.ctypes.data, an)


def mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Host convenience: returns {a} * {b} as len(a)+len(b) limbs."""
    a, b = _np_u64(a), _np_u64(b)
    r = np.zeros(len(a) + len(b), dtype=np.uint64)
    if not nt_mul(r, a, len(a), b, len(b)):
        raise SbgError(2, "nt_mul")
    return r


def sqr(a: np.ndarray) -> np.ndarray:
    a = _np_u64(a)
    r = np.zeros(2 * len(a), dtype=np.uint64)
    if not nt_sqr(r, a, len(a)):
        raise SbgError(2, "nt_sqr")
    return r


def divrem_u64(n: np.ndarray, d: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Reference-signature division (include/divrem.h:218) on host arrays:
    returns (Q, R) trimmed to their lengths as the reference reports them."""
    n = _np_u64(n)
    d = _np_u64(d)
    q = np.zeros(len(n) - len(d) + 1, dtype=np.uint64)
    r = np.zeros(len(d), dtype=np.uint64)
    qn, rn = C.c_uint64(0), C.c_uint64(0)
    if not lib().sbg_divrem_u64(q.ctypes.data, r.ctypes.data, n.ctypes.data, len(n), d.ctypes.data,
                                len(d), C.byref(qn), C.byref(rn)):
        raise SbgError(4, "sbg_divrem_u64")
    return q[: qn.value], r[: rn.value]


def probe_bfly_peak(device: int = 0) -> float:
    """Butterflies/s of the transform butterfly on registers (integer ceiling)."""
    v = C.c_double(0.0)
    _check(lib().sbg_probe_bfly_peak(device, C.byref(v)), "sbg_probe_bfly_peak")
    return v.value


def mpn_mulmid(ctx: Context, a, b):
    """Device middle product of torch tensors; returns a new tensor of
    len(a)-len(b)+3 limbs (GMP mpn_mulmid convention)."""
    import torch
    r = torch.empty(a.numel() - b.numel() + 3, dtype=torch.int64, device=a.device)
    ctx.mulmid(r, a, b)
    return r
