"""ctypes front-end of the oracle libraries.

ORACLE / TEST INFRASTRUCTURE ONLY: imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the
product package (simd_bigint_b200).

Two libraries:
  * port -- oracle/_build/libsbg_oracle.so, our C restatement (oracle/port.c);
  * ref  -- oracle/_ref/libsbref.so, the UNMODIFIED reference compiled from its
            own sources by oracle/Makefile (needs AVX-512 IFMA/VBMI/VBMI2 on
            the host; absent or unusable -> ref_available() is False).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "_build" / "libsbg_oracle.so"
REF_SO = HERE / "_ref" / "libsbref.so"
REF_ISA = ("avx512f", "avx512bw", "avx512dq", "avx512vl", "avx512cd", "avx512ifma",
           "avx512vbmi", "avx512_vbmi2", "avx512_vpopcntdq", "avx512_bitalg")

_u64p = C.POINTER(C.c_uint64)
_port = None
_ref = None


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_u64p)


def host_cpu() -> dict:
    flags = set()
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
                elif line.startswith("model name") and model == "unknown":
                    model = line.split(":", 1)[1].strip()
    except OSError:
        pass
    return {"model": model, "flags": flags, "cores": os.cpu_count() or 1}


def build_port() -> Path:
    if not PORT_SO.exists() or PORT_SO.stat().st_mtime < (HERE / "port.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    return PORT_SO


def port():
    global _port
    if _port is None:
        lib = C.CDLL(str(build_port()))
        i64, u64 = C.c_int64, C.c_uint64
        lib.sbo_xorshift_fill.argtypes = [_u64p, i64, u64]
        lib.sbo_xorshift_fill.restype = u64
        for name in ("sbo_ntt_mul", "sbo_ntt_mulmid"):
            getattr(lib, name).argtypes = [_u64p, _u64p, i64, _u64p, i64]
            getattr(lib, name).restype = C.c_int
        lib.sbo_ntt_sqr.argtypes = [_u64p, _u64p, i64]
        lib.sbo_ntt_sqr.restype = C.c_int
        for name in ("sbo_mul_school", "sbo_mulmid"):
            getattr(lib, name).argtypes = [_u64p, _u64p, i64, _u64p, i64]
            getattr(lib, name).restype = None
        lib.sbo_divrem.argtypes = [_u64p, _u64p, _u64p, i64, _u64p, i64]
        lib.sbo_divrem.restype = None
        lib.sbo_recip.argtypes = [_u64p, _u64p, i64]
        lib.sbo_recip.restype = None
        lib.sbo_mod_u64.argtypes = [_u64p, i64, u64]
        lib.sbo_mod_u64.restype = u64
        lib.sbo_run_threads.argtypes = [C.c_void_p, i64, C.c_int]
        lib.sbo_run_threads.restype = C.c_int
        _port = lib
    return _port


def ref_available() -> bool:
    if not REF_SO.exists():
        return False
    return all(f in host_cpu()["flags"] for f in REF_ISA)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference oracle unavailable (not built or host lacks AVX-512 IFMA/VBMI)")
        lib = C.CDLL(str(REF_SO))
        i64, u64 = C.c_int64, C.c_uint64
        lib.sbref_nt_mul.argtypes = [_u64p, _u64p, i64, _u64p, i64]
        lib.sbref_nt_mul.restype = C.c_int
        lib.sbref_nt_sqr.argtypes = [_u64p, _u64p, i64]
        lib.sbref_nt_sqr.restype = C.c_int
        lib.sbref_simd_mpn_mul.argtypes = [_u64p, _u64p, u64, _u64p, u64]
        lib.sbref_simd_mpn_mul.restype = None
        for name in ("sbref_divrem_u64_dc", "sbref_divrem_u64"):
            getattr(lib, name).argtypes = [_u64p, _u64p, _u64p, u64, _u64p, u64, _u64p, _u64p]
            getattr(lib, name).restype = None
        lib.sbref_mul_router.argtypes = [C.c_int, _u64p, _u64p, u64, _u64p, u64]
        lib.sbref_mul_router.restype = C.c_int
        lib.sbref_u52_from_u64.argtypes = [_u64p, _u64p, u64]
        lib.sbref_u52_from_u64.restype = u64
        lib.sbref_u64_from_u52.argtypes = [_u64p, u64, _u64p, u64, C.c_int]
        lib.sbref_u64_from_u52.restype = None
        lib.sbref_run_threads.argtypes = [C.c_void_p, i64, C.c_int]
        lib.sbref_run_threads.restype = C.c_int
        _ref = lib
    return _ref


# ---------------------------------------------------------------- inputs --
def xorshift(n: int, state: int = 42) -> tuple[np.ndarray, int]:
    """n limbs of the reference tests' xorshift64 stream (tests/p30_test.c:14-15)."""
    out = np.empty(max(n, 1), dtype=np.uint64)
    st = port().sbo_xorshift_fill(_ptr(out), n, state)
    return out[:n], int(st)


def pattern(n: int, pat: str, rng: np.random.Generator | None = None) -> np.ndarray:
    """Fill patterns of the reference batteries: random, all-0xFF (the CRT /
    carry worst case), sparse ((i & 31) == 0 -> 0xFF.., tests/p30_test.c:18-22),
    Weyl-hashed (tests/p50_test.c:19-22)."""
    i = np.arange(n, dtype=np.uint64)
    if pat == "ones":
        return np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF), dtype=np.uint64)
    if pat == "sparse":
        return np.where((i & np.uint64(31)) == 0, np.uint64(0xFFFFFFFFFFFFFFFF), np.uint64(0)).astype(np.uint64)
    if pat == "weyl_a":
        return (i * np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
    if pat == "weyl_b":
        return ((~i) * np.uint64(0xC2B2AE3D27D4EB4F)).astype(np.uint64)
    rng = rng or np.random.default_rng(0)
    return rng.integers(0, 2**64, size=n, dtype=np.uint64)


def to_int(a: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(a, dtype="<u8").tobytes(), "little")


def from_int(x: int, n: int) -> np.ndarray:
    return np.frombuffer(x.to_bytes(8 * n, "little"), dtype="<u8").astype(np.uint64)


# --------------------------------------------------------------- port ops --
def port_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    r = np.zeros(len(a) + len(b), dtype=np.uint64)
    if not port().sbo_ntt_mul(_ptr(r), _ptr(a), len(a), _ptr(b), len(b)):
        raise ValueError("port multiply out of band")
    return r


def port_sqr(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    r = np.zeros(2 * len(a), dtype=np.uint64)
    if not port().sbo_ntt_sqr(_ptr(r), _ptr(a), len(a)):
        raise ValueError("port square out of band")
    return r


def school_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    r = np.zeros(len(a) + len(b), dtype=np.uint64)
    port().sbo_mul_school(_ptr(r), _ptr(a), len(a), _ptr(b), len(b))
    return r


def mulmid(a: np.ndarray, b: np.ndarray, method: str = "school") -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    r = np.zeros(len(a) - len(b) + 3, dtype=np.uint64)
    if method == "school":
        port().sbo_mulmid(_ptr(r), _ptr(a), len(a), _ptr(b), len(b))
    else:
        if not port().sbo_ntt_mulmid(_ptr(r), _ptr(a), len(a), _ptr(b), len(b)):
            raise ValueError("port mulmid out of band")
    return r


def port_divrem(n: np.ndarray, d: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    n = np.ascontiguousarray(n, dtype=np.uint64)
    d = np.ascontiguousarray(d, dtype=np.uint64)
    q = np.zeros(len(n) - len(d) + 1, dtype=np.uint64)
    r = np.zeros(len(d), dtype=np.uint64)
    port().sbo_divrem(_ptr(q), _ptr(r), _ptr(n), len(n), _ptr(d), len(d))
    return q, r


def port_recip(d: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(d, dtype=np.uint64)
    i = np.zeros(len(d), dtype=np.uint64)
    port().sbo_recip(_ptr(i), _ptr(d), len(d))
    return i


def mod_u64(a: np.ndarray, q: int) -> int:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return int(port().sbo_mod_u64(_ptr(a), len(a), q))


# ---------------------------------------------------------------- ref ops --
def ref_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    r = np.zeros(len(a) + len(b) + 2, dtype=np.uint64)
    if not ref().sbref_nt_mul(_ptr(r), _ptr(a), len(a), _ptr(b), len(b)):
        raise ValueError("reference nt_mul returned 0")
    return r[: len(a) + len(b)]


def ref_sqr(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    r = np.zeros(2 * len(a) + 2, dtype=np.uint64)
    if not ref().sbref_nt_sqr(_ptr(r), _ptr(a), len(a)):
        raise ValueError("reference nt_sqr returned 0")
    return r[: 2 * len(a)]


def ref_simd_mpn_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    r = np.zeros(len(a) + len(b), dtype=np.uint64)
    ref().sbref_simd_mpn_mul(_ptr(r), _ptr(a), len(a), _ptr(b), len(b))
    return r


def ref_divrem(n: np.ndarray, d: np.ndarray, dc: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """Q, R of the reference divrem_u64_dc (include/dc_div.h:154), full-length
    (Q: nn-dn+1 limbs, R: dn limbs, zero-padded).  The reference requires a
    divisor of more than 416 bits (include/divrem.h:216); smaller ones raise."""
    n = np.ascontiguousarray(n, dtype=np.uint64)
    d = np.ascontiguousarray(d, dtype=np.uint64)
    if to_int(d).bit_length() <= 416:
        raise ValueError("reference divrem needs a divisor of more than 416 bits")
    q = np.zeros(len(n) - len(d) + 2, dtype=np.uint64)
    r = np.zeros(len(d) + 1, dtype=np.uint64)
    qn = C.c_uint64(0)
    rn = C.c_uint64(0)
    fn = ref().sbref_divrem_u64_dc if dc else ref().sbref_divrem_u64
    fn(_ptr(q), _ptr(r), _ptr(n), len(n), _ptr(d), len(d), C.byref(qn), C.byref(rn))
    return q[: len(n) - len(d) + 1], r[: len(d)]


# ---------------------------------------------------- threaded CPU runs --
class Job(C.Structure):
    _fields_ = [("kind", C.c_int32), ("pad", C.c_int32), ("r", C.c_void_p), ("r2", C.c_void_p),
                ("a", C.c_void_p), ("b", C.c_void_p), ("an", C.c_uint64), ("bn", C.c_uint64)]


# ------------------------------------------------ u52 redundant digits --
M52 = (1 << 52) - 1


def _digits_of(v: int, n: int, out: list) -> None:
    """Appends the n low radix-2^52 digits of v >= 0 (divide and conquer, so
    long numbers cost O(bits log n) instead of O(bits n))."""
    if n <= 64:
        for i in range(n):
            out.append((v >> (52 * i)) & M52)
        return
    h = n // 2
    _digits_of(v & ((1 << (52 * h)) - 1), h, out)
    _digits_of(v >> (52 * h), n - h, out)


def _value_of(d: list, lo: int, hi: int) -> int:
    """sum_{lo <= i < hi} d[i] 2^(52 (i - lo)) for any integer lanes."""
    if hi - lo <= 64:
        v = 0
        for i in range(hi - 1, lo - 1, -1):
            v = (v << 52) + d[i]
        return v
    m = (lo + hi) // 2
    return _value_of(d, lo, m) + (_value_of(d, m, hi) << (52 * (m - lo)))


def u52_from_u64(a: np.ndarray) -> np.ndarray:
    """Canonical radix-2^52 digits of {a}: ceil(bitlength / 52) of them (the
    reference's u52_from_u64, include/u64cvt.h:42-58), by Python integers."""
    v = to_int(np.ascontiguousarray(a, dtype=np.uint64))
    n52 = (v.bit_length() + 51) // 52
    out: list = []
    _digits_of(v, n52, out)
    return np.array(out, dtype=np.uint64)


def u64_from_u52(d: np.ndarray, out_limbs: int, signed: bool = False) -> np.ndarray:
    """sum_i d[i] 2^(52 i) mod 2^(64 out_limbs) for redundant digits: unsigned
    64-bit lanes, or two's-complement signed lanes (the reference's
    u64_from_u52_canon / _canonneg, include/canon.h:303-324)."""
    lanes = np.asarray(d, dtype=np.uint64)
    vals = (lanes.view(np.int64) if signed else lanes).tolist()
    v = _value_of(vals, 0, len(vals)) & ((1 << (64 * out_limbs)) - 1)
    return from_int(v, out_limbs) if out_limbs else np.zeros(0, dtype=np.uint64)


def ref_u52_from_u64(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    out = np.zeros(len(a) * 64 // 52 + 2, dtype=np.uint64)
    n = ref().sbref_u52_from_u64(_ptr(out), _ptr(a) if len(a) else _ptr(out), len(a))
    return out[:n].copy()


def ref_u64_from_u52(d: np.ndarray, out_limbs: int, signed: bool = False) -> np.ndarray:
    d = np.ascontiguousarray(d, dtype=np.uint64)
    r = np.zeros(max(out_limbs, 1), dtype=np.uint64)
    ref().sbref_u64_from_u52(_ptr(r), out_limbs, _ptr(d) if len(d) else _ptr(r), len(d), int(signed))
    return r[:out_limbs]


def run_jobs(jobs: list[tuple], threads: int, which: str) -> int:
    """jobs: (kind, r, r2, a, b) numpy arrays (kind 0 mul, 1 sqr, 2 divrem).
    Runs them on `threads` pthreads in the chosen library; returns failures."""
    arr = (Job * len(jobs))()
    keep = []
    for i, (kind, r, r2, a, b) in enumerate(jobs):
        arr[i].kind = kind
        arr[i].r = r.ctypes.data
        arr[i].r2 = r2.ctypes.data if r2 is not None else None
        arr[i].a = a.ctypes.data
        arr[i].b = (b if b is not None else a).ctypes.data
        arr[i].an = len(a)
        arr[i].bn = len(b) if b is not None else len(a)
        keep.append((r, r2, a, b))
    lib = ref() if which == "ref" else port()
    fn = lib.sbref_run_threads if which == "ref" else lib.sbo_run_threads
    return int(fn(C.cast(arr, C.c_void_p), len(jobs), threads))
