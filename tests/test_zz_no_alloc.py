"""The allocation-free multiply, sbg_mul_noalloc, against the oracle and the
context multiply.

Some callers cannot allocate device memory when they multiply: programs that
reserve all GPU memory up front, plug-ins inside a host that owns the device
allocator, latency-critical loops that cannot take cudaMalloc's implicit
synchronisation.  sbg_mul_noalloc serves them from static device scratch.
These tests call it through the C ABI on several shapes in a row (so a stale
scratch array from one call would show in the next), and require every
product to equal the oracle's (our C restatement of the reference's NTT
product, or the u128 schoolbook) and sbg_mul's bit for bit; a call on a
non-default stream; sbg_noalloc_status reporting a clean run; a fresh process
whose first library call is sbg_mul_noalloc (so its own per-device set-up is
what runs); and the rejection of products beyond SBG_NOALLOC_MAX_LIMBS.

The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def _lib():
    import simd_bigint_b200 as sbg
    L = C.CDLL(str(sbg.lib_path()))
    L.sbg_mul_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                  C.c_void_p]
    L.sbg_mul_noalloc.restype = C.c_int
    L.sbg_noalloc_max_limbs.argtypes = []
    L.sbg_noalloc_max_limbs.restype = C.c_int64
    L.sbg_noalloc_status.argtypes = [C.c_void_p]
    L.sbg_noalloc_status.restype = C.c_int
    return L


def _want(a, b):
    return O.school_mul(a, b) if len(a) + len(b) <= 256 else O.port_mul(a, b)


SHAPES = [(1, 1, "rand"), (3, 5, "rand"), (100, 27, "rand"), (1000, 1000, "rand"),
          (2000, 2097, "rand"), (2048, 2049, "ones"), (4096, 1, "ones"), (7, 4090, "sparse")]


def test_noalloc_matches_oracle_and_context_multiply_on_calls_in_a_row(ctx):
    import torch
    L = _lib()
    assert L.sbg_noalloc_max_limbs() == 4097
    rng = np.random.default_rng(2024)
    for an, bn, pat in SHAPES:
        a = O.pattern(an, pat, rng)
        b = O.pattern(bn, pat, rng)
        ta = torch.from_numpy(a.view(np.int64)).cuda()
        tb = torch.from_numpy(b.view(np.int64)).cuda()
        r_na = torch.full((an + bn,), -1, dtype=torch.int64, device="cuda")
        r_ctx = torch.empty(an + bn, dtype=torch.int64, device="cuda")
        st = L.sbg_mul_noalloc(r_na.data_ptr(), ta.data_ptr(), an, tb.data_ptr(), bn, None)
        assert st == 0, st
        assert L.sbg_noalloc_status(None) == 0
        ctx.mul(r_ctx, ta, tb)
        ctx.sync()
        got = r_na.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, _want(a, b)), (an, bn, pat)
        assert np.array_equal(got, r_ctx.cpu().numpy().view(np.uint64)), (an, bn, pat)


def test_noalloc_on_a_side_stream(ctx):
    import torch
    L = _lib()
    rng = np.random.default_rng(2025)
    s = torch.cuda.Stream()
    outs = []
    with torch.cuda.stream(s):
        for an, bn in ((1500, 1501), (33, 4000)):
            a, b = O.pattern(an, "rand", rng), O.pattern(bn, "rand", rng)
            ta = torch.from_numpy(a.view(np.int64)).to("cuda", non_blocking=False)
            tb = torch.from_numpy(b.view(np.int64)).to("cuda", non_blocking=False)
            r = torch.zeros(an + bn, dtype=torch.int64, device="cuda")
            assert L.sbg_mul_noalloc(r.data_ptr(), ta.data_ptr(), an, tb.data_ptr(), bn,
                                     C.c_void_p(s.cuda_stream)) == 0
            # calls on one stream are ordered; the status waits for that stream
            assert L.sbg_noalloc_status(C.c_void_p(s.cuda_stream)) == 0
            outs.append((a, b, r.cpu().numpy().view(np.uint64).copy()))
    for a, b, got in outs:
        assert np.array_equal(got, _want(a, b))


def test_noalloc_rejects_beyond_its_scratch(ctx):
    import torch
    L = _lib()
    a = torch.zeros(4000, dtype=torch.int64, device="cuda")
    r = torch.zeros(8000, dtype=torch.int64, device="cuda")
    assert L.sbg_mul_noalloc(r.data_ptr(), a.data_ptr(), 4000, a.data_ptr(), 98, None) == 2
    assert L.sbg_mul_noalloc(r.data_ptr(), a.data_ptr(), 0, a.data_ptr(), 5, None) == 1


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import simd_bigint_b200 as sbg
from oracle import oracle as O
L = C.CDLL(str(sbg.lib_path()))
L.sbg_mul_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
L.sbg_noalloc_status.argtypes = [C.c_void_p]
rng = np.random.default_rng(7)
for an, bn in ((9, 11), (2047, 2050)):
    a = rng.integers(0, 2**64, an, dtype=np.uint64)
    b = rng.integers(0, 2**64, bn, dtype=np.uint64)
    ta, tb = torch.from_numpy(a.view(np.int64)).cuda(), torch.from_numpy(b.view(np.int64)).cuda()
    r = torch.zeros(an + bn, dtype=torch.int64, device="cuda")
    assert L.sbg_mul_noalloc(r.data_ptr(), ta.data_ptr(), an, tb.data_ptr(), bn, None) == 0
    assert L.sbg_noalloc_status(None) == 0
    assert np.array_equal(r.cpu().numpy().view(np.uint64), O.port_mul(a, b)), (an, bn)
print("fresh ok")
"""


def test_noalloc_first_call_in_a_fresh_process():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = subprocess.run([sys.executable, "-c", _FRESH, str(ROOT)], capture_output=True, text=True,
                         timeout=300, env={**os.environ, "PYTHONPATH": str(ROOT)})
    assert out.returncode == 0 and "fresh ok" in out.stdout, out.stdout + out.stderr
