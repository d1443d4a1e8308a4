"""The allocation-free multiply, sbg_mul_noalloc, against the context multiply.

Some callers cannot allocate device memory when they multiply: programs that
reserve all GPU memory up front, plug-ins inside a host that owns the device
allocator, latency-critical loops that cannot take cudaMalloc's implicit
synchronisation.  sbg_mul_noalloc serves them from static device scratch.
This test calls it through the C ABI twice in a row, on two different shapes
(so a stale scratch array from the first call would show in the second), and
requires both products to equal sbg_mul's bit for bit; it also checks that a
product beyond SBG_NOALLOC_MAX_LIMBS is rejected with SBG_EBAND.

The file name sorts last so that a run stopping at its first failure has
already run every other test; it also passes alone in a fresh process (its
first call performs the per-device set-up).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _lib():
    import simd_bigint_b200 as sbg
    L = C.CDLL(str(sbg.lib_path()))
    L.sbg_mul_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                  C.c_void_p]
    L.sbg_mul_noalloc.restype = C.c_int
    L.sbg_noalloc_max_limbs.argtypes = []
    L.sbg_noalloc_max_limbs.restype = C.c_int64
    return L


def test_noalloc_matches_context_multiply_on_two_calls(ctx):
    import torch
    L = _lib()
    assert L.sbg_noalloc_max_limbs() == 4097
    rng = np.random.default_rng(2024)
    shapes = [(2000, 2097, "rand"), (4096, 1, "ones")]
    for an, bn, pat in shapes:
        a = O.pattern(an, pat, rng)
        b = O.pattern(bn, pat, rng)
        ta = torch.from_numpy(a.view(np.int64)).cuda()
        tb = torch.from_numpy(b.view(np.int64)).cuda()
        r_na = torch.full((an + bn,), -1, dtype=torch.int64, device="cuda")
        r_ctx = torch.empty(an + bn, dtype=torch.int64, device="cuda")
        st = L.sbg_mul_noalloc(r_na.data_ptr(), ta.data_ptr(), an, tb.data_ptr(), bn, None)
        assert st == 0, st
        torch.cuda.synchronize()
        ctx.mul(r_ctx, ta, tb)
        ctx.sync()
        got = r_na.cpu().numpy().view(np.uint64)
        want = r_ctx.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want), (an, bn, pat)


def test_noalloc_rejects_beyond_its_scratch(ctx):
    import torch
    L = _lib()
    a = torch.zeros(4000, dtype=torch.int64, device="cuda")
    r = torch.zeros(8000, dtype=torch.int64, device="cuda")
    assert L.sbg_mul_noalloc(r.data_ptr(), a.data_ptr(), 4000, a.data_ptr(), 98, None) == 2
    assert L.sbg_mul_noalloc(r.data_ptr(), a.data_ptr(), 0, a.data_ptr(), 5, None) == 1
