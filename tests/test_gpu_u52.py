"""GPU tests of the u52 redundant-digit boundary against the reference's own
conversions (u52_from_u64, include/u64cvt.h:42; u64_from_u52_canon /
_canonneg, include/canon.h:303-324, called through oracle/_ref) where the
reference runs on this host, and against Python integers (oracle.py's
restatement, itself pinned to the reference by the CPU suite) otherwise.
Every comparison is bit-exact."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint64).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _want_digits(a):
    return O.ref_u52_from_u64(a) if O.ref_available() else O.u52_from_u64(a)


def _want_limbs(d, rn, signed):
    return O.ref_u64_from_u52(d, rn, signed) if O.ref_available() else O.u64_from_u52(d, rn, signed)


def test_decode_matches_reference(ctx):
    import torch
    rng = np.random.default_rng(501)
    for n in (1, 2, 3, 12, 13, 64, 65, 1000, 4096, 100001):
        for pat in ("rand", "ones", "sparse"):
            a = O.pattern(n, pat, rng)
            want = _want_digits(a)
            n52 = (64 * n + 51) // 52
            d = torch.full((n52,), -1, dtype=torch.int64, device="cuda")
            ctx.u52_from_u64(d, _dev(a))
            ctx.sync()
            got = _host(d)
            assert np.array_equal(got[:len(want)], want), (n, pat)
            assert not got[len(want):].any()


@pytest.mark.parametrize("signed", [False, True])
def test_encode_redundant_digits_matches_reference(ctx, signed):
    import torch
    rng = np.random.default_rng(502 + signed)
    for n52 in (1, 2, 7, 8, 9, 64, 100, 1023, 1024, 1025, 5000, 200001):
        if signed:
            d = rng.integers(-(1 << 62), 1 << 62, n52).astype(np.int64).view(np.uint64)
        else:
            d = rng.integers(0, 2**64, n52, dtype=np.uint64)
        # the top digits canonical and positive, so the value is non-negative and fits
        d[-min(2, n52):] = rng.integers(0, 1 << 50, min(2, n52), dtype=np.uint64)
        rn = (52 * n52 + 63) // 64 + 1
        want = _want_limbs(d, rn, signed)
        r = torch.full((rn,), -1, dtype=torch.int64, device="cuda")
        ctx.u64_from_u52(r, _dev(d), signed)
        ctx.sync()
        assert np.array_equal(_host(r), want), (n52, signed)


def test_encode_carry_and_borrow_chains(ctx):
    """Long ripple chains: all-ones digits plus a carry at the bottom (the
    carry crosses every limb), and a borrow through zero digits."""
    import torch
    for n52 in (64, 3000, 70000):
        M = (1 << 52) - 1
        d = np.full(n52, M, dtype=np.uint64)
        d[0] = np.uint64(M + 1)             # redundant: carries all the way up
        rn = (52 * n52 + 63) // 64 + 1
        for signed in (False, True):
            want = O.u64_from_u52(d, rn, signed)
            r = torch.zeros(rn, dtype=torch.int64, device="cuda")
            ctx.u64_from_u52(r, _dev(d), signed)
            ctx.sync()
            assert np.array_equal(_host(r), want), (n52, signed)
        e = np.zeros(n52, dtype=np.uint64)
        e[-1] = np.uint64(1)
        e[0] = np.uint64((1 << 64) - 1)     # -1 as a signed lane: borrows through the zeros
        want = O.u64_from_u52(e, rn, True)
        r = torch.zeros(rn, dtype=torch.int64, device="cuda")
        ctx.u64_from_u52(r, _dev(e), True)
        ctx.sync()
        assert np.array_equal(_host(r), want), n52


def test_mul_u52_vs_python_integers(ctx):
    import torch
    rng = np.random.default_rng(503)
    for an52, bn52 in ((1, 1), (3, 5), (40, 40), (200, 7), (5000, 4999), (100000, 30000)):
        a = rng.integers(0, 1 << 52, an52, dtype=np.uint64)
        b = rng.integers(0, 1 << 52, bn52, dtype=np.uint64)
        if an52 > 2:
            a[:] = np.uint64((1 << 52) - 1) if an52 % 2 else a
        r = torch.full((an52 + bn52,), -1, dtype=torch.int64, device="cuda")
        ctx.mul_u52(r, _dev(a), _dev(b))
        ctx.sync()
        va = sum(int(x) << (52 * i) for i, x in enumerate(a.tolist()))
        vb = sum(int(x) << (52 * i) for i, x in enumerate(b.tolist()))
        p = va * vb
        want = np.array([(p >> (52 * i)) & ((1 << 52) - 1) for i in range(an52 + bn52)], dtype=np.uint64)
        assert np.array_equal(_host(r), want), (an52, bn52)
