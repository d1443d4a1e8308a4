"""GPU parity of the 3 * 2^k transform lengths.

A product whose coefficient count lies in (2^(k+1), 3 * 2^k] (k = 16 .. 23)
runs at length 3 * 2^k instead of 2^(k+2): a radix-3 level across column
thirds (clusters of 3 or 6 CTAs), mixed-radix row order in the four-step
twiddle, and the scale 1/L with L = 3 * 2^k.  Every result must equal the
oracle's product bit for bit (C restatement of the reference algorithm up
to 2^20 limbs; beyond, the all-0xFF closed form and the random-prime spot
check), through sbg_mul, sbg_sqr, sbg_mulmid and the batch engine."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import ones_square, rand_limbs, spot_check

pytestmark = pytest.mark.gpu
ALL3 = 0x00FF0000          # every 3 * 2^k class, k = 16 .. 23


@pytest.fixture
def ctx3(ctx):
    """The session context with every 3 * 2^k length enabled."""
    old = ctx.len3_mask
    ctx.set_len3_mask(ALL3)
    yield ctx
    ctx.set_len3_mask(old)


def _mul(ctx, a, b):
    import torch
    ta = torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()
    tb = torch.from_numpy(np.ascontiguousarray(b).view(np.int64)).cuda()
    tr = torch.empty(len(a) + len(b), dtype=torch.int64, device="cuda")
    ctx.mul(tr, ta, tb)
    ctx.sync()
    return tr.cpu().numpy().view(np.uint64)


def _sqr(ctx, a):
    import torch
    ta = torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()
    tr = torch.empty(2 * len(a), dtype=torch.int64, device="cuda")
    ctx.sqr(tr, ta)
    ctx.sync()
    return tr.cpu().numpy().view(np.uint64)


def _three_shapes():
    # (an, bn): an + bn - 1 just above 2^(k+1), in the middle, and at 3 * 2^k
    out = []
    for k in range(16, 20):
        lo, hi = (1 << (k + 1)) + 1, 3 << k
        out += [((lo + 1) // 2 + 1, (lo + 1) // 2), (hi - (1 << k) + 1, 1 << k), (hi // 2 + 1, hi // 2)]
    return out


@pytest.mark.parametrize("an,bn", _three_shapes())
def test_three_lengths_vs_port(ctx3, an, bn):
    rng = np.random.default_rng(an * 7 + bn)
    a = rand_limbs(an, rng)
    b = rand_limbs(bn, rng)
    assert np.array_equal(_mul(ctx3, a, b), O.port_mul(a, b)), (an, bn)


@pytest.mark.parametrize("n", [70000, (3 << 17) // 2, 300001, (3 << 19) // 2])
def test_three_lengths_squares(ctx3, n):
    rng = np.random.default_rng(n)
    a = rand_limbs(n, rng)
    assert np.array_equal(_sqr(ctx3, a), O.port_sqr(a)), n
    ones = O.pattern(n, "ones")
    assert np.array_equal(_sqr(ctx3, ones), ones_square(n))


@pytest.mark.parametrize("n", [(3 << 20) // 2, (3 << 21) // 2 - 5, (3 << 22) // 2, (3 << 23) // 2])
def test_three_lengths_large_closed_form(ctx3, n):
    """m = 9, 10 (clusters of 3, column pairs) and m = 11 (clusters of 6)."""
    ones = O.pattern(n, "ones")
    assert np.array_equal(_sqr(ctx3, ones), ones_square(n))


def test_three_lengths_large_random_and_unbalanced(ctx3):
    rng = np.random.default_rng(33)
    for an, bn in [((1 << 24), (1 << 20)), ((1 << 23) + 12345, (1 << 22) + 999), (6000000, 3000000)]:
        a = rand_limbs(an, rng)
        b = rand_limbs(bn, rng)
        r = _mul(ctx3, a, b)
        assert spot_check(a, b, r), (an, bn)
        assert np.array_equal(_mul(ctx3, b, a), r)


def test_three_lengths_mulmid_and_batch(ctx3):
    import torch

    import simd_bigint_b200 as sbg
    ctx = ctx3
    rng = np.random.default_rng(34)
    # mulmid at length 3 * 2^17 (an in (2^18, 3 * 2^17])
    a = rand_limbs(300000, rng)
    b = rand_limbs(120000, rng)
    ta = torch.from_numpy(a.view(np.int64)).cuda()
    tb = torch.from_numpy(b.view(np.int64)).cuda()
    tr = torch.empty(len(a) - len(b) + 3, dtype=torch.int64, device="cuda")
    ctx.mulmid(tr, ta, tb)
    ctx.sync()
    assert np.array_equal(tr.cpu().numpy().view(np.uint64), O.mulmid(a, b, "ntt"))
    # a batch mixing power-of-two and 3 * 2^k classes
    shapes = [(100000, 90000), (70000, 70000), (200000, 100000), (5000, 300), (131072, 131072)]
    keep, jobs = [], []
    for i, (an, bn) in enumerate(shapes):
        x = rand_limbs(an, rng)
        y = x if i == 1 else rand_limbs(bn, rng)
        tx = torch.from_numpy(x.view(np.int64)).cuda()
        ty = torch.from_numpy(y.view(np.int64)).cuda()
        kind = sbg.JOB_SQR if i == 1 else sbg.JOB_MUL
        out = torch.full((an + bn,), -1, dtype=torch.int64, device="cuda")
        jobs.append((kind, out.data_ptr(), tx.data_ptr(), ty.data_ptr(), an, bn))
        keep.append((x, y, tx, ty, out))
    bt = sbg.Batch(ctx, jobs)
    bt.capture()
    bt.run()
    ctx.sync()
    for x, y, _, _, out in keep:
        assert np.array_equal(out.cpu().numpy().view(np.uint64), O.port_mul(x, y)), (len(x), len(y))
    bt.close()


def test_default_lengths_and_autotune(ctx):
    """The default mask enables 3 * 2^k for k = 16..19 and 21..23 (measured
    on B200); the drop-in's default context multiplies 2^24 x 2^20 at 3 * 2^23."""
    import simd_bigint_b200 as sbg
    assert ctx.len3_mask == 0x00EF0000
    rng = np.random.default_rng(35)
    a = rand_limbs(1 << 24, rng)
    b = rand_limbs(1 << 20, rng)
    assert spot_check(a, b, sbg.mul(a, b))
    c2 = sbg.Context(0)
    r = c2.autotune()
    assert set(r["times"]) == set(range(16, 24)) and all(x > 0 and y > 0 for x, y in r["times"].values())
    assert r["len3_mask"] & ~ALL3 == 0
    c2.close()
