"""GPU tests of the host-operand, stream-ordered products (sbg_mul_host,
sbg_sqr_host): several products queued back to back on page-locked and on
pageable buffers, alternating the two staging slots and growing them, must
each equal the oracle's product once the context is synchronised."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import rand_limbs, spot_check

pytestmark = pytest.mark.gpu


def _pinned(n):
    import torch
    return torch.empty(n, dtype=torch.int64).pin_memory().numpy().view(np.uint64)


def test_queued_host_products_pinned(ctx):
    rng = np.random.default_rng(808)
    shapes = [(1000, 999), (5, 3), (70000, 65000), (4096, 4096), (300000, 1000), (17, 17)]
    jobs = []
    for an, bn in shapes:
        a, b = _pinned(an), _pinned(bn)
        a[:] = rand_limbs(an, rng)
        b[:] = rand_limbs(bn, rng)
        r = _pinned(an + bn)
        r[:] = 0
        ctx.mul_host(r, a, b)
        jobs.append((a, b, r))
    s = _pinned(2 * 5000)
    a5 = rand_limbs(5000, rng)
    sq = _pinned(5000)
    sq[:] = a5
    ctx.sqr_host(s, sq)
    ctx.sync()
    for a, b, r in jobs:
        assert np.array_equal(r, O.port_mul(a, b)), (len(a), len(b))
    assert np.array_equal(s, O.port_sqr(a5))


def test_queued_host_products_pageable_and_large(ctx):
    rng = np.random.default_rng(809)
    a = rand_limbs(1 << 21, rng)
    b = rand_limbs((1 << 21) - 3, rng)
    r1 = np.zeros(len(a) + len(b), dtype=np.uint64)
    r2 = np.zeros(2 * len(a), dtype=np.uint64)
    ctx.mul_host(r1, a, b)
    ctx.sqr_host(r2, a)
    ctx.sync()
    assert spot_check(a, b, r1)
    assert spot_check(a, a, r2)
    assert np.array_equal(r1[:64], O.port_mul(a[:64], b[:64])[:64])
