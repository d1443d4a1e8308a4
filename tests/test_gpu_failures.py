"""Failure paths, exercised without faulting the GPU.

Every failure here is made on purpose in a form that cannot fault, trap or
hang the device:
  * a bounded device-side wait that runs out: the carry scan's first block
    withholds its look-back flag (test hook SBG_INJECT_WITHHOLD, which also
    shortens the wait), the next block's wait expires, the kernel records
    the error bit and returns, and the host reads SBG_ETIMEOUT;
  * corrupted data between the transforms and the CRT: the top
    coefficient's residue altered (the product spills: SBG_ESPILL), or a
    middle one (the device cannot see it; the host's modular spot check and
    the oracle do);
  * a host-side fake of a failing cudaMalloc (SBG_EALLOC);
  * a serving request cancelled while still queued (SBG_ECANCELED).
After each injected failure the hooks are turned off and the same context
must compute a correct product again: the error is reported, not sticky, and
the context stays usable.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import rand_limbs, spot_check

pytestmark = pytest.mark.gpu


def _sbg():
    import simd_bigint_b200 as sbg
    return sbg


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def _mul_status(ctx, a, b):
    """Queue one product, wait; returns (status of sbg_ctx_sync, product)."""
    import torch
    sbg = _sbg()
    ta, tb = _dev(a), _dev(b)
    tr = torch.zeros(len(a) + len(b), dtype=torch.int64, device="cuda")
    ctx.mul(tr, ta, tb)
    st = sbg.lib().sbg_ctx_sync(ctx.handle)
    return st, tr.cpu().numpy().view(np.uint64)


@pytest.fixture
def inject():
    L = _sbg().lib()

    def set_mask(m):
        assert L.sbg_debug_inject(m) == 0

    yield set_mask
    assert L.sbg_debug_inject(0) == 0
    L.sbg_debug_fail_allocs(0)


@pytest.mark.parametrize("an,bn", [(3000, 2500), (20000, 20000), (1 << 20, 1 << 19)])
def test_lookback_wait_runs_out_and_is_reported(ctx, inject, an, bn):
    sbg = _sbg()
    rng = np.random.default_rng(an)
    a, b = rand_limbs(an, rng), rand_limbs(bn, rng)
    inject(sbg.INJECT_WITHHOLD)
    st, _ = _mul_status(ctx, a, b)
    assert st == 5, sbg.STATUS.get(st, st)               # SBG_ETIMEOUT
    inject(0)
    st, r = _mul_status(ctx, a, b)
    assert st == 0
    assert np.array_equal(r, O.port_mul(a, b))


def test_corrupted_top_residue_is_caught_by_the_spill_check(ctx, inject):
    sbg = _sbg()
    rng = np.random.default_rng(11)
    a, b = rand_limbs(70000, rng), rand_limbs(65000, rng)
    inject(sbg.INJECT_TOP)
    st, _ = _mul_status(ctx, a, b)
    assert st == 6, sbg.STATUS.get(st, st)               # SBG_ESPILL
    inject(0)
    st, r = _mul_status(ctx, a, b)
    assert st == 0 and np.array_equal(r, O.port_mul(a, b))


def test_corrupted_middle_residue_is_caught_by_the_modular_check(ctx, inject):
    sbg = _sbg()
    rng = np.random.default_rng(12)
    a, b = rand_limbs(50000, rng), rand_limbs(40000, rng)
    inject(sbg.INJECT_MID)
    st, bad = _mul_status(ctx, a, b)
    inject(0)
    # no device check can see a wrong coefficient that does not spill; the
    # host's checks do
    assert not np.array_equal(bad, O.port_mul(a, b))
    assert not spot_check(a, b, bad)
    st, r = _mul_status(ctx, a, b)
    assert st == 0 and spot_check(a, b, r)


def test_noalloc_reports_an_expired_wait(inject):
    import ctypes as C

    import torch
    sbg = _sbg()
    L = sbg.lib()
    rng = np.random.default_rng(13)
    a, b = rand_limbs(2100, rng), rand_limbs(1997, rng)     # 4097 limbs: two carry-scan blocks
    ta, tb = _dev(a), _dev(b)
    r = torch.zeros(4097, dtype=torch.int64, device="cuda")
    assert L.sbg_noalloc_status(None) == 0
    inject(sbg.INJECT_WITHHOLD)
    assert L.sbg_mul_noalloc(C.c_void_p(r.data_ptr()), C.c_void_p(ta.data_ptr()), 2100,
                             C.c_void_p(tb.data_ptr()), 1997, None) == 0
    assert L.sbg_noalloc_status(None) == 5                  # SBG_ETIMEOUT, then cleared
    inject(0)
    assert L.sbg_noalloc_status(None) == 0
    assert L.sbg_mul_noalloc(C.c_void_p(r.data_ptr()), C.c_void_p(ta.data_ptr()), 2100,
                             C.c_void_p(tb.data_ptr()), 1997, None) == 0
    assert L.sbg_noalloc_status(None) == 0
    assert np.array_equal(r.cpu().numpy().view(np.uint64), O.port_mul(a, b))


def test_allocation_failure_is_reported_and_recoverable(inject):
    sbg = _sbg()
    L = sbg.lib()
    rng = np.random.default_rng(14)
    a, b = rand_limbs(300000, rng), rand_limbs(200000, rng)
    c = sbg.Context(0)
    try:
        L.sbg_debug_fail_allocs(1)           # the workspace (or a plan table) cannot be had
        with pytest.raises(sbg.SbgError) as e:
            _mul_status(c, a, b)
        assert e.value.status == 3           # SBG_EALLOC
        L.sbg_debug_fail_allocs(0)
        st, r = _mul_status(c, a, b)
        assert st == 0 and np.array_equal(r, O.port_mul(a, b))
    finally:
        c.close()


def test_serving_request_cancelled_while_queued(ctx):
    import time

    import torch
    sbg = _sbg()
    rng = np.random.default_rng(15)
    pool = torch.from_numpy(rand_limbs(1 << 21, rng).view(np.int64)).cuda()
    base = pool.data_ptr()
    srv = sbg.Server(ctx, arena_bytes=1 << 30, slots=1, max_batch=2, recip_workers=1)
    try:
        n = 64
        reqs = [(sbg.REQ_MUL, base, 1 << 18, base + 8 * (1 << 19), 1 << 18) for _ in range(n)]
        tickets = srv.submit_many(reqs)
        cancelled = {t for t in tickets[n // 2:] if srv.cancel(t)}
        assert cancelled, "the tail of a 64-request burst on one slot should still be queued"
        assert not srv.cancel(10 ** 9)       # unknown ticket
        seen = {}
        t0 = time.time()
        while len(seen) < n and time.time() - t0 < 120:
            for tk, st, rp, rn, _ in srv.poll(wait_ms=50):
                assert tk not in seen
                seen[tk] = (st, rp, rn)
        assert len(seen) == n
        a = pool[: 1 << 18].cpu().numpy().view(np.uint64)
        b = pool[1 << 19: (1 << 19) + (1 << 18)].cpu().numpy().view(np.uint64)
        want = None
        for tk in tickets:
            st, rp, rn = seen[tk]
            if tk in cancelled:
                assert st == 9 and rp == 0       # SBG_ECANCELED, no result
                continue
            assert st == 0
            got = srv.result(rp, rn).cpu().numpy().view(np.uint64)
            if want is None:
                want = O.port_mul(a, b)
            assert np.array_equal(got, want)
            srv.release(tk)
    finally:
        srv.close()
