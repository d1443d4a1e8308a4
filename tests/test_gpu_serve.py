"""GPU tests of the serving loop (sbg_server_*).

Continuous batching must not change any result: every request submitted
into a busy server -- arriving while earlier batches run, mixed kinds and
sizes -- must return exactly what the same request computes alone through
sbg_mul / sbg_sqr / sbg_recip.  Admission by HBM footprint must reject a
request that can never fit the arena, and results must stay readable until
released.
"""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(rng, count, hi):
    import simd_bigint_b200 as sbg
    out = []
    for i in range(count):
        an = int(np.exp(rng.uniform(np.log(32), np.log(hi))))
        kind = [sbg.REQ_MUL, sbg.REQ_SQR, sbg.REQ_RECIP][i % 3]
        bn = an if (kind != sbg.REQ_MUL or rng.uniform() < 0.7) else max(1, int(an / np.exp(rng.uniform(0, np.log(16)))))
        out.append((kind, an, bn))
    return out


def test_results_alone_equal_results_in_the_mix(ctx):
    import torch

    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(501)
    reqs = _requests(rng, 150, 1 << 17)
    ops = []
    for kind, an, bn in reqs:
        a = rng.integers(0, 2**64, an, dtype=np.uint64)
        if kind == sbg.REQ_RECIP:
            a[-1] |= np.uint64(1 << 63)
        b = rng.integers(0, 2**64, bn, dtype=np.uint64)
        ta = torch.from_numpy(a.view(np.int64)).cuda()
        tb = torch.from_numpy(b.view(np.int64)).cuda()
        ops.append((kind, an, bn, ta, tb))
    srv = sbg.Server(ctx, arena_bytes=2 << 30, slots=4, max_batch=32)
    tickets = {}
    got = {}
    lock = threading.Lock()

    def submitter():
        for i, (kind, an, bn, ta, tb) in enumerate(ops):
            t = srv.submit(kind, ta.data_ptr(), an, tb.data_ptr(), bn)
            with lock:
                tickets[t] = i
            if i % 10 == 0:
                time.sleep(0.002)      # later requests arrive while batches run

    th = threading.Thread(target=submitter)
    th.start()
    deadline = time.time() + 120
    while len(got) < len(ops) and time.time() < deadline:
        for ticket, status, rp, rn, lat in srv.poll(wait_ms=50):
            assert status == 0
            assert lat >= 0
            with lock:
                i = tickets.get(ticket)
            while i is None:                   # submit() returned after completion
                time.sleep(0.001)
                with lock:
                    i = tickets.get(ticket)
            got[i] = srv.result(rp, rn).cpu().numpy().view(np.uint64)
            srv.release(ticket)
    th.join()
    assert len(got) == len(ops)
    st = srv.stats()
    assert st["completed"] == len(ops) and st["pending"] == 0
    assert st["batches"] < len(ops)             # requests were batched together
    srv.close()
    for i, (kind, an, bn, ta, tb) in enumerate(ops):
        if kind == sbg.REQ_MUL:
            r = torch.empty(an + bn, dtype=torch.int64, device="cuda")
            ctx.mul(r, ta, tb)
        elif kind == sbg.REQ_SQR:
            r = torch.empty(2 * an, dtype=torch.int64, device="cuda")
            ctx.sqr(r, ta)
        else:
            r = torch.empty(an, dtype=torch.int64, device="cuda")
            ctx.recip(r, ta)
        ctx.sync()
        assert np.array_equal(got[i], r.cpu().numpy().view(np.uint64)), (kind, an, bn)


def test_admission_rejects_what_cannot_fit(ctx):
    import torch

    import simd_bigint_b200 as sbg
    srv = sbg.Server(ctx, arena_bytes=64 << 20, slots=2, max_batch=8)
    a = torch.zeros(1 << 20, dtype=torch.int64, device="cuda")
    st, _ = srv.try_submit(sbg.REQ_MUL, a.data_ptr(), 1 << 20, a.data_ptr(), 1 << 20)
    assert st == 7                              # SBG_EADMIT: 84 MB of workspace > 64 MB arena
    a[-1] = 1
    ok, t = srv.try_submit(sbg.REQ_SQR, a.data_ptr(), 1000)
    assert ok == 0
    done = []
    deadline = time.time() + 30
    while not done and time.time() < deadline:
        done = srv.poll(wait_ms=50)
    assert done and done[0][0] == t and done[0][1] == 0
    srv.release(t)
    srv.close()


def test_burst_submission_matches_single_requests(ctx):
    import torch

    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(502)
    reqs = _requests(rng, 40, 1 << 15)
    ops, keep = [], []
    for kind, an, bn in reqs:
        a = rng.integers(0, 2**64, an, dtype=np.uint64)
        if kind == sbg.REQ_RECIP:
            a[-1] |= np.uint64(1 << 63)
        b = rng.integers(0, 2**64, bn, dtype=np.uint64)
        ta = torch.from_numpy(a.view(np.int64)).cuda()
        tb = torch.from_numpy(b.view(np.int64)).cuda()
        keep.append((kind, an, bn, ta, tb))
        ops.append((kind, ta.data_ptr(), an, tb.data_ptr(), bn))
    srv = sbg.Server(ctx, arena_bytes=1 << 30, slots=3, max_batch=16, recip_workers=3)
    tickets = srv.submit_many(ops)
    assert len(tickets) == len(ops) and tickets == sorted(tickets)
    where = {t: i for i, t in enumerate(tickets)}
    got = {}
    deadline = time.time() + 60
    while len(got) < len(ops) and time.time() < deadline:
        for ticket, status, rp, rn, lat in srv.poll(wait_ms=50):
            assert status == 0
            got[where[ticket]] = srv.result(rp, rn).cpu().numpy().view(np.uint64)
            srv.release(ticket)
    assert len(got) == len(ops)
    assert srv.launches() > 0
    srv.close()
    for i, (kind, an, bn, ta, tb) in enumerate(keep):
        n = an + bn if kind == sbg.REQ_MUL else (2 * an if kind == sbg.REQ_SQR else an)
        r = torch.empty(n, dtype=torch.int64, device="cuda")
        if kind == sbg.REQ_MUL:
            ctx.mul(r, ta, tb)
        elif kind == sbg.REQ_SQR:
            ctx.sqr(r, ta)
        else:
            ctx.recip(r, ta)
        ctx.sync()
        assert np.array_equal(got[i], r.cpu().numpy().view(np.uint64)), (kind, an, bn)
