"""GPU tests of the batch engine (sbg_batch_*, sbg_mul_batch).

Every product of a mixed batch -- all transform-length classes, mul, sqr and
mulmid, random and all-0xFF operands -- must equal the single-product path
(sbg_mul / sbg_sqr / sbg_mulmid, itself pinned to the reference) bit for bit,
when run plainly, when replayed from a captured CUDA graph, and in repeated
runs.  A sample is also checked against the oracle directly.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def _mixed_jobs(rng, shapes):
    import torch

    import simd_bigint_b200 as sbg
    jobs, keep = [], []
    for kind, an, bn, pat in shapes:
        a = O.pattern(an, pat, rng)
        b = a if kind == sbg.JOB_SQR else O.pattern(bn, pat, rng)
        ta, tb = _dev(a), _dev(b)
        nout = sbg.out_limbs(kind, an, bn)
        tr = torch.full((nout,), -1, dtype=torch.int64, device="cuda")
        jobs.append((kind, tr.data_ptr(), ta.data_ptr(), tb.data_ptr(), an, bn))
        keep.append((kind, a, b, ta, tb, tr))
    return jobs, keep


def _single(ctx, kind, ta, tb, nout):
    import torch

    import simd_bigint_b200 as sbg
    r = torch.empty(nout, dtype=torch.int64, device="cuda")
    if kind == sbg.JOB_MUL:
        ctx.mul(r, ta, tb)
    elif kind == sbg.JOB_SQR:
        ctx.sqr(r, ta)
    else:
        ctx.mulmid(r, ta, tb)
    ctx.sync()
    return r.cpu().numpy().view(np.uint64)


def _shapes(rng, n):
    import simd_bigint_b200 as sbg
    out = []
    for i in range(n):
        an = int(np.exp(rng.uniform(0, np.log(70000)))) + 1
        kind = [sbg.JOB_MUL, sbg.JOB_SQR, sbg.JOB_MULMID][i % 3]
        bn = max(1, int(an / np.exp(rng.uniform(0, np.log(8)))))
        pat = "ones" if i % 7 == 0 else "rand"
        out.append((kind, an, bn, pat))
    return out


def test_batch_matches_single_products(ctx):
    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(301)
    shapes = _shapes(rng, 90) + [(sbg.JOB_MUL, 1, 1, "rand"), (sbg.JOB_MUL, 16384, 16384, "rand"),
                                 (sbg.JOB_SQR, 65536, 65536, "ones"), (sbg.JOB_MUL, 200000, 3, "rand"),
                                 (sbg.JOB_MULMID, 5000, 4999, "ones")]
    jobs, keep = _mixed_jobs(rng, shapes)
    b = sbg.Batch(ctx, jobs)
    b.run()
    ctx.sync()
    for (kind, a, bb, ta, tb, tr), (_, _, _, _, an, bn) in zip(keep, jobs):
        got = tr.cpu().numpy().view(np.uint64)
        want = _single(ctx, kind, ta, tb, sbg.out_limbs(kind, an, bn))
        assert np.array_equal(got, want), (kind, an, bn)
    b.close()


@pytest.mark.parametrize("engine", [0, 1, 2], ids=["persistent", "per-class", "queue-per-cta"])
def test_batch_graph_replay_and_oracle(ctx, engine):
    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(302)
    shapes = _shapes(rng, 40)
    jobs, keep = _mixed_jobs(rng, shapes)
    b = sbg.Batch(ctx, jobs)
    b.set_engine(engine)
    b.capture()
    for rep in range(3):
        for _, _, _, _, _, tr in keep:
            tr.fill_(-1)
        b.run()
        ctx.sync()
        for (kind, a, bb, ta, tb, tr), (_, _, _, _, an, bn) in zip(keep, jobs):
            got = tr.cpu().numpy().view(np.uint64)
            if kind == sbg.JOB_MUL:
                want = O.port_mul(a, bb)
            elif kind == sbg.JOB_SQR:
                want = O.port_sqr(a)
            else:
                want = O.mulmid(a, bb, "ntt")
            assert np.array_equal(got, want), (rep, kind, an, bn)
    b.close()


def test_mul_batch_convenience_and_errors(ctx):
    import ctypes as C

    import torch

    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(303)
    jobs, keep = _mixed_jobs(rng, [(sbg.JOB_MUL, 100, 50, "rand"), (sbg.JOB_SQR, 3000, 3000, "rand")])
    arr = (sbg.Job * 2)()
    for i, (kind, r, a, b_, an, bn) in enumerate(jobs):
        arr[i].kind, arr[i].rp, arr[i].ap, arr[i].bp, arr[i].an, arr[i].bn = kind, r, a, b_, an, bn
    assert sbg.lib().sbg_mul_batch(ctx.handle, C.cast(arr, C.c_void_p), 2) == 0
    for kind, a, bb, ta, tb, tr in keep:
        want = O.port_sqr(a) if kind == sbg.JOB_SQR else O.port_mul(a, bb)
        assert np.array_equal(tr.cpu().numpy().view(np.uint64), want)
    # a mulmid with an < bn is rejected before anything runs
    bad = (sbg.Job * 1)()
    t = torch.zeros(10, dtype=torch.int64, device="cuda")
    bad[0].kind, bad[0].rp, bad[0].ap, bad[0].bp, bad[0].an, bad[0].bn = (
        sbg.JOB_MULMID, t.data_ptr(), t.data_ptr(), t.data_ptr(), 3, 5)
    assert sbg.lib().sbg_mul_batch(ctx.handle, C.cast(bad, C.c_void_p), 1) == 1


def test_batch_of_small_products_vs_schoolbook(ctx):
    """The schoolbook class of the batch engine (an + bn <= 128: one warp per
    product) beside transform classes, checked against the u128 schoolbook."""
    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(304)
    shapes = []
    for i in range(300):
        tot = int(rng.integers(2, 140))
        an = int(rng.integers(1, tot))
        kind = sbg.JOB_SQR if i % 5 == 0 else sbg.JOB_MUL
        shapes.append((kind, an, tot - an, "ones" if i % 4 == 0 else "rand"))
    shapes += [(sbg.JOB_MUL, 5000, 4000, "rand"), (sbg.JOB_MUL, 64, 64, "ones")]
    jobs, keep = _mixed_jobs(rng, shapes)
    b = sbg.Batch(ctx, jobs)
    b.capture()
    for _ in range(2):
        b.run()
        ctx.sync()
        for (kind, a, bb, ta, tb, tr), (_, _, _, _, an, bn) in zip(keep, jobs):
            got = tr.cpu().numpy().view(np.uint64)
            want = O.school_mul(a, a if kind == sbg.JOB_SQR else bb)
            assert np.array_equal(got, want), (kind, an, bn)
    b.close()


@pytest.mark.parametrize("wave_mb", [1, 48])
def test_persistent_queue_on_a_mixed_size_batch(ctx, wave_mb):
    """The persistent kernel (one launch, CTAs drawing (job, stage, tile)
    items from a device queue, per-job progress counters between stages) on
    a batch of the mixed-size configuration's shape distribution -- every
    class it runs, squarings, all-0xFF operands -- with small waves (many
    pipelined steps) and the default ones: every product equals the oracle's."""
    import simd_bigint_b200 as sbg
    from simd_bigint_b200.workloads import mixed_batch_shapes
    rng = np.random.default_rng(305)
    shapes = [(k, an, bn, "ones" if i % 9 == 0 else "rand")
              for i, (k, an, bn) in enumerate(mixed_batch_shapes(160, seed=99, lo=8, hi=70000))]
    shapes += [(sbg.JOB_MUL, 3, 5, "rand"), (sbg.JOB_SQR, 40, 40, "ones"), (sbg.JOB_MUL, 1000, 1, "rand"),
               (sbg.JOB_MUL, 300000, 200000, "rand")]       # the last one beyond the queue's classes
    jobs, keep = _mixed_jobs(rng, shapes)
    b = sbg.Batch(ctx, jobs)
    b.set_engine(0, wave_mb << 20)
    b.capture()
    for rep in range(2):
        for *_, tr in keep:
            tr.fill_(-1)
        b.run()
        ctx.sync()
        for (kind, a, bb, ta, tb, tr), (_, _, _, _, an, bn) in zip(keep, jobs):
            got = tr.cpu().numpy().view(np.uint64)
            want = O.port_sqr(a) if kind == sbg.JOB_SQR else O.port_mul(a, bb)
            assert np.array_equal(got, want), (rep, kind, an, bn)
    b.close()


def test_engine_autotune_keeps_products_exact(ctx):
    """sbg_batch_autotune times the three engines on the batch and keeps the
    fastest; the products it leaves behind, and those of the captured graph
    on the chosen engine, equal the oracle's."""
    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(306)
    shapes = _shapes(rng, 60)
    jobs, keep = _mixed_jobs(rng, shapes)
    b = sbg.Batch(ctx, jobs)
    ms = b.autotune()
    assert len(ms) == 3 and all(m > 0 for m in ms)
    b.capture()
    for *_, tr in keep:
        tr.fill_(-1)
    b.run()
    ctx.sync()
    for (kind, a, bb, ta, tb, tr), (_, _, _, _, an, bn) in zip(keep, jobs):
        got = tr.cpu().numpy().view(np.uint64)
        if kind == sbg.JOB_MUL:
            want = O.port_mul(a, bb)
        elif kind == sbg.JOB_SQR:
            want = O.port_sqr(a)
        else:
            want = O.mulmid(a, bb, "ntt")
        assert np.array_equal(got, want), (kind, an, bn)
    b.close()
