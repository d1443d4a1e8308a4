"""GPU tests of the Newton reciprocal and division (sbg_recip, sbg_divrem,
sbg_divrem_batch).

Quotients and remainders must equal the reference's divrem_u64_dc
(include/dc_div.h:154) bit for bit: against its golden digests
(tests/golden/golden.json, generated by the unmodified reference), and
against our restatement (Knuth D, oracle/port.c) and Python integers on
further shapes, including the all-0xFF and minimal (B^n / 2) divisors.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import digest, div_inputs, golden

pytestmark = pytest.mark.gpu
G = golden()


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _divrem(ctx, N, D):
    import torch
    q = torch.empty(len(N) - len(D) + 1, dtype=torch.int64, device="cuda")
    r = torch.empty(len(D), dtype=torch.int64, device="cuda")
    ctx.divrem(q, r, _dev(N), _dev(D))
    return _host(q), _host(r)


@pytest.mark.parametrize("case", G["div"], ids=lambda c: f'div-{c["nn"]}/{c["dn"]}')
def test_divrem_matches_reference_golden(ctx, case):
    N, D = div_inputs(case["dn"], case["seed"])
    q, r = _divrem(ctx, N, D)
    assert digest(q) == case["q"]["sha256"]
    assert digest(r) == case["r"]["sha256"]


def test_divrem_shapes_vs_python(ctx):
    rng = np.random.default_rng(401)
    for n in [1, 2, 3, 5, 31, 32, 33, 64, 100, 257, 1000, 4097, 20000]:
        for nn in sorted({n, n + 1, (3 * n) // 2 + 1, 2 * n}):
            if nn < n or nn > 2 * n:
                continue
            N = rng.integers(0, 2**64, nn, dtype=np.uint64)
            D = rng.integers(0, 2**64, n, dtype=np.uint64)
            D[-1] |= np.uint64(1 << 63)
            q, r = _divrem(ctx, N, D)
            qq, rr = divmod(O.to_int(N), O.to_int(D))
            assert O.to_int(q) == qq and O.to_int(r) == rr, (n, nn)


def test_divrem_adversarial_divisors(ctx):
    for n in [40, 333, 5000]:
        ones = O.pattern(2 * n, "ones")
        for D in (O.pattern(n, "ones"),
                  np.concatenate([np.zeros(n - 1, np.uint64), np.array([1 << 63], np.uint64)])):
            q, r = _divrem(ctx, ones, D)
            qq, rr = divmod(O.to_int(ones), O.to_int(D))
            assert O.to_int(q) == qq and O.to_int(r) == rr, n


def test_recip_exact(ctx):
    import torch
    rng = np.random.default_rng(402)
    for n in [1, 7, 32, 33, 100, 1000, 8191]:
        D = rng.integers(0, 2**64, n, dtype=np.uint64)
        D[-1] |= np.uint64(1 << 63)
        i = torch.empty(n, dtype=torch.int64, device="cuda")
        ctx.recip(i, _dev(D))
        want = ((1 << (128 * n)) - 1) // O.to_int(D) - (1 << (64 * n))
        assert O.to_int(_host(i)) == want, n
        if n <= 1000:
            assert np.array_equal(_host(i), O.port_recip(D))


def test_divrem_batch_vs_port(ctx):
    import torch
    rng = np.random.default_rng(403)
    ns = [512, 700, 1500, 3000, 9000, 513, 40000]
    jobs, keep = [], []
    for n in ns:
        N = rng.integers(0, 2**64, 2 * n, dtype=np.uint64)
        D = rng.integers(0, 2**64, n, dtype=np.uint64)
        D[-1] |= np.uint64(1 << 63)
        tN, tD = _dev(N), _dev(D)
        q = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
        r = torch.full((n,), -1, dtype=torch.int64, device="cuda")
        jobs.append((q.data_ptr(), r.data_ptr(), tN.data_ptr(), tD.data_ptr(), 2 * n, n))
        keep.append((N, D, tN, tD, q, r))
    ctx.divrem_batch(jobs)
    for N, D, tN, tD, q, r in keep:
        qq, rr = O.port_divrem(N, D)
        assert np.array_equal(_host(q), qq) and np.array_equal(_host(r), rr), len(D)


def test_reference_signature_divrem_any_shape(ctx):
    """sbg_divrem_u64: the reference's divrem_u64 contract (any divisor with
    a nonzero top limb, any nn >= dn, trimmed lengths) on host arrays."""
    import simd_bigint_b200 as sbg
    rng = np.random.default_rng(404)
    for dn, nn in [(1, 1), (1, 9), (2, 5), (7, 7), (7, 30), (50, 260), (300, 1000), (1000, 5000)]:
        N = rng.integers(0, 2**64, nn, dtype=np.uint64)
        D = rng.integers(0, 2**64, dn, dtype=np.uint64)
        D[-1] = np.uint64(int(D[-1]) >> int(rng.integers(0, 63))) | np.uint64(1)
        q, r = sbg.divrem_u64(N, D)
        qq, rr = divmod(O.to_int(N), O.to_int(D))
        assert O.to_int(q) == qq and O.to_int(r) == rr, (dn, nn)
        assert len(q) >= 1 and len(r) >= 1
        assert (len(q) == 1 or q[-1] != 0) and (len(r) == 1 or r[-1] != 0)
        if O.ref_available() and O.to_int(D).bit_length() > 416:
            q2, r2 = O.ref_divrem(N, D)
            assert O.to_int(q2) == qq and O.to_int(r2) == rr


def test_divrem_many_in_flight(ctx):
    """A wide batch (many divisions, many recursion rounds in flight): every
    quotient and remainder satisfies Q D + R = N (mod two 61-bit primes) with
    0 <= R < D.  Guards the per-round descriptor reuse across rounds."""
    import torch

    from simd_bigint_b200.workloads import division_shapes, fill_limbs
    ns = division_shapes(160, seed=77, lo=512, hi=40000)
    rng = np.random.default_rng(405)
    hostN = [fill_limbs(2 * n, rng) for n in ns]
    hostD = [fill_limbs(n, rng, top_bit=True) for n in ns]
    tN = [_dev(x) for x in hostN]
    tD = [_dev(x) for x in hostD]
    tQ = [torch.zeros(n + 1, dtype=torch.int64, device="cuda") for n in ns]
    tR = [torch.zeros(n, dtype=torch.int64, device="cuda") for n in ns]
    ctx.divrem_batch([(q.data_ptr(), r.data_ptr(), a.data_ptr(), d.data_ptr(), 2 * n, n)
                      for q, r, a, d, n in zip(tQ, tR, tN, tD, ns)])
    for N, D, q, r in zip(hostN, hostD, tQ, tR):
        Q, R = _host(q), _host(r)
        for p in (2305843009213693951, 2305843009213693921):
            assert (O.mod_u64(Q, p) * O.mod_u64(D, p) + O.mod_u64(R, p)) % p == O.mod_u64(N, p)
        hi = np.nonzero(R != D)[0]
        assert len(hi) and R[hi[-1]] < D[hi[-1]]


def test_cluster_sized_divisions_extreme_carries(ctx):
    """Divisions large enough for the clustered linear steps (n >= 32768),
    with the carry-heaviest operands: an all-ones numerator over all-ones and
    minimal (B^n / 2) divisors, checked as Q D + R = N with 0 <= R < D."""
    n = 40000
    ones = O.pattern(2 * n, "ones")
    for D in (O.pattern(n, "ones"),
              np.concatenate([np.zeros(n - 1, np.uint64), np.array([1 << 63], np.uint64)])):
        q, r = _divrem(ctx, ones, D)
        Nv, Dv, Qv, Rv = O.to_int(ones), O.to_int(D), O.to_int(q), O.to_int(r)
        assert Qv * Dv + Rv == Nv and 0 <= Rv < Dv


def test_cluster_sized_recip_exact(ctx):
    """The exact reciprocal at a clustered size: V = floor((B^2n - 1) / D) - B^n
    holds iff 0 <= B^2n - 1 - D (V + B^n) < D."""
    import torch
    rng = np.random.default_rng(406)
    n = 40000
    D = rng.integers(0, 2**64, n, dtype=np.uint64)
    D[-1] |= np.uint64(1 << 63)
    i = torch.empty(n, dtype=torch.int64, device="cuda")
    ctx.recip(i, _dev(D))
    Dv, Vv = O.to_int(D), O.to_int(_host(i))
    rem = (1 << (128 * n)) - 1 - Dv * (Vv + (1 << (64 * n)))
    assert 0 <= rem < Dv


def test_async_batches_back_to_back_match_sync(ctx):
    """sbg_divrem_batch_async: three batches queued without waiting (the
    scratch, descriptor ring and padded numerators reused in stream order),
    one sbg_divrem_wait, then every quotient and remainder equals the
    synchronous sbg_divrem_batch on the same inputs."""
    import torch
    rng = np.random.default_rng(407)
    batches = [[700, 1500, 3000], [40000, 513], [9000, 2048, 33000, 600]]
    keep = []
    for ns in batches:
        jobs, held = [], []
        for n in ns:
            N = rng.integers(0, 2**64, 2 * n, dtype=np.uint64)
            D = rng.integers(0, 2**64, n, dtype=np.uint64)
            D[-1] |= np.uint64(1 << 63)
            tN, tD = _dev(N), _dev(D)
            q = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
            r = torch.full((n,), -1, dtype=torch.int64, device="cuda")
            jobs.append((q.data_ptr(), r.data_ptr(), tN.data_ptr(), tD.data_ptr(), 2 * n, n))
            held.append((tN, tD, q, r, n))
        ctx.divrem_batch_async(jobs)
        keep.append(held)
    ctx.divrem_wait()
    for held in keep:
        sync_jobs, outs = [], []
        for tN, tD, q, r, n in held:
            q2 = torch.empty(n + 1, dtype=torch.int64, device="cuda")
            r2 = torch.empty(n, dtype=torch.int64, device="cuda")
            sync_jobs.append((q2.data_ptr(), r2.data_ptr(), tN.data_ptr(), tD.data_ptr(), 2 * n, n))
            outs.append((q, r, q2, r2))
        ctx.divrem_batch(sync_jobs)
        for q, r, q2, r2 in outs:
            assert torch.equal(q, q2) and torch.equal(r, r2)


def test_block_division_small_divisors(ctx):
    """Divisors of at most 127 limbs run as one warp per division (block
    division with 3-by-2 quotient estimates).  Every size 1..127, numerator
    lengths from dn to 2 dn, random and adversarial operands: the all-ones
    numerator, the minimal normalised divisor B^n / 2 (the largest quotient
    limbs), all-ones divisors (the estimate's equal-top-limbs case), and
    remainders that need the add-back."""
    rng = np.random.default_rng(407)
    for dn in list(range(1, 34)) + [47, 63, 64, 65, 100, 126, 127]:
        cases = []
        for nn in sorted({dn, dn + 1, dn + dn // 2, 2 * dn}):
            N = rng.integers(0, 2**64, nn, dtype=np.uint64)
            D = rng.integers(0, 2**64, dn, dtype=np.uint64)
            D[-1] |= np.uint64(1 << 63)
            cases.append((N, D))
        minD = np.zeros(dn, np.uint64)
        minD[-1] = np.uint64(1 << 63)
        cases += [(O.pattern(2 * dn, "ones"), O.pattern(dn, "ones")), (O.pattern(2 * dn, "ones"), minD)]
        # top limbs of the running remainder equal to the divisor's
        D = rng.integers(0, 2**64, dn, dtype=np.uint64)
        D[-1] |= np.uint64(1 << 63)
        Dv = O.to_int(D)
        cases.append((O.from_int(Dv * ((1 << (64 * dn)) - 1) + Dv - 1, 2 * dn), D))
        for N, D in cases:
            q, r = _divrem(ctx, N, D)
            qq, rr = divmod(O.to_int(N), O.to_int(D))
            assert O.to_int(q) == qq and O.to_int(r) == rr, (dn, len(N))


def test_batch_mixing_warp_and_newton_divisions(ctx):
    import torch
    rng = np.random.default_rng(408)
    ns = [1, 5, 64, 127, 128, 500, 127, 3000, 2, 129]
    jobs, keep = [], []
    for n in ns:
        N = rng.integers(0, 2**64, 2 * n, dtype=np.uint64)
        D = rng.integers(0, 2**64, n, dtype=np.uint64)
        D[-1] |= np.uint64(1 << 63)
        tN, tD = _dev(N), _dev(D)
        q = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
        r = torch.full((n,), -1, dtype=torch.int64, device="cuda")
        jobs.append((q.data_ptr(), r.data_ptr(), tN.data_ptr(), tD.data_ptr(), 2 * n, n))
        keep.append((N, D, tN, tD, q, r))
    ctx.divrem_batch(jobs)
    for N, D, _, _, q, r in keep:
        qq, rr = divmod(O.to_int(N), O.to_int(D))
        assert O.to_int(_host(q)) == qq and O.to_int(_host(r)) == rr, len(D)
