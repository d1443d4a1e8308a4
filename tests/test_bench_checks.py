"""CPU checks of the spot check bench.py applies to every timed product
(A B = R modulo 2^61 - 1 and 2^64 - 1, and in the lowest limb): it accepts
the exact product and rejects products with a planted mistake."""
import numpy as np

import bench

M61 = (1 << 61) - 1
M64 = (1 << 64) - 1


def _to_int(v):
    return sum(int(x) << (64 * i) for i, x in enumerate(v))


def _limbs(x, n):
    return np.array([(x >> (64 * i)) & M64 for i in range(n)], dtype=np.uint64)


def test_residues_match_python_integers():
    rng = np.random.default_rng(21)
    for n in (1, 2, 7, 61, 62, 200, 4096):
        a = rng.integers(0, 2**64, n, dtype=np.uint64)
        r61, r64 = bench.residues(a)
        v = _to_int(a)
        assert r61 == v % M61 and r64 == v % M64
    ones = np.full(500, M64, dtype=np.uint64)
    v = _to_int(ones)
    assert bench.residues(ones) == (v % M61, v % M64)


def test_product_check_accepts_exact_and_rejects_planted_mistakes():
    rng = np.random.default_rng(22)
    for an, bn in ((1, 1), (5, 3), (300, 300), (1000, 17)):
        a = rng.integers(0, 2**64, an, dtype=np.uint64)
        b = rng.integers(0, 2**64, bn, dtype=np.uint64)
        r = _limbs(_to_int(a) * _to_int(b), an + bn)
        assert bench.product_ok(a, b, r)
        for pos in {0, (an + bn) // 2, an + bn - 1}:
            for delta in (1, 1 << 63):
                bad = r.copy()
                bad[pos] ^= np.uint64(delta)
                assert not bench.product_ok(a, b, bad), (an, bn, pos, delta)
        swapped = r.copy()
        if an + bn >= 2 and swapped[0] != swapped[1]:
            swapped[[0, 1]] = swapped[[1, 0]]
            assert not bench.product_ok(a, b, swapped)


def test_limbs_mod_matches_python_integers():
    rng = np.random.default_rng(23)
    primes = bench.random_primes(99)
    assert len(set(primes)) == 4 and all(p.bit_length() == 31 for p in primes)
    assert not set(primes) & set(bench.NTT_PRIMES)
    for n in (1, 3, 4095, 4096, 4097, 20000):
        a = rng.integers(0, 2**64, n, dtype=np.uint64)
        v = _to_int(a)
        for q in primes:
            assert bench.limbs_mod(a, q) == v % q, (n, q)


def test_random_prime_spot_check_rejects_planted_mistakes():
    rng = np.random.default_rng(24)
    a = rng.integers(0, 2**64, 3000, dtype=np.uint64)
    b = rng.integers(0, 2**64, 1700, dtype=np.uint64)
    r = _limbs(_to_int(a) * _to_int(b), 4700)
    primes = bench.random_primes(1234)
    assert bench.spot_check_primes(a, b, r, primes)
    for pos in (0, 2349, 4699):
        bad = r.copy()
        bad[pos] ^= np.uint64(1 << 17)
        assert not bench.spot_check_primes(a, b, bad, primes)


def test_xorshift_operands_are_the_reference_batteries_stream():
    """bench.py's operands (workloads.xorshift64_limbs, vectorised) equal the
    oracle's sequential xorshift64, the stream the golden digests were made on."""
    from oracle import oracle as O
    for op, an, bn in (("mul", 16384, 16384), ("sqr", 5000, 5000), ("mul", 70001, 999)):
        a, b = bench.xs_inputs(op, an, bn)
        a2, st = O.xorshift(an, 42)
        b2 = a2 if op == "sqr" else O.xorshift(bn, st)[0]
        assert np.array_equal(a, a2) and np.array_equal(b, b2)
        assert a[-1] != 0 and b[-1] != 0


def test_golden_digests_exist_for_the_single_product_workloads():
    for name in ("mul2p24", "sqr2p24", "mul2p22", "mul2p24x2p20", "mul16k"):
        op, an, bn = bench.WORKLOADS[name]
        assert bench.golden_sha256(op, an, bn), name
