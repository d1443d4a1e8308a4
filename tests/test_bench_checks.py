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
