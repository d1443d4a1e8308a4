"""CPU tests of the oracle: our C restatement (oracle/port.c) pinned against
the reference's own outputs (golden vectors made by the unmodified reference,
and the reference library itself when it is built on this host)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import digest, div_inputs, golden, golden_inputs, ones_square

G = golden()


@pytest.mark.parametrize("case", [c for c in G["mul"] if max(c["an"], c["bn"]) <= (1 << 20)],
                         ids=lambda c: f'{c["op"]}-{c["an"]}x{c["bn"]}-{c["pattern"]}')
def test_port_matches_golden(case):
    a, b = golden_inputs(case["op"], case["an"], case["bn"], case["pattern"], case["seed"])
    r = O.port_sqr(a) if case["op"] == "sqr" else O.port_mul(a, b)
    assert digest(r) == case["sha256"]


def test_golden_digests_agree_with_python_ints():
    for case in G["mul"]:
        if max(case["an"], case["bn"]) > 4096:
            continue
        a, b = golden_inputs(case["op"], case["an"], case["bn"], case["pattern"], case["seed"])
        want = O.to_int(a) * O.to_int(b)
        assert digest(O.from_int(want, case["an"] + case["bn"])) == case["sha256"]


@pytest.mark.parametrize("case", [c for c in G["div"] if c["dn"] <= 65536],
                         ids=lambda c: f'div-{c["nn"]}/{c["dn"]}')
def test_port_divrem_matches_golden(case):
    a, d = div_inputs(case["dn"], case["seed"])
    q, r = O.port_divrem(a, d)
    assert digest(q) == case["q"]["sha256"]
    assert digest(r) == case["r"]["sha256"]


def test_port_small_grid_vs_python():
    rng = np.random.default_rng(1)
    for an in range(1, 25):
        for bn in range(1, 25):
            a = rng.integers(0, 2**64, an, dtype=np.uint64)
            b = rng.integers(0, 2**64, bn, dtype=np.uint64)
            want = O.to_int(a) * O.to_int(b)
            assert O.to_int(O.port_mul(a, b)) == want
            assert O.to_int(O.school_mul(a, b)) == want


@pytest.mark.skipif(not O.ref_available(), reason="reference not built / host lacks AVX-512 IFMA")
def test_port_vs_reference_random_shapes():
    rng = np.random.default_rng(2)
    for _ in range(12):
        an, bn = int(rng.integers(1, 30000)), int(rng.integers(1, 30000))
        pat = ["rand", "ones", "sparse"][int(rng.integers(0, 3))]
        a, b = O.pattern(an, pat, rng), O.pattern(bn, pat, rng)
        assert np.array_equal(O.port_mul(a, b), O.ref_mul(a, b))
        assert np.array_equal(O.port_sqr(a), O.ref_sqr(a))


def test_mulmid_definition():
    rng = np.random.default_rng(3)
    for an, bn in [(1, 1), (5, 1), (5, 5), (17, 4), (64, 33), (100, 99)]:
        a = rng.integers(0, 2**64, an, dtype=np.uint64)
        b = rng.integers(0, 2**64, bn, dtype=np.uint64)
        want = 0
        for i in range(an):
            for j in range(bn):
                if bn - 1 <= i + j <= an - 1:
                    want += int(a[i]) * int(b[j]) << (64 * (i + j - (bn - 1)))
        got = O.mulmid(a, b)
        assert O.to_int(got) == want
        assert np.array_equal(O.mulmid(a, b, "ntt"), got)


def test_mulmid_ntt_vs_school_larger():
    rng = np.random.default_rng(4)
    for an, bn, pat in [(3000, 1500, "rand"), (4097, 2049, "ones"), (2000, 7, "rand")]:
        a, b = O.pattern(an, pat, rng), O.pattern(bn, pat, rng)
        assert np.array_equal(O.mulmid(a, b, "ntt"), O.mulmid(a, b))


def test_recip_and_divrem_vs_python():
    rng = np.random.default_rng(5)
    for n in (1, 2, 7, 30, 300):
        d = rng.integers(0, 2**64, n, dtype=np.uint64)
        d[-1] |= np.uint64(1 << 63)
        i = O.port_recip(d)
        assert O.to_int(i) + (1 << (64 * n)) == ((1 << (128 * n)) - 1) // O.to_int(d)
        num = rng.integers(0, 2**64, 2 * n, dtype=np.uint64)
        q, r = O.port_divrem(num, d)
        qq, rr = divmod(O.to_int(num), O.to_int(d))
        assert O.to_int(q) == qq and O.to_int(r) == rr


def test_ones_square_closed_form():
    for n in (1, 2, 3, 100):
        a = O.pattern(n, "ones")
        assert np.array_equal(O.port_sqr(a), ones_square(n))


@pytest.mark.skipif(not O.ref_available(), reason="reference not built / host lacks AVX-512 IFMA")
def test_u52_restatement_matches_reference():
    """oracle.py's u52 boundary (Python integers) against the reference's own
    u52_from_u64 / u64_from_u52_canon / _canonneg."""
    rng = np.random.default_rng(7)
    for n in (1, 2, 3, 13, 64, 65, 777):
        for pat in ("rand", "ones", "sparse"):
            a = O.pattern(n, pat, rng)
            assert np.array_equal(O.ref_u52_from_u64(a), O.u52_from_u64(a)), (n, pat)
    for n52 in (1, 2, 8, 9, 17, 300, 1001):
        for signed in (False, True):
            d = (rng.integers(-(1 << 62), 1 << 62, n52).astype(np.int64).view(np.uint64) if signed
                 else rng.integers(0, 2**64, n52, dtype=np.uint64))
            d[-min(2, n52):] = rng.integers(0, 1 << 50, min(2, n52), dtype=np.uint64)
            rn = (52 * n52 + 63) // 64 + 1
            assert np.array_equal(O.ref_u64_from_u52(d, rn, signed), O.u64_from_u52(d, rn, signed))
