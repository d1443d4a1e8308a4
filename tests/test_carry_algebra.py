"""CPU checks of the carry algebra the GPU kernels are built on.

These restate, on Python integers, the identities that the CRT carry kernel
and the division's linear steps use, so that a change to them is caught
without a GPU:

* carry resolution from generate / propagate bit masks by one add,
  (p + (g << 1 | c)) ^ p, with positions past the length propagating, and
  the group carry (p + (g << 1 | c)) >> W | g >> (W - 1);
* the division remainder's three chains in one pass (fold of C modulo
  B^L - 1, N_lo - C, + N_hi) and their net end-around correction
  d = c2 - b - c;
* the Newton step's corrections formed as W = k A - E on n + 1 limbs.
"""
import random

M64 = (1 << 64) - 1


def _resolve(g, p, c, width):
    s = p + (((g << 1) | c) & ((1 << width) - 1))
    carries = (s ^ p) & ((1 << width) - 1)
    out = ((s >> width) | (g >> (width - 1))) & 1
    return carries, out


def _ripple(g, p, c, width):
    carries, cur = 0, c
    for i in range(width):
        carries |= cur << i
        gi, pi = (g >> i) & 1, (p >> i) & 1
        cur = gi | (pi & cur)
    return carries, cur


def test_ballot_add_resolves_carries_like_a_ripple():
    rng = random.Random(11)
    for width in (4, 32):
        for _ in range(4000):
            g = rng.getrandbits(width)
            p = rng.getrandbits(width) & ~g          # generate and propagate exclusive
            if rng.random() < 0.3:
                p = ((1 << width) - 1) & ~g          # long propagate runs
            c = rng.getrandbits(1)
            assert _resolve(g, p, c, width) == _ripple(g, p, c, width)


def _limb_chain(a, b, sub, length):
    """Add or subtract limb lists the way a tile does: generate / propagate
    masks per 32-limb row, resolved by one add each, rows in order."""
    out, carry = [], 0
    for r0 in range(0, len(a), 32):
        g = p = 0
        d = []
        for lane in range(32):
            i = r0 + lane
            inside = i < length
            x = a[i] if inside else 0
            y = b[i] if inside else 0
            if sub:
                v = (x - y) & M64
                gi, pi = x < y, (not inside) or v == 0
            else:
                v = (x + y) & M64
                gi, pi = v < x, (not inside) or v == M64
            d.append(v)
            g |= int(gi) << lane
            p |= int(pi) << lane
        cm, carry = _resolve(g, p, carry, 32)
        for lane in range(32):
            if r0 + lane < length:
                bit = (cm >> lane) & 1
                out.append((d[lane] - bit) & M64 if sub else (d[lane] + bit) & M64)
    return out, carry


def _val(v):
    return sum(x << (64 * i) for i, x in enumerate(v))


def test_tiled_add_and_subtract_with_ragged_lengths():
    rng = random.Random(12)
    for length in (1, 31, 32, 33, 100, 257):
        padded = -(-length // 32) * 32
        for pattern in ("random", "ones"):
            a = [rng.getrandbits(64) if pattern == "random" else M64 for _ in range(padded)]
            b = [rng.getrandbits(64) if pattern == "random" else (1 if i == 0 else 0) for i in range(padded)]
            s, c = _limb_chain(a, b, False, length)
            want = _val(a[:length]) + _val(b[:length])
            assert _val(s) == want % (1 << (64 * length)) and c == want >> (64 * length)
            d, bo = _limb_chain(a, b, True, length)
            want = _val(a[:length]) - _val(b[:length])
            assert _val(d) == want % (1 << (64 * length)) and bo == int(want < 0)


def _seq_chain(a, b, sub):
    out, c = [], 0
    for x, y in zip(a, b):
        v = x - y - c if sub else x + y + c
        c = (1 if v < 0 else 0) if sub else v >> 64
        out.append(v & M64)
    return out, c


def _step(v, inc):
    for i in range(len(v)):
        old = v[i]
        v[i] = (old + 1) & M64 if inc else (old - 1) & M64
        if (inc and v[i] != 0) or (not inc and old != 0):
            return False
    return True


def test_end_around_remainder_three_chains():
    rng = random.Random(13)
    for trial in range(1500):
        n = rng.randint(3, 10)
        L = rng.randint(n + 3, 2 * n)
        kind = trial % 4
        if kind == 0:
            P = [rng.getrandbits(64) for _ in range(L + 3)]
            N = [rng.getrandbits(64) for _ in range(2 * n)]
        elif kind == 1:
            P = [M64] * (L + 3)
            N = [M64] * (2 * n)
        elif kind == 2:
            P = [0] * (L + 3)
            P[L] = 1
            N = [rng.getrandbits(64) for _ in range(2 * n)]
        else:
            P = [rng.getrandbits(64) for _ in range(L)] + [0, 0, 0]
            N = (P[:L] + [0] * (2 * n))[:2 * n]
        F, c = _seq_chain(P[:L], [P[L + i] if i < 3 else 0 for i in range(L)], False)
        G, b = _seq_chain(N[:L], F, True)
        H, c2 = _seq_chain(G, [N[L + i] if L + i < 2 * n else 0 for i in range(L)], False)
        d = c2 - b - c
        if d > 0 and _step(H, True):
            H[0] = 1
        for _ in range(-d):
            if _step(H, False):
                _step(H, False)
        mod = (1 << (64 * L)) - 1
        got = _val(H)
        got = 0 if got == mod else got
        assert got == (_val(N) - _val(P)) % mod


def test_newton_corrections_as_k_a_minus_e():
    rng = random.Random(14)
    B = 1 << 64
    for trial in range(2000):
        n = rng.randint(4, 16)
        h = n - (n - 1) // 2
        l = n - h
        A = rng.getrandbits(64 * n) | (1 << (64 * n - 1))
        E = [rng.randrange(0, 2 * B ** n), rng.randint(1, 3) * A, rng.randint(0, 3) * A + 1][trial % 3]
        if E >= min(2 * B ** n, 4 * A):
            continue
        T = B ** (n + h) + E
        k_ref, Tr = 0, T
        while Tr >= B ** (n + h):
            Tr -= A
            k_ref += 1
        tm_ref = ((B ** (n + h) - Tr) >> (64 * l)) % B ** (h + 1)
        mod = B ** (n + 1)
        W = (A - E) % mod
        neg = A < E
        k = 1
        while neg or W == 0:
            s = W + A
            carry = s >= mod
            W = s % mod
            neg = neg and not carry
            k += 1
        assert k == k_ref and (W >> (64 * l)) % B ** (h + 1) == tm_ref
