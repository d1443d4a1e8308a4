"""Shared helpers of the test suite (inputs, digests, fixtures)."""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import numpy as np

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden.json"

def _is_prime(n: int) -> bool:
    """Miller-Rabin with the first twelve prime bases (deterministic below 3.3e24)."""
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for p in small:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def random_primes(seed: int, k: int = 4, bits: int = 61) -> list[int]:
    """k distinct random primes of `bits` bits drawn from `seed`."""
    import random
    rnd = random.Random(seed)
    out: list[int] = []
    while len(out) < k:
        c = rnd.getrandbits(bits) | (1 << (bits - 1)) | 1
        if c not in out and _is_prime(c):
            out.append(c)
    return out


# The modular spot check draws fresh random 61-bit primes in every session,
# from a seed that is logged (and replayable through SBG_SPOT_SEED).
SPOT_SEED = int(os.environ.get("SBG_SPOT_SEED") or int.from_bytes(os.urandom(4), "little"))
SPOT_PRIMES = random_primes(SPOT_SEED)
print(f"[spot check] seed {SPOT_SEED}: primes {SPOT_PRIMES}")


def golden() -> dict:
    return json.loads(GOLDEN.read_text())


def digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<u8").tobytes()).hexdigest()


def golden_inputs(op, an, bn, pat, seed):
    if pat == "xs":
        a, st = O.xorshift(an, seed)
        b = a if op == "sqr" else O.xorshift(bn, st)[0]
    else:
        a = O.pattern(an, pat)
        b = a if op == "sqr" else O.pattern(bn, "weyl_b" if pat == "weyl_a" else pat)
    return a, b


def div_inputs(n, seed):
    a, st = O.xorshift(2 * n, seed)
    d, _ = O.xorshift(n, st)
    d[-1] |= np.uint64(1 << 63)
    return a, d


def rand_limbs(n: int, rng: np.random.Generator, top_nonzero: bool = True) -> np.ndarray:
    x = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if top_nonzero and n and x[-1] == 0:
        x[-1] = 1
    return x


def spot_check(a: np.ndarray, b: np.ndarray, r: np.ndarray, primes=SPOT_PRIMES) -> bool:
    """(A mod q)(B mod q) == R mod q for each q: the random-prime modular check."""
    for q in primes:
        if (O.mod_u64(a, q) * O.mod_u64(b, q)) % q != O.mod_u64(r, q):
            return False
    return True


def ones_square(n: int) -> np.ndarray:
    """(B^n - 1)^2 = B^2n - 2 B^n + 1 in closed form (the all-0xFF worst case)."""
    r = np.zeros(2 * n, dtype=np.uint64)
    r[0] = 1
    r[n] = np.uint64(0xFFFFFFFFFFFFFFFE)
    r[n + 1:] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return r
