"""Shared helpers of the test suite (inputs, digests, fixtures)."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden.json"

# the reference batteries' spot-check idea: random 61-bit primes
SPOT_PRIMES = [2305843009213693951, 2305843009213693921, 2305843009213693907,
               2305843009213693669]


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
