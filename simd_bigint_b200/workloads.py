"""Seeded synthetic workloads of the benchmark configurations (shapes and
value distributions only; limbs are uniform random u64 with the top limb
nonzero).  Used by bench.py and by the tests."""
from __future__ import annotations

import math

import numpy as np

from . import JOB_MUL, JOB_SQR


def mixed_batch_shapes(count: int = 4096, seed: int = 12345, lo: int = 64, hi: int = 65536,
                       rmax: float = 8.0, sq_frac: float = 0.2) -> list[tuple[int, int, int]]:
    """The batched mixed-size configuration: an log-uniform in [lo, hi],
    bn = max(1, floor(an / r)) with r log-uniform in [1, rmax], a fraction
    sq_frac of squarings.  Returns (kind, an, bn) triples."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        an = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        r = math.exp(rng.uniform(0.0, math.log(rmax)))
        bn = max(1, int(an / r))
        sq = rng.uniform() < sq_frac
        out.append((JOB_SQR, an, an) if sq else (JOB_MUL, an, bn))
    return out


def division_shapes(count: int = 1024, seed: int = 4242, lo: int = 512,
                    hi: int = 262144) -> list[int]:
    """Divisor sizes n of the batched division configuration (numerator 2n
    limbs, divisor n limbs, top bit set), n log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return [int(math.exp(rng.uniform(math.log(lo), math.log(hi)))) for _ in range(count)]


_M64 = (1 << 64) - 1


def _xs_step_int(s: int) -> int:
    s ^= (s << 13) & _M64
    s ^= s >> 7
    s ^= (s << 17) & _M64
    return s


def _xs_jump(k: int) -> list[int]:
    """Columns of the GF(2) matrix of k xorshift64 steps (the generator is
    linear over GF(2)^64): column i is the image of the unit state 1 << i."""
    cols = [_xs_step_int(1 << i) for i in range(64)]          # one step
    acc = [1 << i for i in range(64)]                          # identity

    def apply(m, v):
        r = 0
        i = 0
        while v:
            if v & 1:
                r ^= m[i]
            v >>= 1
            i += 1
        return r

    while k:
        if k & 1:
            acc = [apply(cols, c) for c in acc]
        cols = [apply(cols, c) for c in cols]
        k >>= 1
    return acc


def xorshift64_limbs(n: int, state: int = 42, lanes: int = 4096) -> tuple[np.ndarray, int]:
    """n consecutive outputs of the xorshift64 generator (state ^= state << 13,
    ^= state >> 7, ^= state << 17; each output is the new state), the stream
    the reference's test batteries draw their operands from, and the state
    after them (to continue the stream for a second operand).  Vectorised:
    `lanes` independent starting points are found by jumping the linear
    generator ahead, then all lanes step together."""
    if n <= 0:
        return np.zeros(0, dtype=np.uint64), state
    lanes = max(1, min(lanes, n))
    chunk = -(-n // lanes)
    jump = _xs_jump(chunk)
    starts = []
    s = state
    for _ in range(lanes):
        starts.append(s)
        r = 0
        v, i = s, 0
        while v:
            if v & 1:
                r ^= jump[i]
            v >>= 1
            i += 1
        s = r
    st = np.array(starts, dtype=np.uint64)
    out = np.empty((lanes, chunk), dtype=np.uint64)
    a, b, c = np.uint64(13), np.uint64(7), np.uint64(17)
    for i in range(chunk):
        st ^= st << a
        st ^= st >> b
        st ^= st << c
        out[:, i] = st
    flat = out.reshape(-1)[:n].copy()
    return flat, int(flat[-1])


def fill_limbs(n: int, rng: np.random.Generator, top_bit: bool = False) -> np.ndarray:
    x = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if n:
        if top_bit:
            x[-1] |= np.uint64(1 << 63)
        elif x[-1] == 0:
            x[-1] = np.uint64(1)
    return x


def serving_requests(count: int, seed: int = 2025, lo: int = 32, hi: int = 1 << 20,
                     balanced: float = 0.7, rmax: float = 16.0,
                     mix: tuple[float, float, float] = (0.5, 0.3, 0.2)) -> list[tuple[int, int, int]]:
    """The serving configuration's request stream: (kind, an, bn) with an
    log-uniform in [lo, hi], 70% balanced (bn = an) and 30% unbalanced
    (bn = an / r, r log-uniform in (1, rmax]); kind 0 mul, 1 sqr, 2 reciprocal
    of an an-limb divisor, drawn with probabilities `mix`."""
    rng = np.random.default_rng(seed)
    out = []
    cdf = np.cumsum(mix)
    for _ in range(count):
        an = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        u = rng.uniform()
        kind = 0 if u < cdf[0] else (1 if u < cdf[1] else 2)
        if kind == 0:
            bn = an if rng.uniform() < balanced else max(1, int(an / math.exp(rng.uniform(0, math.log(rmax)))))
        else:
            bn = an
        out.append((kind, an, bn))
    return out


def poisson_arrivals(count: int, rate: float, seed: int = 7) -> np.ndarray:
    """Arrival times (seconds from 0) of a Poisson stream of `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))
