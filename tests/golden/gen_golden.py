"""Generate the golden vectors in tests/golden/golden.json from the UNMODIFIED
reference (oracle/_ref/libsbref.so, built by `make -C oracle ref` from the
reference's own sources).  Run in a container that has the reference and an
AVX-512 IFMA host:

    python tests/golden/gen_golden.py [--missing]

Inputs are regenerated from their description (xorshift64 seed or a fixed
fill pattern, see golden_inputs()), so the file stores only the shape, the
pattern and a digest of the reference's output plus a few limbs.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
from oracle import oracle as O  # noqa: E402

# (op, an, bn, pattern, seed): pattern "xs" = xorshift64 stream from `seed`
# (a first, b continues the stream), otherwise a fill pattern of oracle.pattern
MUL_CASES = [
    ("mul", 1, 1, "xs", 42), ("mul", 3, 5, "xs", 42), ("mul", 40, 40, "xs", 42),
    ("mul", 24, 7, "ones", 0), ("mul", 1000, 999, "xs", 7),
    ("mul", 4096, 4096, "ones", 0), ("mul", 4096, 4096, "sparse", 0),
    ("mul", 16384, 16384, "xs", 42),                 # the single balanced config
    ("mul", 65536, 65536, "ones", 0), ("mul", 100000, 17, "ones", 0),
    ("mul", 180224, 180223, "xs", 11),
    ("mul", (1 << 20) + 7, (1 << 19) - 3, "ones", 0),
    ("mul", 1 << 20, 1 << 20, "xs", 42),
    ("mul", (1 << 21) - 3, (1 << 21) - 1, "xs", 3),
    ("mul", 1 << 22, 1 << 22, "xs", 42),             # 2^22 x 2^22
    ("sqr", 80, 80, "xs", 5), ("sqr", 4096, 4096, "ones", 0),
    ("sqr", 65536, 65536, "weyl_a", 0), ("sqr", 1 << 20, 1 << 20, "xs", 9),
    ("sqr", 1 << 21, 1 << 21, "ones", 0),
    # the large single-product configurations, on the same xorshift64 stream
    # (seed 42) that bench.py multiplies: 2^24 x 2^24, sqr 2^24, 2^24 x 2^20
    ("mul", 1 << 24, 1 << 24, "xs", 42),
    ("sqr", 1 << 24, 1 << 24, "xs", 42),
    ("mul", 1 << 24, 1 << 20, "xs", 42),
    ("sqr", 1 << 22, 1 << 22, "xs", 42),
]
DIV_CASES = [(1024, 512, 21), (2000, 1000, 22), (8192, 4096, 23), (131072, 65536, 24),
             (524288, 262144, 25)]                   # the top divisor size of the division batch


def golden_inputs(op: str, an: int, bn: int, pat: str, seed: int):
    if pat == "xs":
        a, st = O.xorshift(an, seed)
        b = a if op == "sqr" else O.xorshift(bn, st)[0]
    else:
        a = O.pattern(an, pat)
        b = a if op == "sqr" else O.pattern(bn, "weyl_b" if pat == "weyl_a" else pat)
    return a, b


def div_inputs(n: int, seed: int):
    a, st = O.xorshift(2 * n, seed)
    d, _ = O.xorshift(n, st)
    d[-1] |= np.uint64(1 << 63)
    return a, d


def digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<u8").tobytes()).hexdigest()


def summary(x: np.ndarray) -> dict:
    return {"sha256": digest(x), "n": int(len(x)),
            "head": [f"{int(v):016x}" for v in x[:4]], "tail": [f"{int(v):016x}" for v in x[-4:]]}


def main():
    """Writes golden.json.  With --missing, entries already in the file are
    kept and only cases not yet present are computed (a reference product at
    2^24 limbs costs minutes including its plan build on a slow host)."""
    if not O.ref_available():
        raise SystemExit("reference oracle not available (make -C oracle ref; AVX-512 IFMA host)")
    keep = "--missing" in sys.argv[1:] and (HERE / "golden.json").exists()
    old = json.loads((HERE / "golden.json").read_text()) if keep else {"mul": [], "div": []}
    have_mul = {(e["op"], e["an"], e["bn"], e["pattern"], e["seed"]): e for e in old["mul"]}
    have_div = {(e["nn"], e["dn"], e["seed"]): e for e in old["div"]}
    out = {"generator": "tests/golden/gen_golden.py", "source": "reference nt_mul / nt_sqr / divrem_u64_dc",
           "mul": [], "div": []}
    for op, an, bn, pat, seed in MUL_CASES:
        if (op, an, bn, pat, seed) in have_mul:
            out["mul"].append(have_mul[(op, an, bn, pat, seed)])
            continue
        t = time.time()
        a, b = golden_inputs(op, an, bn, pat, seed)
        r = O.ref_sqr(a) if op == "sqr" else O.ref_mul(a, b)
        out["mul"].append({"op": op, "an": an, "bn": bn, "pattern": pat, "seed": seed, **summary(r)})
        print(op, an, bn, pat, f"{time.time() - t:.2f}s", flush=True)
    for n2, n, seed in DIV_CASES:
        if (n2, n, seed) in have_div:
            out["div"].append(have_div[(n2, n, seed)])
            continue
        a, d = div_inputs(n, seed)
        q, r = O.ref_divrem(a, d)
        out["div"].append({"nn": n2, "dn": n, "seed": seed, "q": summary(q), "r": summary(r)})
        print("div", n2, n, flush=True)
    (HERE / "golden.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
