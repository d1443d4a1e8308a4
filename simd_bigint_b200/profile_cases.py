"""Small, representative calls of the library's kernels, one case per
command, for capturing them under a profiler:

    python -m simd_bigint_b200.profile_cases <case> [repeats]

Cases (operands seeded, resident on cuda:0, each call repeated `repeats`
times, 3 by default, so a capture can skip the first launch):

    small     one 1500 x 1500-limb product (single-CTA transforms, k_small,
              the short-product carry scan k_crt_carry_s)
    mid       one 16384 x 16384-limb product (four-step kernels at 2^15
              points, k_crt_carry_s)
    school    one 40 x 60-limb product (schoolbook warp, k_school)
    batch     a 512-product mixed batch on the per-class engine (k_*_b)
    persist   the same batch on the persistent queue kernel (k_persist)
    divwarp   256 divisions of 200 by 100 limbs (warp block division)
    recip     one reciprocal of 3000 limbs (Newton path, its base case)
    div       6 divisions of 2n by n limbs, n = 5000 and 40000 (Newton path;
              its linear steps single-CTA and clustered)
    u52       u64 <-> u52 conversions of 2^22 limbs (k_u52_*)

Each run ends with the products checked against a host recomputation of a
sample, so a capture of a wrong result is noticed."""
from __future__ import annotations

import sys

import numpy as np


def _t(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint64).view(np.int64)).cuda()


def _int(a) -> int:
    return int.from_bytes(np.ascontiguousarray(a, dtype="<u8").tobytes(), "little")


def _mixed(ctx, count, rng, sbg):
    import torch
    from .workloads import fill_limbs, mixed_batch_shapes
    keep, jobs = [], []
    for kind, an, bn in mixed_batch_shapes(count, seed=4321):
        a = fill_limbs(an, rng)
        b = a if kind == sbg.JOB_SQR else fill_limbs(bn, rng)
        ta, tb = _t(a), _t(b)
        r = torch.empty(sbg.out_limbs(kind, an, bn), dtype=torch.int64, device="cuda")
        keep.append((a, b, ta, tb, r))
        jobs.append((kind, r.data_ptr(), ta.data_ptr(), tb.data_ptr(), an, bn))
    return jobs, keep


def main(argv: list[str]) -> int:
    import torch

    import simd_bigint_b200 as sbg
    case = argv[0] if argv else "small"
    reps = int(argv[1]) if len(argv) > 1 else 3
    rng = np.random.default_rng(2027)
    ctx = sbg.Context(0)
    ok = True
    if case in ("small", "school", "mid"):
        an, bn = {"small": (1500, 1500), "school": (40, 60), "mid": (16384, 16384)}[case]
        a, b = rng.integers(0, 2**64, an, dtype=np.uint64), rng.integers(0, 2**64, bn, dtype=np.uint64)
        ta, tb = _t(a), _t(b)
        r = torch.empty(an + bn, dtype=torch.int64, device="cuda")
        for _ in range(reps):
            ctx.mul(r, ta, tb)
        ctx.sync()
        ok = _int(r.cpu().numpy().view(np.uint64)) == _int(a) * _int(b)
    elif case in ("batch", "persist"):
        jobs, keep = _mixed(ctx, 512, rng, sbg)
        bt = sbg.Batch(ctx, jobs)
        bt.set_engine(1 if case == "batch" else 0)
        for _ in range(reps):
            bt.run()
        ctx.sync()
        for a, b, _, _, r in keep[::37]:
            ok &= _int(r.cpu().numpy().view(np.uint64)) == _int(a) * _int(b)
        bt.close()
    elif case in ("divwarp", "recip", "div"):
        from .workloads import fill_limbs
        if case in ("divwarp", "div"):
            ns = [100] * 256 if case == "divwarp" else [5000, 40000, 5000, 40000, 5000, 5000]
            count = len(ns)
            Ns = [fill_limbs(2 * n, rng) for n in ns]
            Ds = [fill_limbs(n, rng, top_bit=True) for n in ns]
            tN, tD = [_t(x) for x in Ns], [_t(x) for x in Ds]
            tQ = [torch.empty(n + 1, dtype=torch.int64, device="cuda") for n in ns]
            tR = [torch.empty(n, dtype=torch.int64, device="cuda") for n in ns]
            jobs = [(q.data_ptr(), r.data_ptr(), x.data_ptr(), d.data_ptr(), 2 * n, n)
                    for q, r, x, d, n in zip(tQ, tR, tN, tD, ns)]
            for _ in range(reps):
                ctx.divrem_batch(jobs)
            for i in range(0, count, 31 if case == "divwarp" else 1):
                q, rr = divmod(_int(Ns[i]), _int(Ds[i]))
                ok &= _int(tQ[i].cpu().numpy().view(np.uint64)) == q
                ok &= _int(tR[i].cpu().numpy().view(np.uint64)) == rr
        else:
            n = 3000
            D = fill_limbs(n, rng, top_bit=True)
            tD = _t(D)
            v = torch.empty(n, dtype=torch.int64, device="cuda")
            for _ in range(reps):
                ctx.recip(v, tD)
            Dv = _int(D)
            ok = _int(v.cpu().numpy().view(np.uint64)) == ((1 << (128 * n)) - 1) // Dv - (1 << (64 * n))
    elif case == "u52":
        n = 1 << 22
        a = rng.integers(0, 2**64, n, dtype=np.uint64)
        ta = _t(a)
        n52 = (64 * n + 51) // 52
        d = torch.empty(n52, dtype=torch.int64, device="cuda")
        back = torch.empty(n, dtype=torch.int64, device="cuda")
        for _ in range(reps):
            ctx.u52_from_u64(d, ta)
            ctx.u64_from_u52(back, d)
        ctx.sync()
        ok = bool(np.array_equal(back.cpu().numpy().view(np.uint64), a))
    else:
        print(f"unknown case {case}", file=sys.stderr)
        return 2
    ctx.close()
    print(f"{case}: {'ok' if ok else 'MISMATCH'}")
    return 0 if ok else 1


if __name__ == "__main__":
    raise SystemExit(main(sys.argv[1:]))
