// sbg_school.cu -- the small-size front end: schoolbook products of at most
// SBG_SCHOOL_MAX output limbs, one warp per product.
//
// Below a few dozen limbs a five-prime transform is all overhead (five CTAs,
// three transforms and a CRT launch for a handful of limbs).  The reference
// covers this band with its own basecase kernels (include/u64cvt.h:100-106:
// an asm basecase up to 6 limbs, include/mul.h:764 basecase / Toom below the
// FFT band); here a warp forms the product column by column in exact 64-bit
// arithmetic:
//   * lane l owns the columns k = 32 s + l (s = 0..3), accumulating
//     sum_{i+j=k} a_i b_j in 192 bits (lo, mid, hi) with the PTX multiply-add
//     carry chain (mad.lo.cc / madc.hi.cc / addc);
//   * limb m of the product is lo_m + mid_{m-1} + hi_{m-2} + carries, the
//     same three-stream recombination as the CRT kernel's; the neighbour
//     terms come by shuffles, the sum carries (0..2) from the lane below, and
//     the ripple carries of a 32-limb step are resolved at once from the
//     lanes' generate / propagate ballots: carries = (p + (g << 1 | c)) ^ p.
// Operands are staged in shared memory (2 KB per warp), so each a_i is a
// broadcast and the b_{k-i} of a warp are 32 consecutive words.
#include <cuda_runtime.h>

#include "sbg_internal.h"
#include "sbg_school.cuh"

namespace sbg {

__global__ void __launch_bounds__(32) k_school(const uint64_t* __restrict__ a, int an,
                                               const uint64_t* __restrict__ b, int bn,
                                               uint64_t* __restrict__ out) {
    __shared__ uint64_t sa[SBG_SCHOOL_MAX], sb[SBG_SCHOOL_MAX];
    school_warp(a, an, b, bn, out, sa, sb);
}

// batched: one warp per job (plain products only: cmin = 0, off = 0)
__global__ void __launch_bounds__(32 * SCHOOL_WARPS) k_school_b(const JobDesc* __restrict__ jobs,
                                                                int njobs) {
    __shared__ uint64_t sa[SCHOOL_WARPS][SBG_SCHOOL_MAX], sb[SCHOOL_WARPS][SBG_SCHOOL_MAX];
    const int w = threadIdx.x >> 5;
    const int j = blockIdx.x * SCHOOL_WARPS + w;
    if (j >= njobs) return;
    const JobDesc& J = jobs[j];
    school_warp(J.a, (int)J.an, J.b, (int)J.bn, J.out, sa[w], sb[w]);
}

cudaError_t launch_school(const uint64_t* a, int64_t an, const uint64_t* b, int64_t bn,
                          uint64_t* out, cudaStream_t st) {
    if (an <= 0 || bn <= 0 || an + bn > SBG_SCHOOL_MAX) return cudaErrorInvalidValue;
    k_school<<<1, 32, 0, st>>>(a, (int)an, b, (int)bn, out);
    return cudaGetLastError();
}

cudaError_t launch_school_batch(const JobDesc* djobs, int njobs, cudaStream_t st) {
    if (njobs <= 0) return cudaSuccess;
    k_school_b<<<(njobs + SCHOOL_WARPS - 1) / SCHOOL_WARPS, 32 * SCHOOL_WARPS, 0, st>>>(djobs, njobs);
    return cudaGetLastError();
}

}  // namespace sbg
