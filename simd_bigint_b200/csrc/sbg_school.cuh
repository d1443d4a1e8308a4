// sbg_school.cuh -- the schoolbook warp product (device code shared by the
// schoolbook kernels and the persistent batch kernel).  See sbg_school.cu
// for the method.
#pragma once
#include <cstdint>

#include "sbg_internal.h"

namespace sbg {

#define SCHOOL_WARPS 4                      // warps (products) per CTA of the batched kernel

// (lo, mid, hi) += x * y
__device__ __forceinline__ void mac192(uint64_t& lo, uint64_t& mid, uint32_t& hi, uint64_t x,
                                       uint64_t y) {
    asm("mad.lo.cc.u64 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u64 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+l"(lo), "+l"(mid), "+r"(hi)
        : "l"(x), "l"(y));
}

// y + k 2^64 = lo + mid + hi  (k <= 2)
__device__ __forceinline__ void school_sum3(uint64_t lo, uint64_t mid, uint32_t hi, uint64_t& y,
                                            uint32_t& k) {
    const uint64_t s1 = lo + mid;
    k = s1 < lo;
    y = s1 + hi;
    k += y < s1;
}

// One product {a, an} * {b, bn} -> out[0 .. an+bn), an + bn <= SBG_SCHOOL_MAX,
// by one full warp; sa, sb: this warp's shared-memory staging (128 limbs each).
__device__ __forceinline__ void school_warp(const uint64_t* __restrict__ a, int an,
                                            const uint64_t* __restrict__ b, int bn,
                                            uint64_t* __restrict__ out, uint64_t* sa, uint64_t* sb) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < an; i += 32) sa[i] = __ldg(&a[i]);
    for (int i = lane; i < bn; i += 32) sb[i] = __ldg(&b[i]);
    __syncwarp();
    const int n = an + bn;                  // output limbs; columns 0 .. n-2
    const int steps = (n + 31) >> 5;
    // carried from the previous step: mid of column 32 s - 1, hi of columns
    // 32 s - 2 and 32 s - 1, the sum carry of limb 32 s - 1, the ripple carry
    uint64_t c_mid1 = 0;
    uint32_t c_hi2 = 0, c_hi1 = 0, c_k1 = 0, cin = 0;
    for (int s = 0; s < steps; ++s) {
        const int k = 32 * s + lane;
        uint64_t lo = 0, mid = 0;
        uint32_t hi = 0;
        // terms i in [max(0, k - bn + 1), min(k, an - 1)]; the warp walks the
        // union of its lanes' ranges, each lane masked to its own
        const int ilo = max(0, k - bn + 1), ihi = min(k, an - 1);
        const int wlo = __reduce_min_sync(FULL, (unsigned)(k < n - 1 ? ilo : an));
        const int whi = __reduce_max_sync(FULL, (unsigned)(k < n - 1 ? ihi + 1 : 0)) - 1;
        for (int i = wlo; i <= whi; ++i) {
            const uint64_t x = sa[i];
            const int j = k - i;
            const bool on = k < n - 1 && i >= ilo && i <= ihi;
            const uint64_t y = on ? sb[j < 0 ? 0 : (j >= bn ? bn - 1 : j)] : 0ull;
            mac192(lo, mid, hi, x, y);
        }
        // limb k before ripple carries: lo_k + mid_{k-1} + hi_{k-2} + (sum carry of limb k-1)
        const uint64_t u_mid = __shfl_up_sync(FULL, mid, 1);
        const uint32_t u_hi2 = __shfl_up_sync(FULL, hi, 2);
        const uint64_t b_mid1 = lane == 0 ? c_mid1 : u_mid;
        const uint32_t b_hi2 = lane == 0 ? c_hi2 : (lane == 1 ? c_hi1 : u_hi2);
        uint64_t y;
        uint32_t kk;
        school_sum3(lo, b_mid1, b_hi2, y, kk);
        const uint32_t u_k = __shfl_up_sync(FULL, kk, 1);
        const uint32_t b_k1 = lane == 0 ? c_k1 : u_k;
        const uint64_t z = y + b_k1;
        const uint32_t G = z < y, P = z == ~0ull;
        const uint32_t g = __ballot_sync(FULL, G), p = __ballot_sync(FULL, P);
        const uint64_t sum = (uint64_t)p + ((g << 1) | cin);
        const uint32_t c = (((uint32_t)sum ^ p) >> lane) & 1u;
        cin = (uint32_t)(sum >> 32) | (g >> 31);
        if (k < n) out[k] = z + c;
        c_mid1 = __shfl_sync(FULL, mid, 31);
        c_hi2 = __shfl_sync(FULL, hi, 30);
        c_hi1 = __shfl_sync(FULL, hi, 31);
        c_k1 = __shfl_sync(FULL, kk, 31);
    }
}

}  // namespace sbg
