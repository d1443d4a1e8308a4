// sbg_ntt.cuh -- on-chip NTT engine: radix-2^r register groups.
//
// Forward = radix-2 Gentleman-Sande DIF (natural-order input, bit-reversed
// output).  Its levels run r at a time on a "group": the 2^r points
//     blk*M + j0 + st*t,  t in [0, 2^r),  st = M / 2^r,
// held in registers.  Level l of a group pairs t with t + 2^(r-l-1) and uses
// the twiddle w_{M>>l}^(j0 + st*(t mod 2^(r-l))).
// Inverse = the exact reverse network (levels bottom-up, Cooley-Tukey
// butterflies with inverse twiddles): it returns S * x from the bit-reversed
// spectrum; the 1/S factors are folded into a later constant multiply.
//
// Twiddle tables are "per resolution": for every size S = 2 .. 2^13 the
// entries w_S^j, j < S/2, sit contiguously at index S/2 - 1 + j, each as
// (w, floor(w * 2^32 / p)).  A level's lanes (consecutive j0) therefore read
// consecutive entries: two L1 wavefronts per warp-wide load at every level.
//
// This plays the role of the reference's radix-8 "moths" and in-register
// bottoms (include/p30.h:418 p30_fwd8, :506 p30_inv8; include/p50.h:326,
// :366-450), re-organised for a CTA: the reference walks a depth-first tree
// over cache-resident blocks; here every level of a group runs on registers
// and groups exchange through shared memory or global memory.
#pragma once
#include "sbg_arith.cuh"

namespace sbg {

#define SBG_TW_LG 13                   // largest on-chip transform: 2^13 points
#define SBG_TW_N (1 << SBG_TW_LG)      // entries per (prime, direction) table

__device__ __forceinline__ int pad_idx(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int s) { return s + (s >> 4); }

// table index of w_{2^lgS}^pos
__device__ __forceinline__ int tw_idx(int lgS, int pos) { return (1 << (lgS - 1)) - 1 + pos; }

template <int R>
struct RLog {
    static constexpr int v = (R == 2) ? 1 : (R == 4) ? 2 : (R == 8) ? 3 : (R == 16) ? 4 : 5;
};

// forward DIF levels of one group (block size 2^lgM, stride st).  J0Z: the
// caller's j0 is 0, so the butterflies at tin = 0 have the twiddle 1 and
// skip the multiply (and the table load).
// HZ: the upper half of the inputs is zero (see dif_regs2).
template <int R, bool J0Z = false, bool HZ = false>
__device__ __forceinline__ void dif_regs(uint32_t (&x)[R], const uint2* __restrict__ tw, int j0,
                                         int st, int lgM, uint32_t p) {
    if constexpr (HZ) {
#pragma unroll
        for (int t = 0; t < R / 2; ++t) {
            uint2 w = __ldg(&tw[tw_idx(lgM, j0 + st * t)]);
            x[t + R / 2] = mul_shoup(x[t], w.x, w.y, p);
        }
    }
#pragma unroll
    for (int h = HZ ? R / 4 : R / 2, l = HZ ? 1 : 0; h >= 1; h >>= 1, ++l) {
#pragma unroll
        for (int t = 0; t < R; ++t) {
            if (t & h) continue;
            int tin = t & (2 * h - 1);
            if (J0Z && tin == 0) {
                bfly_triv(x[t], x[t + h], p);
                continue;
            }
            uint2 w = __ldg(&tw[tw_idx(lgM - l, j0 + st * tin)]);
            bfly_gs(x[t], x[t + h], w.x, w.y, p);
        }
    }
}

// two groups sharing (j0, st, lgM): one twiddle load serves both.  HZ: the
// upper half of both groups' inputs is zero (a zero-padded operand), so the
// first level is (u, 0) -> (u, u w): one multiply, no add or reduction.
template <int R, bool J0Z = false, bool HZ = false>
__device__ __forceinline__ void dif_regs2(uint32_t (&x)[R], uint32_t (&y)[R],
                                          const uint2* __restrict__ tw, int j0, int st, int lgM,
                                          uint32_t p) {
    if constexpr (HZ) {
#pragma unroll
        for (int t = 0; t < R / 2; ++t) {
            uint2 w = __ldg(&tw[tw_idx(lgM, j0 + st * t)]);
            x[t + R / 2] = mul_shoup(x[t], w.x, w.y, p);
            y[t + R / 2] = mul_shoup(y[t], w.x, w.y, p);
        }
    }
#pragma unroll
    for (int h = HZ ? R / 4 : R / 2, l = HZ ? 1 : 0; h >= 1; h >>= 1, ++l) {
#pragma unroll
        for (int t = 0; t < R; ++t) {
            if (t & h) continue;
            int tin = t & (2 * h - 1);
            if (J0Z && tin == 0) {
                bfly_triv(x[t], x[t + h], p);
                bfly_triv(y[t], y[t + h], p);
                continue;
            }
            uint2 w = __ldg(&tw[tw_idx(lgM - l, j0 + st * tin)]);
            bfly_gs(x[t], x[t + h], w.x, w.y, p);
            bfly_gs(y[t], y[t + h], w.x, w.y, p);
        }
    }
}

// inverse: the forward group's levels in reverse, Cooley-Tukey with w^-1
template <int R, bool J0Z = false>
__device__ __forceinline__ void dit_regs(uint32_t (&x)[R], const uint2* __restrict__ twi, int j0,
                                         int st, int lgM, uint32_t p) {
    constexpr int r = RLog<R>::v;
#pragma unroll
    for (int l = r - 1; l >= 0; --l) {
        const int h = R >> (l + 1);
#pragma unroll
        for (int t = 0; t < R; ++t) {
            if (t & h) continue;
            int tin = t & (2 * h - 1);
            if (J0Z && tin == 0) {
                bfly_triv(x[t], x[t + h], p);
                continue;
            }
            uint2 w = __ldg(&twi[tw_idx(lgM - l, j0 + st * tin)]);
            bfly_ct(x[t], x[t + h], w.x, w.y, p);
        }
    }
}

template <int R, bool J0Z = false>
__device__ __forceinline__ void dit_regs2(uint32_t (&x)[R], uint32_t (&y)[R],
                                          const uint2* __restrict__ twi, int j0, int st, int lgM,
                                          uint32_t p) {
    constexpr int r = RLog<R>::v;
#pragma unroll
    for (int l = r - 1; l >= 0; --l) {
        const int h = R >> (l + 1);
#pragma unroll
        for (int t = 0; t < R; ++t) {
            if (t & h) continue;
            int tin = t & (2 * h - 1);
            if (J0Z && tin == 0) {
                bfly_triv(x[t], x[t + h], p);
                bfly_triv(y[t], y[t + h], p);
                continue;
            }
            uint2 w = __ldg(&twi[tw_idx(lgM - l, j0 + st * tin)]);
            bfly_ct(x[t], x[t + h], w.x, w.y, p);
            bfly_ct(y[t], y[t + h], w.x, w.y, p);
        }
    }
}

// ---- generic shared-memory passes (single-CTA transforms) ---------------
// G transforms of 2^lgS points, transform g at buf + g * ld (padded index).
template <int R, bool FWD>
__device__ __forceinline__ void ntt_pass(uint32_t* buf, int ld, int G, int lgS, int lgM,
                                         const uint2* __restrict__ tw, uint32_t p) {
    constexpr int r = RLog<R>::v;
    const int lgst = lgM - r;
    const int st = 1 << lgst;
    const int lgper = lgS - r;                          // log2 groups per transform
    const int total = G << lgper;
    for (int gid = threadIdx.x; gid < total; gid += blockDim.x) {
        int g = gid >> lgper;
        int rem = gid & ((1 << lgper) - 1);
        int blk = rem >> lgst;
        int j0 = rem & (st - 1);
        uint32_t* base = buf + g * ld;
        int i0 = (blk << lgM) + j0;
        uint32_t x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = base[pad_idx(i0 + st * t)];
        if (FWD)
            dif_regs<R>(x, tw, j0, st, lgM, p);
        else
            dit_regs<R>(x, tw, j0, st, lgM, p);
#pragma unroll
        for (int t = 0; t < R; ++t) base[pad_idx(i0 + st * t)] = x[t];
    }
}

// Radix schedule: passes of 16 from the top, the remainder (1..3 levels) last.
__host__ __device__ constexpr int pass_radix_lg(int lgS, int k) {
    int full = lgS >> 2;
    return k < full ? 4 : (lgS & 3);
}
__host__ __device__ constexpr int num_passes(int lgS) {
    return (lgS >> 2) + ((lgS & 3) ? 1 : 0);
}

template <bool FWD>
__device__ __forceinline__ void ntt_pass_dispatch(int rlg, uint32_t* buf, int ld, int G, int lgS,
                                                  int lgM, const uint2* __restrict__ tw,
                                                  uint32_t p) {
    switch (rlg) {
        case 4: ntt_pass<16, FWD>(buf, ld, G, lgS, lgM, tw, p); break;
        case 3: ntt_pass<8, FWD>(buf, ld, G, lgS, lgM, tw, p); break;
        case 2: ntt_pass<4, FWD>(buf, ld, G, lgS, lgM, tw, p); break;
        case 1: ntt_pass<2, FWD>(buf, ld, G, lgS, lgM, tw, p); break;
        default: break;
    }
}

__device__ __forceinline__ void ntt_forward(uint32_t* buf, int ld, int G, int lgS,
                                            const uint2* __restrict__ tw, uint32_t p) {
    int np = num_passes(lgS);
    int lgM = lgS;
    for (int k = 0; k < np; ++k) {
        int rlg = pass_radix_lg(lgS, k);
        ntt_pass_dispatch<true>(rlg, buf, ld, G, lgS, lgM, tw, p);
        __syncthreads();
        lgM -= rlg;
    }
}

__device__ __forceinline__ void ntt_inverse(uint32_t* buf, int ld, int G, int lgS,
                                            const uint2* __restrict__ twi, uint32_t p) {
    int np = num_passes(lgS);
    for (int k = np - 1; k >= 0; --k) {
        int lgM = lgS;
        for (int kk = 0; kk < k; ++kk) lgM -= pass_radix_lg(lgS, kk);
        int rlg = pass_radix_lg(lgS, k);
        ntt_pass_dispatch<false>(rlg, buf, ld, G, lgS, lgM, twi, p);
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t bitrev(uint32_t x, int bits) {
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

// floor(w * 2^32 / p): the Shoup companion of a twiddle computed on the fly
__device__ __forceinline__ uint32_t shoup_of(uint32_t w, uint32_t p) {
    return (uint32_t)(((uint64_t)w << 32) / p);
}

}  // namespace sbg
