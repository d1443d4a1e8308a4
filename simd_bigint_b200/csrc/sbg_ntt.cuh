// sbg_ntt.cuh -- on-chip NTT engine: radix-2^r register passes over
// shared-memory arrays, used by every transform kernel.
//
// A transform of S = 2^s points lives in shared memory, one u32 per point,
// with one padding word per 16 points (index i is stored at i + i/16) so that
// the strided group loads below are bank-conflict free.  G independent
// transforms sit back to back (transform g at base + g * ld).
//
// Forward = radix-2 Gentleman-Sande DIF with natural-order input and
// bit-reversed output (the standard iterative network).  Its levels are
// executed r at a time: a "group" is the 2^r points
//     blk*M + j0 + st*t,  t in [0, 2^r),  st = M / 2^r,
// which stay in registers for r levels.  Level l of the group pairs t with
// t + 2^(r-l-1) and uses the twiddle w_{M>>l}^(j0 + st*(t mod 2^(r-l))).
// Inverse = the exact reverse network (passes in reverse order, levels
// bottom-up, Cooley-Tukey butterflies with inverse twiddles), which returns
// S * x from the bit-reversed spectrum; the 1/S factors are folded into the
// CRT scale.
//
// Twiddles come from ONE master table per prime and direction: entry e holds
// (w^e, floor(w^e * 2^32 / p)) for w a primitive 2^13-th root, e < 2^12.  A
// twiddle w_M^j is entry j << (13 - lg M).
//
// This plays the role of the reference's radix-8 "moths" and in-register
// bottoms (include/p30.h:418 p30_fwd8, :506 p30_inv8; include/p50.h:326,
// :366-450), re-organised for a CTA: the reference walks a depth-first tree
// over cache-resident blocks, here every level of a pass runs on registers
// and passes exchange through shared memory.
#pragma once
#include "sbg_arith.cuh"

namespace sbg {

#define SBG_TW_LG 13                     // master twiddle root order 2^13
#define SBG_TW_N (1 << (SBG_TW_LG - 1))  // entries per table (e < 2^12)

__device__ __forceinline__ int pad_idx(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int s) { return s + (s >> 4); }

// One forward group of R = 2^r points, in registers.
template <int R>
__device__ __forceinline__ void dif_group(uint32_t (&x)[R], const uint2* __restrict__ tw, int j0,
                                          int st, int sh, uint32_t p) {
#pragma unroll
    for (int h = R / 2, l = 0; h >= 1; h >>= 1, ++l) {
#pragma unroll
        for (int t = 0; t < R; ++t) {
            if (t & h) continue;
            int tin = t & (2 * h - 1);                  // index inside the sub-block
            int e = (j0 + st * tin) << (sh + l);
            uint2 w = __ldg(&tw[e]);
            bfly_gs(x[t], x[t + h], w.x, w.y, p);
        }
    }
}

// One inverse group (exact reverse of dif_group with inverse twiddles).
template <int R>
__device__ __forceinline__ void dit_group(uint32_t (&x)[R], const uint2* __restrict__ twi, int j0,
                                          int st, int sh, uint32_t p) {
#pragma unroll
    for (int h = 1; h <= R / 2; h <<= 1) {
        int lv = 0;
#pragma unroll
        for (int hh = R / 2; hh > h; hh >>= 1) ++lv;
#pragma unroll
        for (int t = 0; t < R; ++t) {
            if (t & h) continue;
            int tin = t & (2 * h - 1);
            int e = (j0 + st * tin) << (sh + lv);
            uint2 w = __ldg(&twi[e]);
            bfly_ct(x[t], x[t + h], w.x, w.y, p);
        }
    }
}

// Run one pass (radix R) over G transforms of size S = 2^lgS, block size
// M = 2^lgM, on shared memory `buf` (transform g at buf + g * ld).
template <int R, bool FWD>
__device__ __forceinline__ void ntt_pass(uint32_t* buf, int ld, int G, int lgS, int lgM,
                                         const uint2* __restrict__ tw, uint32_t p) {
    constexpr int r = (R == 2) ? 1 : (R == 4) ? 2 : (R == 8) ? 3 : (R == 16) ? 4 : 5;
    const int lgst = lgM - r;
    const int st = 1 << lgst;
    const int lgper = lgS - r;                          // log2 groups per transform
    const int total = G << lgper;
    const int sh = SBG_TW_LG - lgM;
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
            dif_group<R>(x, tw, j0, st, sh, p);
        else
            dit_group<R>(x, tw, j0, st, sh, p);
#pragma unroll
        for (int t = 0; t < R; ++t) base[pad_idx(i0 + st * t)] = x[t];
    }
}

// Radix schedule: passes of 16 from the top, the remainder (1..3 levels) last.
__device__ __forceinline__ int pass_radix_lg(int lgS, int k) {
    // k-th pass (0-based) of a transform of 2^lgS points
    int full = lgS >> 2;
    return k < full ? 4 : (lgS & 3);
}
__host__ __device__ __forceinline__ int num_passes(int lgS) { return (lgS >> 2) + ((lgS & 3) ? 1 : 0); }

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

// Full forward transform (all passes) of G transforms of 2^lgS points.
// Caller syncs before (data written) and after (data read).
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
    // block sizes of the forward passes, replayed backwards
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

}  // namespace sbg
