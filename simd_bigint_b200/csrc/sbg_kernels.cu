// sbg_kernels.cu -- the transform pipeline of one product on the GPU.
//
//   u64 limbs --(K1 k_col_fwd: residues + column DIF)-->
//   spectra   --(K2 k_row12: four-step twiddle, row DIF of A and B, pointwise,
//                row DIT, inverse twiddle x CRT scale)-->
//   products  --(K3 k_col_inv: column DIT)-->
//   residues  --(K4 k_crt_carry: Garner CRT + 3-stream compose + carry scan)--> limbs
//
// A length-L sequence is an N1 x 4096 matrix (N1 = L / 4096 rows, 2^a or
// 3 * 2^m): K1 / K3 transform its columns (tiles of adjacent columns, split
// over thread-block clusters when a column is long; k_col3* for 3 * 2^m
// rows), K2 its rows.  Transforms of L <= 2^12 points skip the four-step
// split and run whole in one CTA per prime (k_small).  This is the reference's p30 pipeline
// (include/p30.h:1847-1938: input -> forward -> fused pointwise+inverse ->
// scale -> Garner/carry), laid out as a four-step NTT over HBM: every pass
// reads and writes each spectrum once, all levels inside a pass stay on chip.
#include <cooperative_groups.h>

#include <algorithm>

#include "sbg_internal.h"
#include "sbg_ntt.cuh"

namespace cg = cooperative_groups;

namespace sbg {

__constant__ PrimeConst c_pr[SBG_NP];
__constant__ CrtConst c_crt;

#define SBG_ROW_LG 12
#define SBG_FS_LO_LG 13
#define SBG_FS_LO_N (1 << SBG_FS_LO_LG)

// ------------------------------------------------------------------------
// table generation
// ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pow_mod_dev(uint32_t b, uint32_t e, uint32_t p) {
    uint64_t r = 1, x = b;
    while (e) {
        if (e & 1) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

// out[q * n + e] = (root_q^(e * stride), shoup) for e < n
__global__ void k_gen_pow(uint2* out, int n, const uint32_t* roots, uint32_t stride) {
    int q = blockIdx.y;
    uint32_t p = c_pr[q].p;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        uint32_t w = pow_mod_dev(roots[q], (uint32_t)((uint64_t)e * stride % (p - 1)), p);
        uint32_t ws = (uint32_t)(((uint64_t)w << 32) / p);
        out[(size_t)q * n + e] = make_uint2(w, ws);
    }
}

// per-resolution table: out[q * 2^13 + (S/2 - 1 + j)] = (w_S^j, shoup), S = 2..2^13
__global__ void k_gen_res(uint2* out, const uint32_t* roots13) {
    int q = blockIdx.y;
    uint32_t p = c_pr[q].p;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < SBG_TW_N - 1;
         idx += gridDim.x * blockDim.x) {
        int lgS = 32 - __clz(idx + 1);                 // S/2 - 1 <= idx < S - 1
        int j = idx - ((1 << (lgS - 1)) - 1);
        uint32_t e = (uint32_t)j << (SBG_TW_LG - lgS);
        uint32_t w = pow_mod_dev(roots13[q], e, p);
        out[(size_t)q * SBG_TW_N + idx] = make_uint2(w, shoup_of(w, p));
    }
}

// ------------------------------------------------------------------------
// K0: single-CTA product for L <= 2^12 (one CTA per prime)
// ------------------------------------------------------------------------
__device__ __forceinline__ void small_body(int q, const uint64_t* __restrict__ a, int64_t an,
                                           const uint64_t* __restrict__ b, int64_t bn, int sq,
                                           int lgL, const uint2* __restrict__ twf,
                                           const uint2* __restrict__ twi, const ScaleArg& sc,
                                           uint32_t* __restrict__ R) {
    extern __shared__ uint32_t sm[];
    const PrimeConst pc = c_pr[q];
    const int L = 1 << lgL;
    const int ld = padded_len(L);
    uint32_t* A = sm;
    uint32_t* B = sm + ld;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        A[pad_idx(i)] = i < an ? limb_residue(a[i], pc) : 0u;
        if (!sq) B[pad_idx(i)] = i < bn ? limb_residue(b[i], pc) : 0u;
    }
    __syncthreads();
    ntt_forward(sm, ld, sq ? 1 : 2, lgL, twf + q * SBG_TW_N, pc.p);
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        uint32_t x = A[pad_idx(i)];
        uint32_t y = sq ? x : B[pad_idx(i)];
        A[pad_idx(i)] = mul_shoup(mont_mul(x, y, pc.p, pc.pinv), sc.w[q], sc.ws[q], pc.p);
    }
    __syncthreads();
    ntt_inverse(sm, ld, 1, lgL, twi + q * SBG_TW_N, pc.p);
    for (int i = threadIdx.x; i < L; i += blockDim.x) R[(size_t)q * L + i] = A[pad_idx(i)];
}

__global__ void __launch_bounds__(256) k_small(const uint64_t* __restrict__ a, int64_t an,
                                               const uint64_t* __restrict__ b, int64_t bn, int sq,
                                               int lgL, const uint2* __restrict__ twf,
                                               const uint2* __restrict__ twi, ScaleArg sc,
                                               uint32_t* __restrict__ R) {
    small_body(blockIdx.x, a, an, b, bn, sq, lgL, twf, twi, sc, R);
}

// batched: one CTA per (job, prime); every job of the launch has length 2^lgL
__global__ void __launch_bounds__(256) k_small_b(const JobDesc* __restrict__ jobs, int lgL,
                                                 const uint2* __restrict__ twf,
                                                 const uint2* __restrict__ twi, ScaleArg sc) {
    const JobDesc& J = jobs[blockIdx.x / SBG_NP];
    small_body(blockIdx.x % SBG_NP, J.a, J.an, J.b, J.bn, J.sq, lgL, twf, twi, sc, J.ws);
}

// ------------------------------------------------------------------------
// Four-step layout: the length-L sequence is an N1 x N2 row-major matrix
// (n = n1*N2 + n2).  K1 runs the column DIFs, K2 the row DIFs (after the
// four-step twiddle w_L^(k1*n2)), the pointwise product and the row DITs
// (followed by the inverse twiddle and the CRT scale), K3 the column DITs.
// ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t fs_value(const FsTables& fs, int q, uint32_t e, uint32_t p) {
    uint2 a = __ldg(&fs.lo[(size_t)q * SBG_FS_LO_N + (e & (SBG_FS_LO_N - 1))]);
    uint2 b = __ldg(&fs.hi[(size_t)q * fs.hi_n + (e >> SBG_FS_LO_LG)]);
    return mul_shoup(a.x, b.x, b.y, p);
}

// Column tiles.  A CTA owns W adjacent columns of one operand and one prime
// over a slab of M rows (M * W = 2^13 points, fewer when the whole transform
// is smaller).  Two thread mappings:
//  * lane per column (columns of at most 2^8 rows, W >= 32): a warp covers 32
//    adjacent columns of one group, so every global access of a warp is one
//    128-byte row piece (256 for limbs), each level's twiddle is one
//    broadcast load, and the columns live in shared memory as planes of M + 1
//    words (odd stride: the 32 lanes hit 32 distinct banks);
//  * column pairs (longer columns, M up to 2^10, W = 2^13 / M): a thread owns
//    two adjacent columns of one group, so one twiddle load serves two
//    butterflies and the global accesses are 16-byte (two limbs) or 8-byte
//    (two residues) row pieces.  The pair's two columns sit side by side in
//    shared memory (one 8-byte word per row, planes padded one word per
//    16 rows), so every shared-memory and distributed-shared-memory access
//    moves both columns in one 64-bit instruction.
// Columns of more than 2^10 rows (transform lengths 2^23..2^25) are split
// over a thread-block cluster of C = N1 / 2^10 CTAs, one slab of 2^10 rows
// each, exchanging through distributed shared memory: the top lg C DIF levels
// pair rows r + 2^10 t across the slabs.  Forward: each CTA reads the C rows
// of its share of those groups from global memory, runs the lg C levels in
// registers and stores each result into the shared memory of the CTA that
// owns its slab; after a cluster barrier every CTA transforms its slab (an
// independent 2^10-point DIF per column) and writes it out.  The inverse runs
// the same network backwards.  The in-place result is the one a single CTA
// holding the whole column would produce.  (Measured on B200 at 2^25 points:
// 256-thread CTAs, four per SM, beat 512-thread ones; slabs of 2^8 or 2^9
// rows need clusters of 16 whose shared-memory exchange costs more than the
// wider rows save; lane-per-column wins where no exchange is needed.)
#define SBG_COL_SLAB_LG 10
#ifndef SBG_COL_TILE_LG
#define SBG_COL_TILE_LG 13        // points per CTA (log2)
#endif
#define SBG_COL_LANE_MAX_LG 8
#define COL_THREADS 256
// resident CTAs per SM the register budget is set for: forward columns 5
// (48 registers; their cross-slab loads wait longest, and more CTAs hide
// them: 2^25 points 1.28 -> 1.21 ms against 4), inverse columns 4 (64
// registers; at 5 they spill and slow down)
#ifndef COL_MINB
#define COL_MINB 4
#endif
#ifndef COL_FWD_MINB
#define COL_FWD_MINB 5
#endif
#ifndef COL3_FWD_MINB
#define COL3_FWD_MINB COL_MINB
#endif
__host__ __device__ constexpr bool col_lanes(int lgN1) { return lgN1 <= SBG_COL_LANE_MAX_LG; }
__host__ __device__ constexpr int col_lgc(int lgN1) {
    return lgN1 > SBG_COL_SLAB_LG ? lgN1 - SBG_COL_SLAB_LG : 0;
}
__host__ __device__ constexpr int col_lgs(int lgN1) { return lgN1 - col_lgc(lgN1); }
__host__ __device__ constexpr int col_lgw_of(bool lanes, int lgs) {
    return (SBG_COL_TILE_LG - lgs) > 12 ? 12
                                         : ((lanes && SBG_COL_TILE_LG - lgs < 5) ? 5 : SBG_COL_TILE_LG - lgs);
}
__host__ __device__ constexpr int col_lgw(int lgN1) { return col_lgw_of(col_lanes(lgN1), col_lgs(lgN1)); }
// single-CTA 3 * 2^m columns (m <= SBG_COL3S_MAX): W = 2^(12 - m) columns of 3 * 2^m rows
#define SBG_COL3S_MAX 7
__host__ __device__ constexpr int col3s_lgw(int m) { return 12 - m; }
// Plane strides: lanes, M + 1 words (odd); pairs, padded length + 32/W
// 8-byte words, so that each half-warp's W/2 column pairs x 32/W consecutive
// rows (a 64-bit access is served half a warp at a time) fall in distinct
// bank pairs.
__host__ __device__ constexpr int col_ld_of(bool lanes, int lgs) {
    return lanes ? (1 << lgs) + 1 : padded_len(1 << lgs) + (32 >> col_lgw_of(false, lgs));
}
__host__ __device__ constexpr int col_ld(int lgN1) { return col_ld_of(col_lanes(lgN1), col_lgs(lgN1)); }
// Column radix schedule: passes of 16 from the top, the remainder (1..3
// levels) last.  (A radix-32 last pass spills under the 64-register cap, and
// the remainder first costs an extra shared-memory round trip; both were
// slower on B200.)
__host__ __device__ constexpr int col_np(int lg) { return num_passes(lg); }
// rf: the remainder pass first instead of last (the slabs of clustered
// columns: the inverse then reads global memory with a radix-16 pass)
__host__ __device__ constexpr int prl(int lg, int k, bool rf = false) {
    return (rf && (lg & 3)) ? (k == 0 ? (lg & 3) : 4) : (k < (lg >> 2) ? 4 : (lg & 3));
}
__host__ __device__ constexpr int lgm_of(int lg, int k, bool rf = false) {
    int m = lg;
    for (int i = 0; i < k; ++i) m -= prl(lg, i, rf);
    return m;
}
__host__ __device__ constexpr int col_smem_bytes(int lgN1) {
    return (col_np(col_lgs(lgN1)) > 1 || col_lgc(lgN1) > 0)
               ? (1 << col_lgw(lgN1)) * col_ld(lgN1) * 4
               : 0;
}
__host__ __device__ constexpr int col_ntiles(int lgN1) { return 1 << (SBG_ROW_LG - col_lgw(lgN1)); }

template <int LGST>
__device__ __forceinline__ int padded_at(int i0, int t) {
    constexpr int ST = 1 << LGST;
    if constexpr (LGST >= 4) {
        return pad_idx(i0) + t * (ST + (ST >> 4));
    } else {
        return pad_idx(i0 + ST * t);
    }
}

// Operand limbs and residue rows stream through a CTA once: they are loaded
// L2-only (ld.global.cg) so that they do not evict the twiddle tables, which
// every pass re-reads, from L1.
//
// two limbs of row n (columns c, c+1) -> residues; zero beyond xn
__device__ __forceinline__ void load_limb_pair(const uint64_t* __restrict__ X, int64_t xn, int64_t n,
                                               bool al16, const PrimeConst& pc, uint32_t& x,
                                               uint32_t& y) {
    if (al16 && n + 1 < xn) {
        ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(X + n));
        x = limb_residue(v.x, pc);
        y = limb_residue(v.y, pc);
    } else {
        x = n < xn ? limb_residue(__ldcg(&X[n]), pc) : 0u;
        y = n + 1 < xn ? limb_residue(__ldcg(&X[n + 1]), pc) : 0u;
    }
}

// Pass K (0-based, forward numbering) of the DIF/DIT of length 2^LGS on the
// slab whose first row is row0.  SRC_G: read from global (limbs when FWD,
// residues otherwise); DST_G: write residues to global; else shared memory.
template <int LGS, int K, bool FWD, bool SRC_G, bool DST_G, bool RF = false>
__device__ __forceinline__ void col_pass_pair(uint32_t* sm, const uint64_t* __restrict__ X,
                                           int64_t xn, uint32_t* __restrict__ Y, int c0, int row0,
                                           const uint2* __restrict__ tw, const PrimeConst& pc) {
    constexpr int r = prl(LGS, K, RF);
    constexpr int R = 1 << r;
    constexpr int LGM = lgm_of(LGS, K, RF);
    constexpr int LGST = LGM - r;
    constexpr int ST = 1 << LGST;
    constexpr int LGW = col_lgw_of(false, LGS);
    constexpr int LD = col_ld_of(false, LGS);
    constexpr int TOTAL = (1 << (LGW - 1)) << (LGS - r);
    const uint32_t p = pc.p;
    // groups per thread is a compile-time constant (TOTAL / COL_THREADS, or 1
    // when the tile has fewer groups than threads): unrolled, so every
    // group's global loads are in flight together
    constexpr int ITER = TOTAL >= COL_THREADS ? TOTAL / COL_THREADS : 1;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int gid = threadIdx.x + it * COL_THREADS;
        if (TOTAL < COL_THREADS && gid >= TOTAL) break;
        // column pairs of a row fastest: a warp covers W/2 pairs x 64/W rows,
        // few row pieces per global access, and in the planes (stride
        // padded length + 32/W) its accesses fall in distinct banks for the
        // radix-16 passes (consecutive groups fastest would put 32
        // consecutive rows across a padding step: two-way conflicts)
        const int cp = gid & ((1 << (LGW - 1)) - 1);
        const int rest = gid >> (LGW - 1);
        const int j0 = rest & (ST - 1);
        const int blk = rest >> LGST;
        const int i0 = (blk << LGM) + j0;
        const int g0 = 2 * cp;
        uint32_t x[R], y[R];
        // first forward pass of a zero-padded operand: its upper half rows are empty
        bool hz = false;
        if constexpr (SRC_G) {
            const int64_t n0 = ((int64_t)(i0 + row0) << SBG_ROW_LG) + c0 + g0;
            if constexpr (FWD) {
                const bool al16 = (reinterpret_cast<uintptr_t>(X) & 15) == 0;
                if constexpr (K == 0 && R >= 2) hz = n0 + ((int64_t)(ST * (R / 2)) << SBG_ROW_LG) >= xn;
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    if (hz && t >= R / 2) break;
                    load_limb_pair(X, xn, n0 + ((int64_t)(ST * t) << SBG_ROW_LG), al16, pc, x[t], y[t]);
                }
            } else {
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    const int64_t n = n0 + ((int64_t)(ST * t) << SBG_ROW_LG);
                    uint2 v = __ldcg(reinterpret_cast<const uint2*>(Y + n));
                    x[t] = v.x;
                    y[t] = v.y;
                }
            }
        } else {
            const uint2* s0 = reinterpret_cast<const uint2*>(sm) + cp * LD;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const uint2 v = s0[padded_at<LGST>(i0, t)];
                x[t] = v.x;
                y[t] = v.y;
            }
        }
        if constexpr (FWD && SRC_G && K == 0) {
            if (hz)
                dif_regs2<R, ST == 1, true>(x, y, tw, j0, ST, LGM, p);
            else
                dif_regs2<R, ST == 1>(x, y, tw, j0, ST, LGM, p);
        } else if constexpr (FWD) {
            dif_regs2<R, ST == 1>(x, y, tw, j0, ST, LGM, p);
        } else {
            dit_regs2<R, ST == 1>(x, y, tw, j0, ST, LGM, p);
        }
        if constexpr (DST_G) {
            const int64_t n0 = ((int64_t)(i0 + row0) << SBG_ROW_LG) + c0 + g0;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int64_t n = n0 + ((int64_t)(ST * t) << SBG_ROW_LG);
                *reinterpret_cast<uint2*>(Y + n) = make_uint2(x[t], y[t]);
            }
        } else {
            uint2* s0 = reinterpret_cast<uint2*>(sm) + cp * LD;
#pragma unroll
            for (int t = 0; t < R; ++t) s0[padded_at<LGST>(i0, t)] = make_uint2(x[t], y[t]);
        }
    }
}

__device__ __forceinline__ uint32_t load_limb(const uint64_t* __restrict__ X, int64_t xn, int64_t n,
                                              const PrimeConst& pc) {
    return n < xn ? limb_residue(__ldcg(&X[n]), pc) : 0u;
}

// Pass K of the lane-per-column mapping (a warp = 32 adjacent columns of one
// group, one column per lane).  NSUB = 3: three 2^LGS-row slabs stacked in
// the planes (the thirds of a 3 * 2^m column held by one CTA), transformed
// independently.
template <int LGS, int K, bool FWD, bool SRC_G, bool DST_G, int NSUB = 1, bool RF = false>
__device__ __forceinline__ void col_pass_lane(uint32_t* sm, const uint64_t* __restrict__ X,
                                           int64_t xn, uint32_t* __restrict__ Y, int c0, int row0,
                                           const uint2* __restrict__ tw, const PrimeConst& pc) {
    constexpr int r = prl(LGS, K, RF);
    constexpr int R = 1 << r;
    constexpr int LGM = lgm_of(LGS, K, RF);
    constexpr int LGST = LGM - r;
    constexpr int ST = 1 << LGST;
    constexpr int LGW = NSUB == 1 ? col_lgw_of(true, LGS) : col3s_lgw(LGS);
    constexpr int LD = NSUB == 1 ? col_ld_of(true, LGS) : NSUB * (1 << LGS) + 1;
    constexpr int LGT1 = LGW + LGS - r;              // (column, group) pairs per slab
    constexpr int TOTAL = NSUB << LGT1;
    const uint32_t p = pc.p;
    constexpr int ITER = TOTAL >= COL_THREADS ? TOTAL / COL_THREADS : 1;
    // bounded unrolling: at most two radix-16 groups, eight short ones in flight
    constexpr int UNR = R >= 16 ? (ITER > 2 ? 1 : ITER) : (ITER > 8 ? 8 : ITER);
#pragma unroll UNR
    for (int it = 0; it < ITER; ++it) {
        const int gid = threadIdx.x + it * COL_THREADS;
        if (TOTAL < COL_THREADS && gid >= TOTAL) break;
        const int g = gid & ((1 << LGT1) - 1);
        const int col = g & ((1 << LGW) - 1);
        const int grp = g >> LGW;
        const int j0 = grp & (ST - 1);
        const int i0 = ((gid >> LGT1) << LGS) + ((grp >> LGST) << LGM) + j0;
        uint32_t x[R];
        // first forward pass of a zero-padded operand: its upper half rows are empty
        bool hz = false;
        if constexpr (SRC_G) {
            const int64_t n0 = ((int64_t)(i0 + row0) << SBG_ROW_LG) + c0 + col;
            if constexpr (FWD && K == 0 && NSUB == 1) hz = n0 + ((int64_t)(ST * (R / 2)) << SBG_ROW_LG) >= xn;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                if (hz && t >= R / 2) break;
                const int64_t n = n0 + ((int64_t)(ST * t) << SBG_ROW_LG);
                if constexpr (FWD)
                    x[t] = load_limb(X, xn, n, pc);
                else
                    x[t] = __ldcg(&Y[n]);
            }
        } else {
            const uint32_t* s0 = sm + col * LD + i0;
#pragma unroll
            for (int t = 0; t < R; ++t) x[t] = s0[ST * t];
        }
        if constexpr (FWD && SRC_G && K == 0 && NSUB == 1) {
            if (hz)
                dif_regs<R, ST == 1, true>(x, tw, j0, ST, LGM, p);
            else
                dif_regs<R, ST == 1>(x, tw, j0, ST, LGM, p);
        } else if constexpr (FWD) {
            dif_regs<R, ST == 1>(x, tw, j0, ST, LGM, p);
        } else {
            dit_regs<R, ST == 1>(x, tw, j0, ST, LGM, p);
        }
        if constexpr (DST_G) {
            const int64_t n0 = ((int64_t)(i0 + row0) << SBG_ROW_LG) + c0 + col;
#pragma unroll
            for (int t = 0; t < R; ++t) Y[n0 + ((int64_t)(ST * t) << SBG_ROW_LG)] = x[t];
        } else {
            uint32_t* s0 = sm + col * LD + i0;
#pragma unroll
            for (int t = 0; t < R; ++t) s0[ST * t] = x[t];
        }
    }
}

// Pass K (0-based, forward numbering) of the DIF/DIT of length 2^LGS on the
// slab whose first row is row0, in the mapping LANES selects.  SRC_G: read
// from global (limbs when FWD, residues otherwise); DST_G: write residues to
// global; else shared memory.
template <bool LANES, int LGS, int K, bool FWD, bool SRC_G, bool DST_G, int NSUB = 1, bool RF = false>
__device__ __forceinline__ void col_pass_t(uint32_t* sm, const uint64_t* __restrict__ X,
                                           int64_t xn, uint32_t* __restrict__ Y, int c0, int row0,
                                           const uint2* __restrict__ tw, const PrimeConst& pc) {
    if constexpr (LANES) {
        col_pass_lane<LGS, K, FWD, SRC_G, DST_G, NSUB, RF>(sm, X, xn, Y, c0, row0, tw, pc);
    } else {
        static_assert(NSUB == 1, "stacked slabs use the lane mapping");
        col_pass_pair<LGS, K, FWD, SRC_G, DST_G, RF>(sm, X, xn, Y, c0, row0, tw, pc);
    }
}

// The local passes of a slab: forward K = 0 .. NP-1, inverse NP-1 .. 0.
// FIRST_G / LAST_G: whether the first / last pass touches global memory.
template <bool LANES, int LGS, bool FIRST_G, bool LAST_G, int NSUB = 1, bool RF = false>
__device__ __forceinline__ void col_slab_fwd(uint32_t* sm, const uint64_t* __restrict__ X, int64_t xn,
                                             uint32_t* __restrict__ Y, int c0, int row0,
                                             const uint2* __restrict__ tw, const PrimeConst& pc) {
    constexpr int NP = col_np(LGS);
    col_pass_t<LANES, LGS, 0, true, FIRST_G, LAST_G && NP == 1, NSUB, RF>(sm, X, xn, Y, c0, row0, tw, pc);
    if constexpr (NP > 1) {
        __syncthreads();
        col_pass_t<LANES, LGS, 1, true, false, LAST_G && NP == 2, NSUB, RF>(sm, X, xn, Y, c0, row0, tw, pc);
    }
    if constexpr (NP > 2) {
        __syncthreads();
        col_pass_t<LANES, LGS, 2, true, false, LAST_G && NP == 3, NSUB, RF>(sm, X, xn, Y, c0, row0, tw, pc);
    }
    if constexpr (NP > 3) {
        __syncthreads();
        col_pass_t<LANES, LGS, 3, true, false, LAST_G && NP == 4, NSUB, RF>(sm, X, xn, Y, c0, row0, tw, pc);
    }
}

template <bool LANES, int LGS, bool FIRST_G, bool LAST_G, int NSUB = 1, bool RF = false>
__device__ __forceinline__ void col_slab_inv(uint32_t* sm, uint32_t* __restrict__ Y, int c0, int row0,
                                             const uint2* __restrict__ tw, const PrimeConst& pc) {
    constexpr int NP = col_np(LGS);
    if constexpr (NP > 3) {
        col_pass_t<LANES, LGS, 3, false, FIRST_G, false, NSUB, RF>(sm, nullptr, 0, Y, c0, row0, tw, pc);
        __syncthreads();
    }
    if constexpr (NP > 2) {
        col_pass_t<LANES, LGS, 2, false, FIRST_G && NP == 3, false, NSUB, RF>(sm, nullptr, 0, Y, c0, row0, tw, pc);
        __syncthreads();
    }
    if constexpr (NP > 1) {
        col_pass_t<LANES, LGS, 1, false, FIRST_G && NP == 2, false, NSUB, RF>(sm, nullptr, 0, Y, c0, row0, tw, pc);
        __syncthreads();
    }
    col_pass_t<LANES, LGS, 0, false, FIRST_G && NP == 1, LAST_G, NSUB, RF>(sm, nullptr, 0, Y, c0, row0, tw, pc);
}

// clustered columns: slab passes with the remainder first (0: last)
#ifndef SBG_COL_REMFIRST
#define SBG_COL_REMFIRST 1
#endif

// cluster barrier; RELEASE publishes this CTA's shared-memory stores (local
// and remote) to the cluster, otherwise it only waits for every CTA to arrive
template <bool RELEASE>
__device__ __forceinline__ void cluster_barrier() {
    if constexpr (RELEASE)
        asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    else
        asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Distributed shared memory by explicit shared::cluster accesses: the
// address of this CTA's shared word p in the shared memory of cluster CTA
// `rank`, and 64-bit stores and loads there.
__device__ __forceinline__ uint32_t dsmem_addr(const void* p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n"
                 : "=r"(r)
                 : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))), "r"(rank));
    return r;
}
__device__ __forceinline__ void dsmem_st2(uint32_t a, uint32_t x, uint32_t y) {
    asm volatile("st.shared::cluster.v2.u32 [%0], {%1, %2};\n" ::"r"(a), "r"(x), "r"(y) : "memory");
}
__device__ __forceinline__ uint2 dsmem_ld2(uint32_t a) {
    uint2 v;
    asm volatile("ld.shared::cluster.v2.u32 {%0, %1}, [%2];\n" : "=r"(v.x), "=r"(v.y) : "r"(a) : "memory");
    return v;
}

// Cluster levels (forward): this CTA's share of the radix-C groups
// {r + M t : t < C}, rows r in [slab * M / C, (slab + 1) * M / C) of every
// column pair, read from global, DIF'd, and scattered into the owning slabs.
template <int LGN1>
__device__ __forceinline__ void col_cross_fwd(uint32_t* sm, const uint64_t* __restrict__ X, int64_t xn,
                                              int c0, int slab, const uint2* __restrict__ tw,
                                              const PrimeConst& pc) {
    constexpr int LGC = col_lgc(LGN1);
    constexpr int C = 1 << LGC;
    constexpr int LGS = col_lgs(LGN1);
    constexpr int M = 1 << LGS;
    constexpr int LGW = col_lgw(LGN1);
    constexpr int LD = col_ld(LGN1);
    constexpr int RPS = M >> LGC;
    constexpr int TOTAL = RPS << (LGW - 1);
    static_assert(TOTAL % COL_THREADS == 0, "cluster groups must fill the CTA");
    constexpr int ITER = TOTAL / COL_THREADS;
    const bool al16 = (reinterpret_cast<uintptr_t>(X) & 15) == 0;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int gid = threadIdx.x + it * COL_THREADS;
        const int cp = gid & ((1 << (LGW - 1)) - 1);
        const int r = slab * RPS + (gid >> (LGW - 1));
        uint32_t x[C], y[C];
        const int64_t n0 = ((int64_t)r << SBG_ROW_LG) + c0 + 2 * cp;
        // a zero-padded operand (the usual case: an operand of at most half
        // the transform) has nothing in rows r + M t, t >= C / 2
        if (n0 + ((int64_t)(M * (C / 2)) << SBG_ROW_LG) >= xn) {
#pragma unroll
            for (int t = 0; t < C / 2; ++t)
                load_limb_pair(X, xn, n0 + ((int64_t)(M * t) << SBG_ROW_LG), al16, pc, x[t], y[t]);
            dif_regs2<C, false, true>(x, y, tw, r, M, LGN1, pc.p);
        } else {
#pragma unroll
            for (int t = 0; t < C; ++t)
                load_limb_pair(X, xn, n0 + ((int64_t)(M * t) << SBG_ROW_LG), al16, pc, x[t], y[t]);
            dif_regs2<C>(x, y, tw, r, M, LGN1, pc.p);
        }
        const uint2* a = reinterpret_cast<const uint2*>(sm) + cp * LD + pad_idx(r);
#pragma unroll
        for (int t = 0; t < C; ++t) dsmem_st2(dsmem_addr(a, t), x[t], y[t]);
    }
}

// Cluster levels (inverse): gather the C slabs' rows r + M t from their
// CTAs' shared memory, DIT, and write them to global memory.
template <int LGN1>
__device__ __forceinline__ void col_cross_inv(uint32_t* sm, uint32_t* __restrict__ Y, int c0, int slab,
                                              const uint2* __restrict__ tw, const PrimeConst& pc) {
    constexpr int LGC = col_lgc(LGN1);
    constexpr int C = 1 << LGC;
    constexpr int LGS = col_lgs(LGN1);
    constexpr int M = 1 << LGS;
    constexpr int LGW = col_lgw(LGN1);
    constexpr int LD = col_ld(LGN1);
    constexpr int RPS = M >> LGC;
    constexpr int TOTAL = RPS << (LGW - 1);
    static_assert(TOTAL % COL_THREADS == 0, "cluster groups must fill the CTA");
    constexpr int ITER = TOTAL / COL_THREADS;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int gid = threadIdx.x + it * COL_THREADS;
        const int cp = gid & ((1 << (LGW - 1)) - 1);
        const int r = slab * RPS + (gid >> (LGW - 1));
        uint32_t x[C], y[C];
        const uint2* a = reinterpret_cast<const uint2*>(sm) + cp * LD + pad_idx(r);
#pragma unroll
        for (int t = 0; t < C; ++t) {
            const uint2 v = dsmem_ld2(dsmem_addr(a, t));
            x[t] = v.x;
            y[t] = v.y;
        }
        dit_regs2<C>(x, y, tw, r, M, LGN1, pc.p);
        const int64_t n0 = ((int64_t)r << SBG_ROW_LG) + c0 + 2 * cp;
#pragma unroll
        for (int t = 0; t < C; ++t)
            *reinterpret_cast<uint2*>(Y + n0 + ((int64_t)(M * t) << SBG_ROW_LG)) = make_uint2(x[t], y[t]);
    }
}

// K1: limbs -> residues -> column DIF (bit-reversed rows) for one operand,
// one prime, one tile (one slab of it when the column spans a cluster).
template <int LGN1>
__device__ __forceinline__ void col_fwd_body(int q, int tile, int slab, int op,
                                             const uint64_t* __restrict__ a, int64_t an,
                                             const uint64_t* __restrict__ b, int64_t bn,
                                             const uint2* __restrict__ twf,
                                             uint32_t* __restrict__ YA,
                                             uint32_t* __restrict__ YB) {
    extern __shared__ uint32_t sm[];
    constexpr int LGC = col_lgc(LGN1);
    constexpr int LGS = col_lgs(LGN1);
    const uint64_t* X = op ? b : a;
    const int64_t xn = op ? bn : an;
    uint32_t* Y = (op ? YB : YA) + ((size_t)q << (LGN1 + SBG_ROW_LG));
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twf + (size_t)q * SBG_TW_N;
    const int c0 = tile << col_lgw(LGN1);
    if constexpr (LGC == 0) {
        col_slab_fwd<col_lanes(LGN1), LGS, true, true>(sm, X, xn, Y, c0, 0, tw, pc);
    } else {
        cluster_barrier<false>();       // every CTA of the cluster is running
        col_cross_fwd<LGN1>(sm, X, xn, c0, slab, tw, pc);
        cluster_barrier<true>();        // all slabs complete in shared memory
        col_slab_fwd<col_lanes(LGN1), LGS, false, true, 1, SBG_COL_REMFIRST != 0>(sm, X, xn, Y, c0, slab << LGS,
                                                                                  tw, pc);
    }
}

// Block order: cluster slab fastest, then prime, so the five primes' CTAs of
// one tile run together and share its limbs through L2.
template <int LGN1>
__global__ void __launch_bounds__(COL_THREADS, COL_FWD_MINB) k_col_fwd(const uint64_t* __restrict__ a, int64_t an,
                                                    const uint64_t* __restrict__ b, int64_t bn,
                                                    const uint2* __restrict__ twf,
                                                    uint32_t* __restrict__ YA,
                                                    uint32_t* __restrict__ YB, int nops) {
    constexpr int LGC = col_lgc(LGN1);
    constexpr int NTILES = col_ntiles(LGN1);
    const int slab = blockIdx.x & ((1 << LGC) - 1);
    int rest = blockIdx.x >> LGC;
    const int q = rest % SBG_NP;
    rest /= SBG_NP;
    col_fwd_body<LGN1>(q, rest % NTILES, slab, rest / NTILES, a, an, b, bn, twf, YA, YB);
}

// batched: blocks (job, operand, tile, prime, slab), job slowest; the second
// operand's blocks of a squaring exit at once (whole clusters together)
template <int LGN1>
__global__ void __launch_bounds__(COL_THREADS, COL_FWD_MINB) k_col_fwd_b(const JobDesc* __restrict__ jobs,
                                                      const uint2* __restrict__ twf) {
    constexpr int LGC = col_lgc(LGN1);
    constexpr int NTILES = col_ntiles(LGN1);
    constexpr int PER_JOB = (SBG_NP * 2 * NTILES) << LGC;
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    const int slab = r & ((1 << LGC) - 1);
    int rest = r >> LGC;
    const int q = rest % SBG_NP;
    rest /= SBG_NP;
    const int op = rest / NTILES;
    if (op && J.sq) return;
    uint32_t* YB = J.ws + ((size_t)SBG_NP << (LGN1 + SBG_ROW_LG));
    col_fwd_body<LGN1>(q, rest % NTILES, slab, op, J.a, J.an, J.b, J.bn, twf, J.ws, YB);
}

// K3: column DIT (reverse of K1), in place, natural row order out.
template <int LGN1>
__device__ __forceinline__ void col_inv_body(int q, int tile, int slab, uint32_t* __restrict__ YA,
                                             const uint2* __restrict__ twi) {
    extern __shared__ uint32_t sm[];
    constexpr int LGC = col_lgc(LGN1);
    constexpr int LGS = col_lgs(LGN1);
    uint32_t* Y = YA + ((size_t)q << (LGN1 + SBG_ROW_LG));
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twi + (size_t)q * SBG_TW_N;
    const int c0 = tile << col_lgw(LGN1);
    if constexpr (LGC == 0) {
        col_slab_inv<col_lanes(LGN1), LGS, true, true>(sm, Y, c0, 0, tw, pc);
    } else {
        col_slab_inv<col_lanes(LGN1), LGS, true, false, 1, SBG_COL_REMFIRST != 0>(sm, Y, c0, slab << LGS, tw, pc);
        cluster_barrier<true>();        // all slabs complete in shared memory
        col_cross_inv<LGN1>(sm, Y, c0, slab, tw, pc);
        cluster_barrier<false>();       // peers read this CTA's slab until here
    }
}

template <int LGN1>
__global__ void __launch_bounds__(COL_THREADS, COL_MINB) k_col_inv(uint32_t* __restrict__ YA,
                                                    const uint2* __restrict__ twi) {
    constexpr int LGC = col_lgc(LGN1);
    const int slab = blockIdx.x & ((1 << LGC) - 1);
    const int rest = blockIdx.x >> LGC;
    col_inv_body<LGN1>(rest % SBG_NP, rest / SBG_NP, slab, YA, twi);
}

template <int LGN1>
__global__ void __launch_bounds__(COL_THREADS, COL_MINB) k_col_inv_b(const JobDesc* __restrict__ jobs,
                                                      const uint2* __restrict__ twi) {
    constexpr int LGC = col_lgc(LGN1);
    constexpr int NTILES = col_ntiles(LGN1);
    constexpr int PER_JOB = (SBG_NP * NTILES) << LGC;
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    const int slab = r & ((1 << LGC) - 1);
    const int rest = r >> LGC;
    col_inv_body<LGN1>(rest % SBG_NP, rest / SBG_NP, slab, J.ws, twi);
}

// ------------------------------------------------------------------------
// Columns of 3 * 2^m rows (transform lengths L = 3 * 2^(m + 12)).
//
// DIF: a radix-3 level over the thirds (rows r, r + M, r + 2M, M = 2^m; the
// second and third outputs twiddled by w_N1^r and w_N1^2r), then a 2^m-point
// DIF in each third, so row t M + j ends up holding frequency 3 bitrev(j) + t.
// A cluster of C = 3 * 2^c CTAs (one slab of M / 2^c <= 2^10 rows each, same
// tile geometry as the power-of-two columns) runs the radix-3 level -- and,
// for c = 1, the top radix-2 level of each third -- in registers across the
// slabs, exchanging through distributed shared memory, then each CTA
// transforms its slab.  The inverse is the exact reverse (DIT, inverse
// twiddles and cube root); its factor 3 is part of the CRT scale 1/L.
//   radix-3 DIF:  y0 = a + b + c, y1 = (a - c + w(b - c)) t, y2 = (a - b - w(b - c)) t^2
// with w the cube root of unity w_N1^M (w^2 = -1 - w).
// ------------------------------------------------------------------------
__device__ __forceinline__ void r3_dif(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t w3,
                                       uint32_t w3s, uint2 t1, uint2 t2, uint32_t p) {
    const uint32_t e = mul_shoup(sub_mod(b, c, p), w3, w3s, p);
    const uint32_t y0 = add_mod(a, add_mod(b, c, p), p);
    const uint32_t y1 = add_mod(sub_mod(a, c, p), e, p);
    const uint32_t y2 = sub_mod(sub_mod(a, b, p), e, p);
    a = y0;
    b = mul_shoup(y1, t1.x, t1.y, p);
    c = mul_shoup(y2, t2.x, t2.y, p);
}

// exact reverse of r3_dif (inverse twiddles t1 = w_N1^-r, t2 = w_N1^-2r and
// inverse cube root): returns 3 (a, b, c)
__device__ __forceinline__ void r3_dit(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t w3i,
                                       uint32_t w3is, uint2 t1, uint2 t2, uint32_t p) {
    const uint32_t y1 = mul_shoup(b, t1.x, t1.y, p);
    const uint32_t y2 = mul_shoup(c, t2.x, t2.y, p);
    const uint32_t e = mul_shoup(sub_mod(y1, y2, p), w3i, w3is, p);
    const uint32_t x0 = add_mod(a, add_mod(y1, y2, p), p);
    const uint32_t x1 = add_mod(sub_mod(a, y2, p), e, p);
    const uint32_t x2 = sub_mod(sub_mod(a, y1, p), e, p);
    a = x0;
    b = x1;
    c = x2;
}

__host__ __device__ constexpr int col3_lgs(int m) { return m < SBG_COL_SLAB_LG ? m : SBG_COL_SLAB_LG; }
__host__ __device__ constexpr int col3_lgc(int m) { return m - col3_lgs(m); }
__host__ __device__ constexpr int col3_csize(int m) { return 3 << col3_lgc(m); }
__host__ __device__ constexpr bool col3_lanes(int m) { return col3_lgs(m) <= SBG_COL_LANE_MAX_LG; }
__host__ __device__ constexpr int col3_lgw(int m) { return col_lgw_of(col3_lanes(m), col3_lgs(m)); }
__host__ __device__ constexpr int col3_smem_bytes(int m) {
    return (1 << col3_lgw(m)) * col_ld_of(col3_lanes(m), col3_lgs(m)) * 4;
}
__host__ __device__ constexpr int col3_ntiles(int m) { return 1 << (SBG_ROW_LG - col3_lgw(m)); }
#define SBG_COL3_CASES(X) X(8) X(9) X(10) X(11)

// shared-memory word of (column, row) in a slab's planes (column pairs: the
// pair's plane of 8-byte words, the column's half of the row's word)
template <bool LANES, int LD>
__device__ __forceinline__ int slab_addr(int col, int r) {
    return LANES ? col * LD + r : (col >> 1) * (2 * LD) + 2 * pad_idx(r) + (col & 1);
}

// cross-slab levels, forward: this CTA's share of rows r of a slab (split
// evenly among the C CTAs), all columns; rows r + MS t of the whole column
template <int M3>
__device__ __forceinline__ void col3_cross_fwd(uint32_t* sm, const uint64_t* __restrict__ X, int64_t xn,
                                               int c0, int slab, const uint2* __restrict__ tw,
                                               const uint2* __restrict__ t3, uint32_t w3, uint32_t w3s,
                                               const PrimeConst& pc) {
    constexpr int LGS = col3_lgs(M3);
    constexpr int MS = 1 << LGS;
    constexpr int G = 1 << col3_lgc(M3);          // slabs per third
    constexpr int C = 3 * G;
    constexpr bool LANES = col3_lanes(M3);
    constexpr int LGW = col3_lgw(M3);
    constexpr int LD = col_ld_of(LANES, LGS);
    const int r_lo = (slab * MS) / C, r_hi = ((slab + 1) * MS) / C;
    const int items = (r_hi - r_lo) << LGW;
    cg::cluster_group cl = cg::this_cluster();
    for (int gid = threadIdx.x; gid < items; gid += COL_THREADS) {
        const int col = gid & ((1 << LGW) - 1);
        const int r = r_lo + (gid >> LGW);
        uint32_t x[C];
        const int64_t n0 = ((int64_t)r << SBG_ROW_LG) + c0 + col;
#pragma unroll
        for (int t = 0; t < C; ++t) x[t] = load_limb(X, xn, n0 + ((int64_t)(MS * t) << SBG_ROW_LG), pc);
#pragma unroll
        for (int u = 0; u < G; ++u) {
            const int rr = r + u * MS;                 // row within a third
            r3_dif(x[u], x[u + G], x[u + 2 * G], w3, w3s, __ldg(&t3[rr]), __ldg(&t3[2 * rr]), pc.p);
        }
        if constexpr (G == 2) {                        // top radix-2 level of each third
            const uint2 w = __ldg(&tw[tw_idx(M3, r)]);
#pragma unroll
            for (int k = 0; k < 3; ++k) bfly_gs(x[2 * k], x[2 * k + 1], w.x, w.y, pc.p);
        }
        const int a = slab_addr<LANES, LD>(col, r);
#pragma unroll
        for (int t = 0; t < C; ++t) cl.map_shared_rank(sm, t)[a] = x[t];
    }
}

template <int M3>
__device__ __forceinline__ void col3_cross_inv(uint32_t* sm, uint32_t* __restrict__ Y, int c0, int slab,
                                               const uint2* __restrict__ tw, const uint2* __restrict__ t3,
                                               uint32_t w3, uint32_t w3s, const PrimeConst& pc) {
    constexpr int LGS = col3_lgs(M3);
    constexpr int MS = 1 << LGS;
    constexpr int G = 1 << col3_lgc(M3);
    constexpr int C = 3 * G;
    constexpr bool LANES = col3_lanes(M3);
    constexpr int LGW = col3_lgw(M3);
    constexpr int LD = col_ld_of(LANES, LGS);
    const int r_lo = (slab * MS) / C, r_hi = ((slab + 1) * MS) / C;
    const int items = (r_hi - r_lo) << LGW;
    cg::cluster_group cl = cg::this_cluster();
    for (int gid = threadIdx.x; gid < items; gid += COL_THREADS) {
        const int col = gid & ((1 << LGW) - 1);
        const int r = r_lo + (gid >> LGW);
        uint32_t x[C];
        const int a = slab_addr<LANES, LD>(col, r);
#pragma unroll
        for (int t = 0; t < C; ++t) x[t] = cl.map_shared_rank(sm, t)[a];
        if constexpr (G == 2) {
            const uint2 w = __ldg(&tw[tw_idx(M3, r)]);
#pragma unroll
            for (int k = 0; k < 3; ++k) bfly_ct(x[2 * k], x[2 * k + 1], w.x, w.y, pc.p);
        }
#pragma unroll
        for (int u = 0; u < G; ++u) {
            const int rr = r + u * MS;
            r3_dit(x[u], x[u + G], x[u + 2 * G], w3, w3s, __ldg(&t3[rr]), __ldg(&t3[2 * rr]), pc.p);
        }
        const int64_t n0 = ((int64_t)r << SBG_ROW_LG) + c0 + col;
#pragma unroll
        for (int t = 0; t < C; ++t) Y[n0 + ((int64_t)(MS * t) << SBG_ROW_LG)] = x[t];
    }
}

template <int M3>
__device__ __forceinline__ void col3_fwd_body(int q, int tile, int slab, int op,
                                              const uint64_t* __restrict__ a, int64_t an,
                                              const uint64_t* __restrict__ b, int64_t bn,
                                              const uint2* __restrict__ twf, const Radix3Arg& r3,
                                              uint32_t* __restrict__ YA, uint32_t* __restrict__ YB) {
    extern __shared__ uint32_t sm[];
    constexpr int LGS = col3_lgs(M3);
    constexpr size_t L = (size_t)3 << (M3 + SBG_ROW_LG);
    const uint64_t* X = op ? b : a;
    const int64_t xn = op ? bn : an;
    uint32_t* Y = (op ? YB : YA) + (size_t)q * L;
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twf + (size_t)q * SBG_TW_N;
    const int c0 = tile << col3_lgw(M3);
    cluster_barrier<false>();           // every CTA of the cluster is running
    col3_cross_fwd<M3>(sm, X, xn, c0, slab, tw, r3.t3 + ((size_t)q << (M3 + 1)), r3.w[q], r3.ws[q], pc);
    cluster_barrier<true>();            // all slabs complete in shared memory
    col_slab_fwd<col3_lanes(M3), LGS, false, true>(sm, X, xn, Y, c0, slab << LGS, tw, pc);
}

template <int M3>
__device__ __forceinline__ void col3_inv_body(int q, int tile, int slab, uint32_t* __restrict__ YA,
                                              const uint2* __restrict__ twi, const Radix3Arg& r3) {
    extern __shared__ uint32_t sm[];
    constexpr int LGS = col3_lgs(M3);
    constexpr size_t L = (size_t)3 << (M3 + SBG_ROW_LG);
    uint32_t* Y = YA + (size_t)q * L;
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twi + (size_t)q * SBG_TW_N;
    const int c0 = tile << col3_lgw(M3);
    col_slab_inv<col3_lanes(M3), LGS, true, false>(sm, Y, c0, slab << LGS, tw, pc);
    cluster_barrier<true>();            // all slabs complete in shared memory
    col3_cross_inv<M3>(sm, Y, c0, slab, tw, r3.t3 + ((size_t)q << (M3 + 1)), r3.w[q], r3.ws[q], pc);
    cluster_barrier<false>();           // peers read this CTA's slab until here
}

// Short 3 * 2^m columns (m <= SBG_COL3S_MAX): the whole column in one CTA,
// W = 2^(12 - m) >= 32 columns of 3 * 2^m rows (12288 points) stacked as
// three 2^m-row slabs in planes of 3 * 2^m + 1 words; the radix-3 level is
// one pass between global memory and the planes, no cluster exchange.
template <int M3, bool FWD>
__device__ __forceinline__ void col3s_r3_pass(uint32_t* sm, const uint64_t* __restrict__ X, int64_t xn,
                                              uint32_t* __restrict__ Y, int c0, const uint2* __restrict__ t3,
                                              uint32_t w3, uint32_t w3s, const PrimeConst& pc) {
    constexpr int M = 1 << M3;
    constexpr int LGW = col3s_lgw(M3);
    constexpr int LD = 3 * M + 1;
    constexpr int ITER = (M << LGW) / COL_THREADS;
#pragma unroll 2
    for (int it = 0; it < ITER; ++it) {
        const int gid = threadIdx.x + it * COL_THREADS;
        const int col = gid & ((1 << LGW) - 1);
        const int r = gid >> LGW;
        uint32_t* s0 = sm + col * LD + r;
        const uint2 ta = __ldg(&t3[r]), tb = __ldg(&t3[2 * r]);
        const int64_t n0 = ((int64_t)r << SBG_ROW_LG) + c0 + col;
        constexpr int64_t DM = (int64_t)M << SBG_ROW_LG;
        if constexpr (FWD) {
            uint32_t a = load_limb(X, xn, n0, pc), b = load_limb(X, xn, n0 + DM, pc),
                     c = load_limb(X, xn, n0 + 2 * DM, pc);
            r3_dif(a, b, c, w3, w3s, ta, tb, pc.p);
            s0[0] = a;
            s0[M] = b;
            s0[2 * M] = c;
        } else {
            uint32_t a = s0[0], b = s0[M], c = s0[2 * M];
            r3_dit(a, b, c, w3, w3s, ta, tb, pc.p);
            Y[n0] = a;
            Y[n0 + DM] = b;
            Y[n0 + 2 * DM] = c;
        }
    }
}

__host__ __device__ constexpr int col3s_smem_bytes(int m) { return (1 << col3s_lgw(m)) * (3 * (1 << m) + 1) * 4; }
__host__ __device__ constexpr int col3s_ntiles(int m) { return 1 << m; }
#define SBG_COL3S_CASES(X) X(4) X(5) X(6) X(7)

template <int M3>
__device__ __forceinline__ void col3s_fwd_body(int q, int tile, int op, const uint64_t* __restrict__ a, int64_t an,
                                               const uint64_t* __restrict__ b, int64_t bn,
                                               const uint2* __restrict__ twf, const Radix3Arg& r3,
                                               uint32_t* __restrict__ YA, uint32_t* __restrict__ YB) {
    extern __shared__ uint32_t sm[];
    constexpr size_t L = (size_t)3 << (M3 + SBG_ROW_LG);
    const uint64_t* X = op ? b : a;
    const int64_t xn = op ? bn : an;
    uint32_t* Y = (op ? YB : YA) + (size_t)q * L;
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twf + (size_t)q * SBG_TW_N;
    const int c0 = tile << col3s_lgw(M3);
    col3s_r3_pass<M3, true>(sm, X, xn, Y, c0, r3.t3 + ((size_t)q << (M3 + 1)), r3.w[q], r3.ws[q], pc);
    __syncthreads();
    col_slab_fwd<true, M3, false, true, 3>(sm, X, xn, Y, c0, 0, tw, pc);
}

template <int M3>
__device__ __forceinline__ void col3s_inv_body(int q, int tile, uint32_t* __restrict__ YA,
                                               const uint2* __restrict__ twi, const Radix3Arg& r3) {
    extern __shared__ uint32_t sm[];
    constexpr size_t L = (size_t)3 << (M3 + SBG_ROW_LG);
    uint32_t* Y = YA + (size_t)q * L;
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twi + (size_t)q * SBG_TW_N;
    const int c0 = tile << col3s_lgw(M3);
    col_slab_inv<true, M3, true, false, 3>(sm, Y, c0, 0, tw, pc);
    __syncthreads();
    col3s_r3_pass<M3, false>(sm, nullptr, 0, Y, c0, r3.t3 + ((size_t)q << (M3 + 1)), r3.w[q], r3.ws[q], pc);
}

// blocks: prime fastest, then tile, operand
template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL3_FWD_MINB) k_col3s_fwd(const uint64_t* __restrict__ a, int64_t an,
                                                                   const uint64_t* __restrict__ b, int64_t bn,
                                                                   const uint2* __restrict__ twf, Radix3Arg r3,
                                                                   uint32_t* __restrict__ YA,
                                                                   uint32_t* __restrict__ YB) {
    constexpr int NTILES = col3s_ntiles(M3);
    const int q = blockIdx.x % SBG_NP;
    const int rest = blockIdx.x / SBG_NP;
    col3s_fwd_body<M3>(q, rest % NTILES, rest / NTILES, a, an, b, bn, twf, r3, YA, YB);
}

template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL3_FWD_MINB) k_col3s_fwd_b(const JobDesc* __restrict__ jobs,
                                                                     const uint2* __restrict__ twf, Radix3Arg r3) {
    constexpr int NTILES = col3s_ntiles(M3);
    constexpr int PER_JOB = SBG_NP * 2 * NTILES;
    constexpr size_t L = (size_t)3 << (M3 + SBG_ROW_LG);
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    const int q = r % SBG_NP;
    const int rest = r / SBG_NP;
    const int op = rest / NTILES;
    if (op && J.sq) return;
    col3s_fwd_body<M3>(q, rest % NTILES, op, J.a, J.an, J.b, J.bn, twf, r3, J.ws, J.ws + SBG_NP * L);
}

template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL_MINB) k_col3s_inv(uint32_t* __restrict__ YA,
                                                                   const uint2* __restrict__ twi, Radix3Arg r3) {
    col3s_inv_body<M3>(blockIdx.x % SBG_NP, blockIdx.x / SBG_NP, YA, twi, r3);
}

template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL_MINB) k_col3s_inv_b(const JobDesc* __restrict__ jobs,
                                                                     const uint2* __restrict__ twi, Radix3Arg r3) {
    constexpr int NTILES = col3s_ntiles(M3);
    constexpr int PER_JOB = SBG_NP * NTILES;
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    col3s_inv_body<M3>(r % SBG_NP, r / SBG_NP, J.ws, twi, r3);
}

// blocks: slab fastest (a cluster), then prime, tile, operand
template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL3_FWD_MINB) k_col3_fwd(const uint64_t* __restrict__ a, int64_t an,
                                                                  const uint64_t* __restrict__ b, int64_t bn,
                                                                  const uint2* __restrict__ twf, Radix3Arg r3,
                                                                  uint32_t* __restrict__ YA,
                                                                  uint32_t* __restrict__ YB) {
    constexpr int C = col3_csize(M3);
    constexpr int NTILES = col3_ntiles(M3);
    const int slab = blockIdx.x % C;
    int rest = blockIdx.x / C;
    const int q = rest % SBG_NP;
    rest /= SBG_NP;
    col3_fwd_body<M3>(q, rest % NTILES, slab, rest / NTILES, a, an, b, bn, twf, r3, YA, YB);
}

template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL3_FWD_MINB) k_col3_fwd_b(const JobDesc* __restrict__ jobs,
                                                                    const uint2* __restrict__ twf, Radix3Arg r3) {
    constexpr int C = col3_csize(M3);
    constexpr int NTILES = col3_ntiles(M3);
    constexpr int PER_JOB = SBG_NP * 2 * NTILES * C;
    constexpr size_t L = (size_t)3 << (M3 + SBG_ROW_LG);
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    const int slab = r % C;
    int rest = r / C;
    const int q = rest % SBG_NP;
    rest /= SBG_NP;
    const int op = rest / NTILES;
    if (op && J.sq) return;             // whole clusters together
    col3_fwd_body<M3>(q, rest % NTILES, slab, op, J.a, J.an, J.b, J.bn, twf, r3, J.ws, J.ws + SBG_NP * L);
}

template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL_MINB) k_col3_inv(uint32_t* __restrict__ YA,
                                                                  const uint2* __restrict__ twi, Radix3Arg r3) {
    constexpr int C = col3_csize(M3);
    const int slab = blockIdx.x % C;
    const int rest = blockIdx.x / C;
    col3_inv_body<M3>(rest % SBG_NP, rest / SBG_NP, slab, YA, twi, r3);
}

template <int M3>
__global__ void __launch_bounds__(COL_THREADS, COL_MINB) k_col3_inv_b(const JobDesc* __restrict__ jobs,
                                                                    const uint2* __restrict__ twi, Radix3Arg r3) {
    constexpr int C = col3_csize(M3);
    constexpr int NTILES = col3_ntiles(M3);
    constexpr int PER_JOB = SBG_NP * NTILES * C;
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    const int slab = r % C;
    const int rest = r / C;
    col3_inv_body<M3>(rest % SBG_NP, rest / SBG_NP, slab, J.ws, twi, r3);
}

// K2: one row of N2 = 2^12 points for one prime, 256 threads.
//   P1  global -> four-step twiddle -> DIF levels 1-4 (A and B) -> smem
//   P2  DIF levels 5-8 (A and B)
//   P3  DIF levels 9-12, pointwise Montgomery product, DIT levels 12-9
//   P2' DIT levels 8-5
//   P1' DIT levels 4-1 -> inverse twiddle x CRT scale -> global (over A)
// The last forward pass, the product and the first inverse pass share one
// register group, so that stage never touches shared memory.
#define ROW_LG 12
#define ROW_N (1 << ROW_LG)
#ifndef ROW_MINB
#define ROW_MINB 4                // resident CTAs per SM the register budget is set for
#endif
// shared memory of one row: both operands' planes and the 16 four-step
// twiddle steps of each direction
struct RowSmem {
    uint32_t A[padded_len(ROW_N)];
    uint32_t B[padded_len(ROW_N)];
    uint2 f[16];
    uint2 i[16];
};

// (scw, scws): the CRT scale of prime q and its Shoup companion
__device__ __forceinline__ void row_body(int q, int row, uint32_t* __restrict__ YA,
                                         const uint32_t* __restrict__ YB, int sq, int lgN1, int m3,
                                         const FsTables& fsf, const FsTables& fsi,
                                         uint32_t scw, uint32_t scws, const uint2* __restrict__ twf,
                                         const uint2* __restrict__ twi, RowSmem& S) {
    uint32_t* smA = S.A;
    uint32_t* smB = S.B;
    uint2* s_f = S.f;
    uint2* s_i = S.i;
    const int tid = threadIdx.x;
    const PrimeConst pc = c_pr[q];
    const uint32_t p = pc.p;
    // rows: 2^lgN1, or 3 * 2^m3 (m3 >= 0); the column DIF left row p holding
    // frequency bitrev(p) resp. 3 bitrev(p mod 2^m3) + p / 2^m3
    const size_t n1 = m3 >= 0 ? (size_t)3 << m3 : (size_t)1 << lgN1;
    const size_t base = ((size_t)q * n1 << ROW_LG) + ((size_t)row << ROW_LG);
    const uint2* tf = twf + (size_t)q * SBG_TW_N;
    const uint2* ti = twi + (size_t)q * SBG_TW_N;
    const uint32_t k1 = m3 >= 0 ? 3u * bitrev((uint32_t)row & ((1u << m3) - 1u), m3) + ((uint32_t)row >> m3)
                                : bitrev((uint32_t)row, lgN1);
    // four-step twiddles: w_L^(k1 (tid + 256 t)) = b * s^t
    if (tid < 16) {
        uint32_t e = k1 * 256u * (uint32_t)tid;          // < L: no reduction
        uint32_t v = fs_value(fsf, q, e, p);
        s_f[tid] = make_uint2(v, shoup_fast(v, pc));
        uint32_t vi = mul_shoup(fs_value(fsi, q, e, p), scw, scws, p);
        s_i[tid] = make_uint2(vi, shoup_fast(vi, pc));
    }
    const uint32_t eb = k1 * (uint32_t)tid;
    const uint32_t bf = fs_value(fsf, q, eb, p), bfs = shoup_fast(bf, pc);
    const uint32_t bi = fs_value(fsi, q, eb, p), bis = shoup_fast(bi, pc);
    __syncthreads();

    uint32_t xa[16], xb[16];
    // P1
    {
        const uint32_t* Ar = YA + base;
        const uint32_t* Br = YB + base;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            uint2 s = s_f[t];
            xa[t] = mul_shoup(mul_shoup(__ldcg(&Ar[tid + 256 * t]), s.x, s.y, p), bf, bfs, p);
            if (!sq) xb[t] = mul_shoup(mul_shoup(__ldcg(&Br[tid + 256 * t]), s.x, s.y, p), bf, bfs, p);
        }
        if (sq) {
            dif_regs<16>(xa, tf, tid, 256, 12, p);
        } else {
            dif_regs2<16>(xa, xb, tf, tid, 256, 12, p);
        }
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            smA[pad_idx(tid + 256 * t)] = xa[t];
            if (!sq) smB[pad_idx(tid + 256 * t)] = xb[t];
        }
    }
    __syncthreads();
    // P2: M = 256, st = 16
    {
        const int j0 = tid & 15, i0 = ((tid >> 4) << 8) + j0;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            xa[t] = smA[pad_idx(i0 + 16 * t)];
            if (!sq) xb[t] = smB[pad_idx(i0 + 16 * t)];
        }
        if (sq) {
            dif_regs<16>(xa, tf, j0, 16, 8, p);
        } else {
            dif_regs2<16>(xa, xb, tf, j0, 16, 8, p);
        }
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            smA[pad_idx(i0 + 16 * t)] = xa[t];
            if (!sq) smB[pad_idx(i0 + 16 * t)] = xb[t];
        }
    }
    __syncthreads();
    // P3: M = 16, st = 1, fused product
    {
        const int i0 = tid << 4;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            xa[t] = smA[pad_idx(i0 + t)];
            if (!sq) xb[t] = smB[pad_idx(i0 + t)];
        }
        if (sq) {
            dif_regs<16, true>(xa, tf, 0, 1, 4, p);
#pragma unroll
            for (int t = 0; t < 16; ++t) xa[t] = mont_mul(xa[t], xa[t], p, pc.pinv);
        } else {
            dif_regs2<16, true>(xa, xb, tf, 0, 1, 4, p);
#pragma unroll
            for (int t = 0; t < 16; ++t) xa[t] = mont_mul(xa[t], xb[t], p, pc.pinv);
        }
        dit_regs<16, true>(xa, ti, 0, 1, 4, p);
#pragma unroll
        for (int t = 0; t < 16; ++t) smA[pad_idx(i0 + t)] = xa[t];
    }
    __syncthreads();
    // P2'
    {
        const int j0 = tid & 15, i0 = ((tid >> 4) << 8) + j0;
#pragma unroll
        for (int t = 0; t < 16; ++t) xa[t] = smA[pad_idx(i0 + 16 * t)];
        dit_regs<16>(xa, ti, j0, 16, 8, p);
#pragma unroll
        for (int t = 0; t < 16; ++t) smA[pad_idx(i0 + 16 * t)] = xa[t];
    }
    __syncthreads();
    // P1'
    {
#pragma unroll
        for (int t = 0; t < 16; ++t) xa[t] = smA[pad_idx(tid + 256 * t)];
        dit_regs<16>(xa, ti, tid, 256, 12, p);
        uint32_t* Ar = YA + base;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            uint2 s = s_i[t];
            Ar[tid + 256 * t] = mul_shoup(mul_shoup(xa[t], s.x, s.y, p), bi, bis, p);
        }
    }
}

__global__ void __launch_bounds__(256, ROW_MINB) k_row12(uint32_t* __restrict__ YA,
                                                  const uint32_t* __restrict__ YB, int sq,
                                                  int lgN1, int m3, FsTables fsf, FsTables fsi,
                                                  ScaleArg sc, const uint2* __restrict__ twf,
                                                  const uint2* __restrict__ twi) {
    __shared__ RowSmem S;
    const int n1 = m3 >= 0 ? 3 << m3 : 1 << lgN1;
    const int q = blockIdx.x / n1;
    row_body(q, blockIdx.x - q * n1, YA, YB, sq, lgN1, m3, fsf, fsi, sc.w[q], sc.ws[q], twf, twi, S);
}

// batched: blocks (job, prime, row), job slowest
__global__ void __launch_bounds__(256, ROW_MINB) k_row12_b(const JobDesc* __restrict__ jobs, int lgN1,
                                                    int m3, FsTables fsf, FsTables fsi, ScaleArg sc,
                                                    const uint2* __restrict__ twf,
                                                    const uint2* __restrict__ twi) {
    const int n1 = m3 >= 0 ? 3 << m3 : 1 << lgN1;
    const int per_job = SBG_NP * n1;
    const JobDesc& J = jobs[blockIdx.x / per_job];
    const int r = blockIdx.x % per_job;
    __shared__ RowSmem S;
    uint32_t* YB = J.ws + (size_t)SBG_NP * n1 * ROW_N;
    const int q = r / n1;
    row_body(q, r % n1, J.ws, YB, J.sq, lgN1, m3, fsf, fsi, sc.w[q], sc.ws[q], twf, twi, S);
}

// ------------------------------------------------------------------------
// K4: Garner CRT + three-stream compose + carry resolution.
//
// Coefficient c_j (j in [cmin, cmax]) is rebuilt from its five residues by
// Garner's mixed radix (ascending primes), then composed by Horner into
// 160 bits = lo (bits 0-63) + mid (64-127) + hi (128-159).  Limb m of the
// window sum  sum_j c_j 2^(64 (j - off))  is
//     z_m = lo_{m+off} + mid_{m+off-1} + hi_{m+off-2} + carry,
// the reference's lo/mid/hi stream recombination (include/p30.h:1695-1842).
// Each warp owns CRT_SEG consecutive limbs and walks them 128 at a time,
// lane l on the four limbs seg + 128 s + 4 l + (0..3): the residue loads are
// one 16-byte vector per prime and the limb stores two 16-byte vectors, all
// coalesced across the warp.  The neighbour terms (mid and hi of the lane
// below's top coefficients, and the sum carry of its top limb) come by a
// rotating shuffle; lane 0 keeps the previous step's lane 31 values, and a
// prologue of three coefficients starts the segment.  Before carries, limb m
// is z'_m = lo + mid + hi + (sum carry of limb m-1) mod 2^64; it generates
// a carry (G) when that wraps and propagates one (P) when z'_m = 2^64 - 1.
// For G and P bit masks g, p (exclusive per position) the carries into the
// positions for carry-in c are  (p + (g << 1 | c)) ^ p,  one add: over a
// lane's four limbs, and over the warp's 32 lanes with the lanes' (G, P) as
// ballot masks.  The z' wait in shared memory while the warp's carry-in is
// found: the steps' (G, P) compose to the warp's, and a block scan of the
// warps plus a decoupled look-back across blocks (block order from an atomic
// ticket, so every predecessor is already resident) give the block's.
// ------------------------------------------------------------------------
#define CRT_T 256
#define CRT_V 4                                 // consecutive limbs per lane and step
#ifndef CRT_NSTEP
#define CRT_NSTEP 4                             // steps per warp
#endif
#define CRT_SEG (32 * CRT_V * CRT_NSTEP)        // limbs per warp
#ifndef CRT_MINB
#define CRT_MINB 4                              // blocks per SM (64 registers)
#endif
#define CRT_BLK ((CRT_T / 32) * CRT_SEG)        // limbs per block
#define LB_SPIN_LIMIT (1 << 22)
#define LB_SPIN_LIMIT_TEST (1 << 12)

// Test hooks for the error paths (sbg_debug_inject, 0 = off): they change
// data or withhold a flag, never an address, so an injected failure shows as
// an error status and never as a fault or an unbounded wait.
__device__ uint32_t g_inject;
#define FLAG_AGG 1u
#define FLAG_INC 2u

// Garner (ascending primes) + Horner compose of one coefficient from its
// five residues (already scaled to the true coefficient residues).
__device__ __forceinline__ void garner(const uint32_t (&r)[SBG_NP], uint64_t& lo, uint64_t& mid,
                                       uint32_t& hi) {
    uint32_t v[SBG_NP];
#pragma unroll
    for (int q = 0; q < SBG_NP; ++q) v[q] = r[q];
#pragma unroll
    for (int i = 1; i < SBG_NP; ++i) {
        uint32_t p = c_pr[i].p;
        uint32_t acc = v[0];
#pragma unroll
        for (int k = 1; k < i; ++k)
            acc = add_mod(acc, mul_shoup(v[k], c_crt.ppm[i][k], c_crt.ppms[i][k], p), p);
        v[i] = mul_shoup(sub_mod(v[i], acc, p), c_crt.inv[i], c_crt.invs[i], p);
    }
    // Horner: c = v0 + p0 (v1 + p1 (v2 + p2 (v3 + p3 v4)))
    uint32_t w0 = v[4], w1 = 0, w2 = 0, w3 = 0, w4 = 0;
    {
        uint64_t t = (uint64_t)w0 * c_pr[3].p + v[3];
        w0 = (uint32_t)t;
        w1 = (uint32_t)(t >> 32);
    }
    {
        uint64_t t = (uint64_t)w0 * c_pr[2].p + v[2];
        w0 = (uint32_t)t;
        t = (uint64_t)w1 * c_pr[2].p + (t >> 32);
        w1 = (uint32_t)t;
        w2 = (uint32_t)(t >> 32);
    }
    {
        uint64_t t = (uint64_t)w0 * c_pr[1].p + v[1];
        w0 = (uint32_t)t;
        t = (uint64_t)w1 * c_pr[1].p + (t >> 32);
        w1 = (uint32_t)t;
        t = (uint64_t)w2 * c_pr[1].p + (t >> 32);
        w2 = (uint32_t)t;
        w3 = (uint32_t)(t >> 32);
    }
    {
        uint64_t t = (uint64_t)w0 * c_pr[0].p + v[0];
        w0 = (uint32_t)t;
        t = (uint64_t)w1 * c_pr[0].p + (t >> 32);
        w1 = (uint32_t)t;
        t = (uint64_t)w2 * c_pr[0].p + (t >> 32);
        w2 = (uint32_t)t;
        t = (uint64_t)w3 * c_pr[0].p + (t >> 32);
        w3 = (uint32_t)t;
        w4 = (uint32_t)(t >> 32);
    }
    lo = ((uint64_t)w1 << 32) | w0;
    mid = ((uint64_t)w3 << 32) | w2;
    hi = w4;
}

// (G, P) carry pairs packed in 2 bits: bit0 = G (carry out with carry-in 0),
// bit1 = P (carry-in passes through).  compose(left, right) = right o left.
__device__ __forceinline__ uint32_t gp_compose(uint32_t left, uint32_t right) {
    uint32_t gl = left & 1, pl = (left >> 1) & 1, gr = right & 1, pr = (right >> 1) & 1;
    return (gr | (pr & gl)) | ((pr & pl) << 1);
}

// y + k 2^64 = lo + mid + hi  (k <= 2)
__device__ __forceinline__ void sum3(uint64_t lo, uint64_t mid, uint32_t hi, uint64_t& y, uint32_t& k) {
    const uint64_t s1 = lo + mid;
    k = s1 < lo;
    y = s1 + hi;
    k += y < s1;
}

// NSTEP: steps of 128 limbs per warp (a block covers 8 * 128 * NSTEP limbs)
template <int NSTEP>
struct CrtSmemT {
    ulonglong2 z[(CRT_T / 32) * 32 * CRT_V * NSTEP / 2];   // limbs before carries
    uint32_t gp[CRT_T / 32][NSTEP][2];                     // per warp and step: g, p
    uint32_t warp[CRT_T / 32];
    uint32_t cin;
};
using CrtSmem = CrtSmemT<CRT_NSTEP>;

template <int NSTEP>
__device__ __forceinline__ void crt_body_t(uint32_t bid, const uint32_t* __restrict__ R, int64_t L,
                                           int64_t cmin, int64_t cmax, int64_t off,
                                           uint64_t* __restrict__ out, int64_t nout,
                                           uint32_t* flags, uint32_t* err, CrtSmemT<NSTEP>& S) {
    constexpr int SEG = 32 * CRT_V * NSTEP;                // limbs per warp
    constexpr int BLK = (CRT_T / 32) * SEG;                // limbs per block
    ulonglong2* s_z = S.z;
    auto& s_gp = S.gp;
    uint32_t* s_warp = S.warp;
    uint32_t& s_cin = S.cin;
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int src1 = (lane + 31) & 31;
    const int64_t seg = (int64_t)bid * BLK + (int64_t)wid * SEG;
    const uint32_t inj = *(volatile uint32_t*)&g_inject;
    // injected residue corruption: the top coefficient (the product then
    // spills) or a middle one (a wrong product no device check sees)
    auto corrupt = [&](int64_t j, uint32_t& r0) {
        if (((inj & SBG_INJECT_TOP) && j == cmax) ||
            ((inj & SBG_INJECT_MID) && j == cmin + (cmax - cmin) / 2))
            r0 ^= 1u;
    };
    ulonglong2* zs = s_z + wid * (SEG / 2);         // unit (2 s + half) * 32 + lane
    // residues of the coefficients j = m + off of limbs m .. m+3; zero outside
    // [cmin, cmax], which Garner maps to lo = mid = hi = 0
    auto fetch4 = [&](int64_t m, uint32_t (&r)[CRT_V][SBG_NP]) {
        const int64_t j = m + off;
        if (((j & 3) == 0) && j >= cmin && j + 3 <= cmax) {
#pragma unroll
            for (int q = 0; q < SBG_NP; ++q) {
                const uint4 v = __ldcg(reinterpret_cast<const uint4*>(R + (size_t)q * L + j));
                r[0][q] = v.x;
                r[1][q] = v.y;
                r[2][q] = v.z;
                r[3][q] = v.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < CRT_V; ++k) {
                const bool in = j + k >= cmin && j + k <= cmax;
#pragma unroll
                for (int q = 0; q < SBG_NP; ++q) r[k][q] = in ? __ldcg(&R[(size_t)q * L + j + k]) : 0u;
            }
        }
    };
    // what lane 0 takes from below: mid and hi of the limb below, hi two
    // below, the sum carry of the limb below.  Prologue: lanes 29..31 rebuild
    // the coefficients of limbs seg-3 .. seg-1.
    uint64_t c_mid3;
    uint32_t c_hi2, c_hi3, c_k3;
    {
        uint64_t lo = 0, mid = 0;
        uint32_t hi = 0;
        if (lane >= 29) {
            uint32_t r[SBG_NP];
            const int64_t j = seg - 32 + lane + off;
            const bool in = j >= cmin && j <= cmax;
#pragma unroll
            for (int q = 0; q < SBG_NP; ++q) r[q] = in ? __ldcg(&R[(size_t)q * L + j]) : 0u;
            if (inj && in) corrupt(j, r[0]);
            garner(r, lo, mid, hi);
        }
        uint64_t y;
        uint32_t k;
        sum3(lo, __shfl_up_sync(FULL, mid, 1), __shfl_up_sync(FULL, hi, 2), y, k);
        c_mid3 = __shfl_sync(FULL, mid, 31);
        c_hi2 = __shfl_sync(FULL, hi, 30);
        c_hi3 = __shfl_sync(FULL, hi, 31);
        c_k3 = __shfl_sync(FULL, k, 31);
        if (seg - 1 < 0) c_k3 = 0;      // limb -1 carries nothing into limb 0
    }
    uint32_t wG = 0, wP = 1;            // the warp's (G, P) so far: identity
    uint32_t bits = 0;                  // per step: 4 G bits, 4 P bits
    uint64_t zv = 0;                    // the spill limb nout, before carries,
    uint32_t vbad = 0;                  //   what it must not carry out,
    int vpos = -1;                      //   and where it sits (4 s + k)
    // a runtime loop: each step holds four Garner reconstructions, and
    // unrolling the steps quadruples the code the warps fetch
#pragma unroll 1
    for (int s = 0; s < NSTEP; ++s) {
        const int64_t m0 = seg + 128 * s + 4 * lane;
        uint32_t r[CRT_V][SBG_NP];
        fetch4(m0, r);
        if (inj) {
#pragma unroll
            for (int k = 0; k < CRT_V; ++k)
                if (m0 + off + k >= cmin && m0 + off + k <= cmax) corrupt(m0 + off + k, r[k][0]);
        }
        // top coefficients first: the lane above needs them
        uint64_t lo3, mid3, lo2, mid2;
        uint32_t hi3, hi2;
        garner(r[3], lo3, mid3, hi3);
        garner(r[2], lo2, mid2, hi2);
        const uint64_t n_mid3 = __shfl_sync(FULL, mid3, src1);
        const uint32_t n_hi2 = __shfl_sync(FULL, hi2, src1);
        const uint32_t n_hi3 = __shfl_sync(FULL, hi3, src1);
        const uint64_t b_mid3 = lane == 0 ? c_mid3 : n_mid3;
        const uint32_t b_hi2 = lane == 0 ? c_hi2 : n_hi2;
        const uint32_t b_hi3 = lane == 0 ? c_hi3 : n_hi3;
        c_mid3 = n_mid3;                // lane 0: this step's lane 31
        c_hi2 = n_hi2;
        c_hi3 = n_hi3;
        uint64_t lo0, mid0, lo1, mid1;
        uint32_t hi0, hi1;
        garner(r[0], lo0, mid0, hi0);
        garner(r[1], lo1, mid1, hi1);
        uint64_t y[CRT_V];
        uint32_t kk[CRT_V];
        sum3(lo0, b_mid3, b_hi2, y[0], kk[0]);
        sum3(lo1, mid0, b_hi3, y[1], kk[1]);
        sum3(lo2, mid1, hi0, y[2], kk[2]);
        sum3(lo3, mid2, hi1, y[3], kk[3]);
        const uint32_t n_k3 = __shfl_sync(FULL, kk[3], src1);
        const uint32_t b_k3 = lane == 0 ? c_k3 : n_k3;
        c_k3 = n_k3;
        uint64_t z[CRT_V];
        uint32_t gb = 0, pb = 0;
#pragma unroll
        for (int k = 0; k < CRT_V; ++k) {
            z[k] = y[k] + (k == 0 ? b_k3 : kk[k - 1]);
            uint32_t G = z[k] < y[k], P = z[k] == ~0ull;
            if (m0 + k >= nout) {
                if (m0 + k == nout) {   // must end zero with no carry beyond it
                    zv = z[k];
                    vbad = G | kk[k];
                    vpos = CRT_V * s + k;
                }
                G = 0;
                P = 0;
            }
            gb |= G << k;
            pb |= P << k;
        }
        zs[(2 * s) * 32 + lane] = make_ulonglong2(z[0], z[1]);
        zs[(2 * s + 1) * 32 + lane] = make_ulonglong2(z[2], z[3]);
        bits |= (gb | (pb << 4)) << (8 * s);
        // the lane's (G, P) over its limbs, then the warp's for the step
        const uint32_t lG = (pb + (gb << 1)) >> CRT_V, lP = pb == (1u << CRT_V) - 1u;
        const uint32_t g = __ballot_sync(FULL, lG), p = __ballot_sync(FULL, lP);
        if (lane == 0) {
            s_gp[wid][s][0] = g;
            s_gp[wid][s][1] = p;
        }
        const uint32_t sG = (uint32_t)(((uint64_t)p + (g << 1)) >> 32) | (g >> 31);
        const uint32_t sP = p == FULL;
        wG = sG | (sP & wG);
        wP = sP & wP;
    }
    const uint32_t gp = wG | (wP << 1);
    if (lane == 0) s_warp[wid] = gp;
    __syncthreads();

    // block scan of the warps' (G, P), then the look-back
    if (wid == 0) {
        uint32_t wv = lane < CRT_T / 32 ? s_warp[lane] : 2u;   // identity = (G0, P1)
        uint32_t wi = wv;
#pragma unroll
        for (int d = 1; d < CRT_T / 32; d <<= 1) {
            uint32_t o = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi = gp_compose(o, wi);
        }
        if (lane < CRT_T / 32) s_warp[lane] = wi;       // inclusive warp prefixes
        if (lane == CRT_T / 32 - 1) {
            // block aggregate wi; look-back for the block carry-in
            uint32_t agg = wi;
            uint32_t cin = 0;
            volatile uint32_t* vf = flags + 1;
            if (bid == 0) {
                cin = 0;
            } else {
                atomicExch(&flags[1 + bid], FLAG_AGG | ((agg & 3u) << 2));
                uint32_t gacc = 0, pacc = 1;
                int64_t jb = (int64_t)bid - 1;
                int spins = 0;
                const int limit = (inj & SBG_INJECT_WITHHOLD) ? LB_SPIN_LIMIT_TEST : LB_SPIN_LIMIT;
                while (true) {
                    uint32_t f = vf[jb];
                    if (f == 0) {
                        if (++spins > limit) {
                            atomicOr(err, 1u);
                            cin = 0;
                            break;
                        }
                        __nanosleep(32);
                        continue;
                    }
                    if (f & FLAG_INC) {
                        uint32_t cj = (f >> 2) & 1u;
                        cin = gacc | (pacc & cj);
                        break;
                    }
                    uint32_t gj = (f >> 2) & 1u, pj = (f >> 3) & 1u;
                    gacc = gacc | (pacc & gj);
                    pacc = pacc & pj;
                    if (!pacc) {
                        cin = gacc;
                        break;
                    }
                    --jb;
                    if (jb < 0) {   // cannot happen: block 0 publishes inclusive
                        atomicOr(err, 4u);
                        cin = gacc;
                        break;
                    }
                }
            }
            uint32_t cout = (agg & 1u) | (((agg >> 1) & 1u) & cin);
            __threadfence();
            if (!((inj & SBG_INJECT_WITHHOLD) && bid == 0))     // injected: block 0 stays silent
                atomicExch(&flags[1 + bid], FLAG_INC | (cout << 2));
            s_cin = cin;
        }
    }
    __syncthreads();
    // warp carry-in, then each step's carries: into the lanes from the g, p
    // masks, into each lane's limbs from its own bits
    const uint32_t wpre = (wid > 0) ? s_warp[wid - 1] : 2u;
    uint32_t cin = (wpre & 1u) | ((wpre >> 1) & s_cin);
    const bool al16 = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
#pragma unroll
    for (int s = 0; s < NSTEP; ++s) {
        const uint32_t g = s_gp[wid][s][0], p = s_gp[wid][s][1];
        const uint64_t sum = (uint64_t)p + ((g << 1) | cin);
        const uint32_t c = (((uint32_t)sum ^ p) >> lane) & 1u;
        cin = (uint32_t)(sum >> 32) | (g >> 31);
        const uint32_t gb = (bits >> (8 * s)) & 15u, pb = (bits >> (8 * s + 4)) & 15u;
        const uint32_t cm = (pb + ((gb << 1) | c)) ^ pb;
        const ulonglong2 z01 = zs[(2 * s) * 32 + lane], z23 = zs[(2 * s + 1) * 32 + lane];
        const uint64_t z0 = z01.x + (cm & 1u), z1 = z01.y + ((cm >> 1) & 1u);
        const uint64_t z2 = z23.x + ((cm >> 2) & 1u), z3 = z23.y + ((cm >> 3) & 1u);
        const int64_t m0 = seg + 128 * s + 4 * lane;
        if (al16 && m0 + 3 < nout) {
            *reinterpret_cast<ulonglong2*>(out + m0) = make_ulonglong2(z0, z1);
            *reinterpret_cast<ulonglong2*>(out + m0 + 2) = make_ulonglong2(z2, z3);
        } else {
            if (m0 < nout) out[m0] = z0;
            if (m0 + 1 < nout) out[m0 + 1] = z1;
            if (m0 + 2 < nout) out[m0 + 2] = z2;
            if (m0 + 3 < nout) out[m0 + 3] = z3;
        }
        if (vpos >= CRT_V * s && vpos < CRT_V * (s + 1)) {
            const uint64_t zf = zv + ((cm >> (vpos - CRT_V * s)) & 1u);
            if (vbad | (zf != 0) | (zf < zv)) atomicOr(err, 2u);
        }
    }
}

// Block order comes from an atomic ticket (flags[0]), not blockIdx, so every
// block's look-back predecessors were scheduled before it.
__device__ __forceinline__ void crt_body(uint32_t bid, const uint32_t* __restrict__ R, int64_t L,
                                         int64_t cmin, int64_t cmax, int64_t off,
                                         uint64_t* __restrict__ out, int64_t nout,
                                         uint32_t* flags, uint32_t* err, CrtSmem& S) {
    crt_body_t<CRT_NSTEP>(bid, R, L, cmin, cmax, off, out, nout, flags, err, S);
}

__global__ void __launch_bounds__(CRT_T, CRT_MINB) k_crt_carry(const uint32_t* __restrict__ R, int64_t L,
                                                     int64_t cmin, int64_t cmax, int64_t off,
                                                     uint64_t* __restrict__ out, int64_t nout,
                                                     uint32_t* flags, uint32_t* err) {
    __shared__ uint32_t s_bid;
    if (threadIdx.x == 0) s_bid = atomicAdd(&flags[0], 1u);
    __syncthreads();
    __shared__ CrtSmem S;
    crt_body(s_bid, R, L, cmin, cmax, off, out, nout, flags, err, S);
}

// Short single products: one step of 128 limbs per warp (1024 limbs a
// block), four times the blocks of k_crt_carry, so a short carry scan is
// spread over more SMs (16384 x 16384 limbs: 14.7 -> 10.3 us); long ones
// keep four steps, which fetch and compose fewer neighbour terms per limb.
#define CRT_SHORT_NSTEP 1
#define CRT_SHORT_BLK ((CRT_T / 32) * 32 * CRT_V * CRT_SHORT_NSTEP)
#ifndef CRT_SHORT_MAX
#define CRT_SHORT_MAX (1 << 17)                 // product limbs up to which the short scan runs
#endif
__global__ void __launch_bounds__(CRT_T, CRT_MINB) k_crt_carry_s(const uint32_t* __restrict__ R, int64_t L,
                                                       int64_t cmin, int64_t cmax, int64_t off,
                                                       uint64_t* __restrict__ out, int64_t nout,
                                                       uint32_t* flags, uint32_t* err) {
    __shared__ uint32_t s_bid;
    if (threadIdx.x == 0) s_bid = atomicAdd(&flags[0], 1u);
    __syncthreads();
    __shared__ CrtSmemT<CRT_SHORT_NSTEP> S;
    crt_body_t<CRT_SHORT_NSTEP>(s_bid, R, L, cmin, cmax, off, out, nout, flags, err, S);
}

// batched: blocks_per_job CTAs per job (enough for the longest output of the
// launch); each takes a ticket on its own job's counter, surplus ones exit.
__global__ void __launch_bounds__(CRT_T, CRT_MINB) k_crt_carry_b(const JobDesc* __restrict__ jobs, int64_t L,
                                                       int blocks_per_job, uint32_t* err) {
    __shared__ uint32_t s_bid;
    const JobDesc& J = jobs[blockIdx.x / blocks_per_job];
    if (threadIdx.x == 0) s_bid = atomicAdd(&J.flags[0], 1u);
    __syncthreads();
    const int64_t need = (J.nout + 1 + CRT_BLK - 1) / CRT_BLK;
    if ((int64_t)s_bid >= need) return;
    __shared__ CrtSmem S;
    crt_body(s_bid, J.ws, L, J.cmin, J.cmax, J.off, J.out, J.nout, J.flags, err, S);
}

// ------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------
// per-device kernel attributes (called once per context, device current)
template <int LGN1>
static cudaError_t col_attr() {
    const int big = 200 * 1024;
    cudaError_t e = cudaFuncSetAttribute(k_col_fwd<LGN1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col_inv<LGN1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col_fwd_b<LGN1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col_inv_b<LGN1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (col_lgc(LGN1) > 3) {        // clusters of 16 CTAs
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_col_fwd<LGN1>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_col_inv<LGN1>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_col_fwd_b<LGN1>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_col_inv_b<LGN1>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    return e;
}

#define SBG_COL_CASES(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13)

template <int M3>
static cudaError_t col3s_attr() {
    const int big = 200 * 1024;
    cudaError_t e = cudaFuncSetAttribute(k_col3s_fwd<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col3s_inv<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col3s_fwd_b<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col3s_inv_b<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    return e;
}

template <int M3>
static cudaError_t col3_attr() {
    const int big = 200 * 1024;
    cudaError_t e = cudaFuncSetAttribute(k_col3_fwd<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col3_inv<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col3_fwd_b<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col3_inv_b<M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    return e;
}

int col_tiles(int lgN1) { return col_ntiles(lgN1); }

cudaError_t set_inject(uint32_t mask) { return cudaMemcpyToSymbol(g_inject, &mask, sizeof(mask)); }

cudaError_t set_kernel_attributes() {
    const int big = 200 * 1024;
    cudaError_t e = cudaSuccess;
#define SBG_ATTR(n) if (e == cudaSuccess) e = col_attr<n>();
    SBG_COL_CASES(SBG_ATTR)
#undef SBG_ATTR
#define SBG_ATTR3(n) if (e == cudaSuccess) e = col3_attr<n>();
    SBG_COL3_CASES(SBG_ATTR3)
#undef SBG_ATTR3
#define SBG_ATTR3S(n) if (e == cudaSuccess) e = col3s_attr<n>();
    SBG_COL3S_CASES(SBG_ATTR3S)
#undef SBG_ATTR3S
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_small, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_small_b, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    return e;
}

cudaError_t upload_constants(cudaStream_t st) {
    PrimeConst pc[SBG_NP];
    host_prime_consts(pc);
    CrtConst cc;
    host_crt_consts(&cc);
    cudaError_t e = cudaMemcpyToSymbolAsync(c_pr, pc, sizeof(pc), 0, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbolAsync(c_crt, &cc, sizeof(cc), 0, cudaMemcpyHostToDevice, st);
}

// roots of order `order` (a divisor of every p - 1: 2^a or 3 * 2^a, a <= 25)
static cudaError_t gen_table(uint2* out, int n, int64_t order, bool inverse, uint32_t stride,
                             cudaStream_t st, bool per_resolution = false) {
    uint32_t roots[SBG_NP];
    for (int q = 0; q < SBG_NP; ++q) {
        uint32_t p = kPrimes[q];
        uint32_t w = host_powmod(kGenerators[q], (p - 1) / (uint64_t)order, p);
        if (inverse) w = host_powmod(w, p - 2, p);
        roots[q] = w;
    }
    uint32_t* droots = nullptr;
    cudaError_t e = cudaMallocAsync(&droots, sizeof(roots), st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(droots, roots, sizeof(roots), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        dim3 grid((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024, SBG_NP);
        if (per_resolution)
            k_gen_res<<<grid, 256, 0, st>>>(out, droots);
        else
            k_gen_pow<<<grid, 256, 0, st>>>(out, n, droots, stride);
        e = cudaGetLastError();
    }
    cudaFreeAsync(droots, st);
    return e;
}

size_t master_table_entries() { return (size_t)SBG_NP * SBG_TW_N; }

cudaError_t gen_master_tables(uint2* tw_f, uint2* tw_i, cudaStream_t st) {
    cudaError_t e = gen_table(tw_f, SBG_TW_N, SBG_TW_N, false, 1, st, true);
    if (e != cudaSuccess) return e;
    return gen_table(tw_i, SBG_TW_N, SBG_TW_N, true, 1, st, true);
}

cudaError_t gen_len_tables(LenPlan* lp, cudaStream_t st) {
    // lo: w_L^e for e < 2^13; hi: w_L^(e * 2^13) for e < L / 2^13
    cudaError_t e = gen_table(lp->fs_lo_f, SBG_FS_LO_N, lp->L, false, 1, st);
    if (e == cudaSuccess) e = gen_table(lp->fs_lo_i, SBG_FS_LO_N, lp->L, true, 1, st);
    if (e == cudaSuccess)
        e = gen_table(lp->fs_hi_f, lp->hi_n, lp->L, false, SBG_FS_LO_N, st);
    if (e == cudaSuccess)
        e = gen_table(lp->fs_hi_i, lp->hi_n, lp->L, true, SBG_FS_LO_N, st);
    // radix-3 level: w_N1^j, j < 2M, N1 = 3M rows
    if (e == cudaSuccess && lp->m3 >= 0) {
        const int64_t n1 = (int64_t)3 << lp->m3;
        e = gen_table(lp->t3_f, 2 << lp->m3, n1, false, 1, st);
        if (e == cudaSuccess) e = gen_table(lp->t3_i, 2 << lp->m3, n1, true, 1, st);
    }
    return e;
}

size_t ws_words(int lgL, int sq) {
    if (lgL == SBG_CODE_SCHOOL) return 0;
    size_t L = (size_t)code_len(lgL);
    return (sq ? 1 : 2) * SBG_NP * L;
}

// Column kernels: COL_THREADS threads, dynamic shared memory, and a
// cluster of `cluster` CTAs when a column spans several slabs.
template <typename... KArgs, typename... Args>
static cudaError_t launch_colx(void (*kern)(KArgs...), int64_t blocks, int smem, int cluster,
                               cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks, 1, 1);
    cfg.blockDim = dim3(COL_THREADS, 1, 1);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = cluster > 1 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}
template <typename... KArgs, typename... Args>
static cudaError_t launch_col(void (*kern)(KArgs...), int lgN1, int64_t blocks, cudaStream_t st,
                              Args... args) {
    return launch_colx(kern, blocks, col_smem_bytes(lgN1), 1 << col_lgc(lgN1), st, args...);
}


static Radix3Arg radix3_arg(const LenPlan* lp, bool inverse) {
    Radix3Arg r{};
    r.t3 = inverse ? lp->t3_i : lp->t3_f;
    for (int q = 0; q < SBG_NP; ++q) {
        r.w[q] = inverse ? lp->w3i[q] : lp->w3f[q];
        r.ws[q] = inverse ? lp->w3is[q] : lp->w3fs[q];
    }
    return r;
}

cudaError_t launch_conv(const uint64_t* a, int64_t an, const uint64_t* b, int64_t bn, int sq,
                        int lgL, const LenPlan* lp, const uint2* tw_f, const uint2* tw_i,
                        uint32_t* ws, cudaStream_t st, KTimer* kt, cudaEvent_t b_ready) {
    const size_t L = (size_t)code_len(lgL);
    // the first operand's forward columns may start before the second
    // operand has arrived only on the power-of-two four-step path
    const bool split = b_ready && !sq && lgL > SBG_SMALL_MAX_LG && lp->m3 < 0;
    if (b_ready && !split) {
        cudaError_t e = cudaStreamWaitEvent(st, b_ready, 0);
        if (e != cudaSuccess) return e;
    }
    uint32_t* YA = ws;
    uint32_t* YB = ws + SBG_NP * L;
    ScaleArg sc;
    for (int q = 0; q < SBG_NP; ++q) {
        sc.w[q] = lp->scale[q].w;
        sc.ws[q] = lp->scale[q].ws;
    }
    if (lgL <= SBG_SMALL_MAX_LG) {
        size_t smem = (size_t)2 * padded_len((int)L) * 4;
        KT_BEGIN(kt, KID_SMALL, st);
        k_small<<<SBG_NP, 256, smem, st>>>(a, an, b, bn, sq, lgL, tw_f, tw_i, sc, YA);
        KT_END(kt, KID_SMALL, st);
        return cudaGetLastError();
    }
    const int lgN1 = lp->lgN1;   // rows: 2^lgN1 (or 3 * 2^m3), columns: 2^12
    const int m3 = lp->m3;
    FsTables fsf{lp->fs_lo_f, lp->fs_hi_f, lp->hi_n};
    FsTables fsi{lp->fs_lo_i, lp->fs_hi_i, lp->hi_n};
    const int nops = sq ? 1 : 2;
    cudaError_t e = cudaSuccess;
    if (m3 >= 0) {
        const Radix3Arg r3f = radix3_arg(lp, false), r3i = radix3_arg(lp, true);
        KT_BEGIN(kt, KID_COL_FWD, st);
        switch (m3) {
#define SBG_LAUNCH_F3S(n)                                                                          \
    case n:                                                                                        \
        e = launch_colx(k_col3s_fwd<n>, (int64_t)nops * col3s_ntiles(n) * SBG_NP, col3s_smem_bytes(n), 1, \
                        st, a, an, b, bn, tw_f, r3f, YA, YB);                                       \
        break;
            SBG_COL3S_CASES(SBG_LAUNCH_F3S)
#undef SBG_LAUNCH_F3S
#define SBG_LAUNCH_F3(n)                                                                          \
    case n:                                                                                       \
        e = launch_colx(k_col3_fwd<n>, (int64_t)nops * col3_ntiles(n) * SBG_NP * col3_csize(n),    \
                        col3_smem_bytes(n), col3_csize(n), st, a, an, b, bn, tw_f, r3f, YA, YB); \
        break;
            SBG_COL3_CASES(SBG_LAUNCH_F3)
#undef SBG_LAUNCH_F3
            default: return cudaErrorInvalidValue;
        }
        KT_END(kt, KID_COL_FWD, st);
        if (e != cudaSuccess) return e;
        KT_BEGIN(kt, KID_ROW, st);
        k_row12<<<(3 << m3) * SBG_NP, 256, 0, st>>>(YA, YB, sq, 0, m3, fsf, fsi, sc, tw_f, tw_i);
        KT_END(kt, KID_ROW, st);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        KT_BEGIN(kt, KID_COL_INV, st);
        switch (m3) {
#define SBG_LAUNCH_I3S(n)                                                                          \
    case n:                                                                                        \
        e = launch_colx(k_col3s_inv<n>, (int64_t)col3s_ntiles(n) * SBG_NP, col3s_smem_bytes(n), 1, st, YA, \
                        tw_i, r3i);                                                                 \
        break;
            SBG_COL3S_CASES(SBG_LAUNCH_I3S)
#undef SBG_LAUNCH_I3S
#define SBG_LAUNCH_I3(n)                                                                             \
    case n:                                                                                          \
        e = launch_colx(k_col3_inv<n>, (int64_t)col3_ntiles(n) * SBG_NP * col3_csize(n),               \
                        col3_smem_bytes(n), col3_csize(n), st, YA, tw_i, r3i);                        \
        break;
            SBG_COL3_CASES(SBG_LAUNCH_I3)
#undef SBG_LAUNCH_I3
            default: return cudaErrorInvalidValue;
        }
        KT_END(kt, KID_COL_INV, st);
        if (e != cudaSuccess) return e;
        return cudaGetLastError();
    }
    const int64_t col_blocks = ((int64_t)col_ntiles(lgN1) * SBG_NP) << col_lgc(lgN1);
    KT_BEGIN(kt, KID_COL_FWD, st);
    switch (lgN1) {
#define SBG_LAUNCH_F(n)                                                                          \
    case n:                                                                                      \
        if (split) {                                                                             \
            e = launch_col(k_col_fwd<n>, n, col_blocks, st, a, an, a, an, tw_f, YA, YA, 1);        \
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b_ready, 0);                        \
            if (e == cudaSuccess)                                                                \
                e = launch_col(k_col_fwd<n>, n, col_blocks, st, b, bn, b, bn, tw_f, YB, YB, 1);    \
        } else {                                                                                 \
            e = launch_col(k_col_fwd<n>, n, nops * col_blocks, st, a, an, b, bn, tw_f, YA, YB, nops); \
        }                                                                                        \
        break;
        SBG_COL_CASES(SBG_LAUNCH_F)
#undef SBG_LAUNCH_F
        default: return cudaErrorInvalidValue;
    }
    KT_END(kt, KID_COL_FWD, st);
    if (e != cudaSuccess) return e;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_ROW, st);
    k_row12<<<(1 << lgN1) * SBG_NP, 256, 0, st>>>(YA, YB, sq, lgN1, -1, fsf, fsi, sc, tw_f, tw_i);
    KT_END(kt, KID_ROW, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_COL_INV, st);
    switch (lgN1) {
#define SBG_LAUNCH_I(n) \
    case n: e = launch_col(k_col_inv<n>, n, col_blocks, st, YA, tw_i); break;
        SBG_COL_CASES(SBG_LAUNCH_I)
#undef SBG_LAUNCH_I
        default: return cudaErrorInvalidValue;
    }
    KT_END(kt, KID_COL_INV, st);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

int64_t crt_blocks(int64_t nout) { return (nout + 1 + CRT_BLK - 1) / CRT_BLK; }

cudaError_t launch_batch_class(const JobDesc* djobs, int njobs, int lgL, const LenPlan* lp,
                               const uint2* tw_f, const uint2* tw_i, int64_t max_nout,
                               uint32_t* flags, size_t flag_words, uint32_t* err,
                               cudaStream_t st, KTimer* kt) {
    if (njobs <= 0) return cudaSuccess;
    if (lgL == SBG_CODE_SCHOOL) {
        KT_BEGIN(kt, KID_BATCH, st);
        cudaError_t e = launch_school_batch(djobs, njobs, st);
        KT_END(kt, KID_BATCH, st);
        return e;
    }
    ScaleArg sc;
    for (int q = 0; q < SBG_NP; ++q) {
        sc.w[q] = lp->scale[q].w;
        sc.ws[q] = lp->scale[q].ws;
    }
    cudaError_t e = cudaMemsetAsync(flags, 0, flag_words * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_BATCH, st);
    if (lgL <= SBG_SMALL_MAX_LG) {
        size_t smem = (size_t)2 * padded_len(1 << lgL) * 4;
        k_small_b<<<njobs * SBG_NP, 256, smem, st>>>(djobs, lgL, tw_f, tw_i, sc);
    } else if (lp->m3 >= 0) {
        const int m3 = lp->m3;
        FsTables fsf{lp->fs_lo_f, lp->fs_hi_f, lp->hi_n};
        FsTables fsi{lp->fs_lo_i, lp->fs_hi_i, lp->hi_n};
        const Radix3Arg r3f = radix3_arg(lp, false), r3i = radix3_arg(lp, true);
        switch (m3) {
#define SBG_LAUNCH_FB3S(n)                                                                              \
    case n:                                                                                             \
        e = launch_colx(k_col3s_fwd_b<n>, (int64_t)njobs * 2 * col3s_ntiles(n) * SBG_NP, col3s_smem_bytes(n), \
                        1, st, djobs, tw_f, r3f);                                                        \
        break;
            SBG_COL3S_CASES(SBG_LAUNCH_FB3S)
#undef SBG_LAUNCH_FB3S
#define SBG_LAUNCH_FB3(n)                                                                       \
    case n:                                                                                     \
        e = launch_colx(k_col3_fwd_b<n>, (int64_t)njobs * 2 * col3_ntiles(n) * SBG_NP * col3_csize(n), \
                        col3_smem_bytes(n), col3_csize(n), st, djobs, tw_f, r3f);                \
        break;
            SBG_COL3_CASES(SBG_LAUNCH_FB3)
#undef SBG_LAUNCH_FB3
            default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
        k_row12_b<<<njobs * SBG_NP * (3 << m3), 256, 0, st>>>(djobs, 0, m3, fsf, fsi, sc, tw_f, tw_i);
        switch (m3) {
#define SBG_LAUNCH_IB3S(n)                                                                           \
    case n:                                                                                          \
        e = launch_colx(k_col3s_inv_b<n>, (int64_t)njobs * col3s_ntiles(n) * SBG_NP, col3s_smem_bytes(n), \
                        1, st, djobs, tw_i, r3i);                                                     \
        break;
            SBG_COL3S_CASES(SBG_LAUNCH_IB3S)
#undef SBG_LAUNCH_IB3S
#define SBG_LAUNCH_IB3(n)                                                                     \
    case n:                                                                                   \
        e = launch_colx(k_col3_inv_b<n>, (int64_t)njobs * col3_ntiles(n) * SBG_NP * col3_csize(n), \
                        col3_smem_bytes(n), col3_csize(n), st, djobs, tw_i, r3i);              \
        break;
            SBG_COL3_CASES(SBG_LAUNCH_IB3)
#undef SBG_LAUNCH_IB3
            default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
    } else {
        const int lgN1 = lp->lgN1;
        FsTables fsf{lp->fs_lo_f, lp->fs_hi_f, lp->hi_n};
        FsTables fsi{lp->fs_lo_i, lp->fs_hi_i, lp->hi_n};
        const int64_t col_blocks = ((int64_t)njobs * col_ntiles(lgN1) * SBG_NP) << col_lgc(lgN1);
        switch (lgN1) {
#define SBG_LAUNCH_FB(n) \
    case n: e = launch_col(k_col_fwd_b<n>, n, 2 * col_blocks, st, djobs, tw_f); break;
            SBG_COL_CASES(SBG_LAUNCH_FB)
#undef SBG_LAUNCH_FB
            default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
        k_row12_b<<<(njobs * SBG_NP) << lgN1, 256, 0, st>>>(djobs, lgN1, -1, fsf, fsi, sc, tw_f, tw_i);
        switch (lgN1) {
#define SBG_LAUNCH_IB(n) \
    case n: e = launch_col(k_col_inv_b<n>, n, col_blocks, st, djobs, tw_i); break;
            SBG_COL_CASES(SBG_LAUNCH_IB)
#undef SBG_LAUNCH_IB
            default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
    }
    const int bpj = (int)crt_blocks(max_nout);
    k_crt_carry_b<<<njobs * bpj, CRT_T, 0, st>>>(djobs, code_len(lgL), bpj, err);
    KT_END(kt, KID_BATCH, st);
    return cudaGetLastError();
}

// ticket + one flag per block + the error word's slot, for either block
// size; monotone in nout, so a workspace reserved for a product length
// covers every shorter one
size_t carry_flag_words(int64_t nout) {
    const int64_t nshort = nout < CRT_SHORT_MAX ? nout : CRT_SHORT_MAX;
    const int64_t b = std::max((nshort + CRT_SHORT_BLK) / CRT_SHORT_BLK, (nout + CRT_BLK) / CRT_BLK);
    return 1 + (size_t)b + 1;
}

cudaError_t launch_crt_carry(const uint32_t* R, int lgL, const LenPlan* lp, int64_t cmin,
                             int64_t cmax, int64_t off, uint64_t* out, int64_t nout,
                             uint32_t* flags, uint32_t* err, cudaStream_t st,
                             KTimer* kt) {
    (void)lp;
    // blocks cover limbs [0, nout] (limb nout is the spill check)
    const bool shortp = nout <= CRT_SHORT_MAX;
    const int64_t blk = shortp ? CRT_SHORT_BLK : CRT_BLK;
    int64_t nblk = (nout + 1 + blk - 1) / blk;
    cudaError_t e = cudaMemsetAsync(flags, 0, (1 + nblk) * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_CRT, st);
    if (shortp)
        k_crt_carry_s<<<(unsigned)nblk, CRT_T, 0, st>>>(R, code_len(lgL), cmin, cmax, off, out, nout, flags, err);
    else
        k_crt_carry<<<(unsigned)nblk, CRT_T, 0, st>>>(R, code_len(lgL), cmin, cmax, off, out, nout, flags, err);
    KT_END(kt, KID_CRT, st);
    return cudaGetLastError();
}

}  // namespace sbg

#include "sbg_school.cuh"
#include "sbg_persist.cuh"
