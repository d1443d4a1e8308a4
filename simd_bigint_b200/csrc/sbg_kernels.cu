// sbg_kernels.cu -- the transform pipeline of one product on the GPU.
//
//   u64 limbs --(K1 k_col_fwd: residues + column DIF + four-step twiddle)-->
//   spectra   --(K2 k_row: row DIF of A and B, pointwise, row DIT)-->
//   products  --(K3 k_col_inv: inverse twiddle + column DIT)-->
//   residues  --(K4 k_crt_carry: Garner CRT + 3-stream compose + carry scan)--> limbs
//
// Transforms of L <= 2^12 points skip the four-step split and run whole in
// one CTA per prime (k_small).  This is the reference's p30 pipeline
// (include/p30.h:1847-1938: input -> forward -> fused pointwise+inverse ->
// scale -> Garner/carry), laid out as a four-step NTT over HBM: every pass
// reads and writes each spectrum once, all levels inside a pass stay on chip.
#include "sbg_internal.h"
#include "sbg_ntt.cuh"

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

// Column tiles.  A CTA owns w adjacent columns (all N1 rows) of one operand
// and one prime: 2^14 points (fewer when N1 * N2 is smaller).  Each thread
// owns a PAIR of adjacent columns of one group per pass, so one twiddle load
// serves two columns and the global accesses are 16-byte (two limbs) or
// 8-byte (two residues) per row.  Columns live in shared memory as separate
// planes (padded one word per 16, plane stride COL_LD), and every stride is a
// compile-time constant of the column length.
__host__ __device__ constexpr int col_lgw(int lgN1) {
    return (14 - lgN1) > 12 ? 12 : ((14 - lgN1) < 1 ? 1 : (14 - lgN1));
}
__host__ __device__ constexpr int col_ld(int lgN1) { return padded_len(1 << lgN1) + 1; }
// Column radix schedule: passes of 16 from the top, the remainder (1..3
// levels) last.  (Measured alternatives on B200 at 2^25 points: a radix-32
// last pass spills under the 64-register cap, and the remainder first costs
// an extra shared-memory round trip in the forward kernel; both were slower.)
__host__ __device__ constexpr int col_np(int lg) { return num_passes(lg); }
__host__ __device__ constexpr int prl(int lg, int k) { return k < (lg >> 2) ? 4 : (lg & 3); }
__host__ __device__ constexpr int lgm_of(int lg, int k) {
    int m = lg;
    for (int i = 0; i < k; ++i) m -= prl(lg, i);
    return m;
}
__host__ __device__ constexpr int col_smem_bytes(int lgN1) {
    return col_np(lgN1) > 1 ? (1 << col_lgw(lgN1)) * col_ld(lgN1) * 4 : 0;
}

#define COL_THREADS 512

template <int LGST>
__device__ __forceinline__ int padded_at(int i0, int t) {
    constexpr int ST = 1 << LGST;
    if constexpr (LGST >= 4) {
        return pad_idx(i0) + t * (ST + (ST >> 4));
    } else {
        return pad_idx(i0 + ST * t);
    }
}

// Pass K (0-based, forward numbering) of the column transform.
template <int LGN1, int K, bool FWD>
__device__ __forceinline__ void col_pass_t(uint32_t* sm, const uint64_t* __restrict__ X,
                                           int64_t xn, uint32_t* __restrict__ Y, int c0,
                                           const uint2* __restrict__ tw, const PrimeConst& pc) {
    constexpr int NP = col_np(LGN1);
    constexpr int r = prl(LGN1, K);
    constexpr int R = 1 << r;
    constexpr int LGM = lgm_of(LGN1, K);
    constexpr int LGST = LGM - r;
    constexpr int ST = 1 << LGST;
    constexpr int LGW = col_lgw(LGN1);
    constexpr int LD = col_ld(LGN1);
    constexpr int TOTAL = (1 << (LGW - 1)) << (LGN1 - r);
    constexpr bool SRC_G = FWD ? (K == 0) : (K == NP - 1);
    constexpr bool DST_G = FWD ? (K == NP - 1) : (K == 0);
    const uint32_t p = pc.p;
    if constexpr (R == 32) {
        // single-column groups, column index fastest across lanes
        constexpr int TOT1 = 1 << (LGW + LGN1 - 5);
#pragma unroll 1
        for (int gid = threadIdx.x; gid < TOT1; gid += COL_THREADS) {
            const int g = gid & ((1 << LGW) - 1);
            const int rest = gid >> LGW;
            const int j0 = rest & (ST - 1);
            const int blk = rest >> LGST;
            const int i0 = (blk << LGM) + j0;
            uint32_t x[32];
            if constexpr (SRC_G) {
                const int64_t n0 = ((int64_t)i0 << SBG_ROW_LG) + c0 + g;
#pragma unroll
                for (int t = 0; t < 32; ++t) {
                    const int64_t n = n0 + ((int64_t)(ST * t) << SBG_ROW_LG);
                    if constexpr (FWD)
                        x[t] = n < xn ? limb_residue(__ldg(&X[n]), pc) : 0u;
                    else
                        x[t] = Y[n];
                }
            } else {
                const uint32_t* s0 = sm + g * LD;
#pragma unroll
                for (int t = 0; t < 32; ++t) x[t] = s0[padded_at<LGST>(i0, t)];
            }
            if constexpr (FWD)
                dif_regs<32>(x, tw, j0, ST, LGM, p);
            else
                dit_regs<32>(x, tw, j0, ST, LGM, p);
            if constexpr (DST_G) {
                const int64_t n0 = ((int64_t)i0 << SBG_ROW_LG) + c0 + g;
#pragma unroll
                for (int t = 0; t < 32; ++t) Y[n0 + ((int64_t)(ST * t) << SBG_ROW_LG)] = x[t];
            } else {
                uint32_t* s0 = sm + g * LD;
#pragma unroll
                for (int t = 0; t < 32; ++t) s0[padded_at<LGST>(i0, t)] = x[t];
            }
        }
    } else {
    // groups per thread is a compile-time constant (TOTAL / COL_THREADS, or 1
    // when the tile has fewer groups than threads): unrolled, so every
    // group's global loads are in flight together
    constexpr int ITER = TOTAL >= COL_THREADS ? TOTAL / COL_THREADS : 1;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int gid = threadIdx.x + it * COL_THREADS;
        if (TOTAL < COL_THREADS && gid >= TOTAL) break;
        const int j0 = gid & (ST - 1);
        const int rest = gid >> LGST;
        const int blk = rest & ((1 << (LGN1 - LGM)) - 1);
        const int cp = rest >> (LGN1 - LGM);
        const int i0 = (blk << LGM) + j0;
        const int g0 = 2 * cp;
        uint32_t x[R], y[R];
        if constexpr (SRC_G) {
            const int64_t n0 = ((int64_t)i0 << SBG_ROW_LG) + c0 + g0;
            if constexpr (FWD) {
                const bool al16 = (reinterpret_cast<uintptr_t>(X) & 15) == 0;
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    const int64_t n = n0 + ((int64_t)(ST * t) << SBG_ROW_LG);
                    if (al16 && n + 1 < xn) {
                        ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(X + n));
                        x[t] = limb_residue(v.x, pc);
                        y[t] = limb_residue(v.y, pc);
                    } else {
                        x[t] = n < xn ? limb_residue(__ldg(&X[n]), pc) : 0u;
                        y[t] = n + 1 < xn ? limb_residue(__ldg(&X[n + 1]), pc) : 0u;
                    }
                }
            } else {
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    const int64_t n = n0 + ((int64_t)(ST * t) << SBG_ROW_LG);
                    uint2 v = *reinterpret_cast<const uint2*>(Y + n);
                    x[t] = v.x;
                    y[t] = v.y;
                }
            }
        } else {
            const uint32_t* s0 = sm + g0 * LD;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int a = padded_at<LGST>(i0, t);
                x[t] = s0[a];
                y[t] = s0[LD + a];
            }
        }
        if constexpr (FWD)
            dif_regs2<R>(x, y, tw, j0, ST, LGM, p);
        else
            dit_regs2<R>(x, y, tw, j0, ST, LGM, p);
        if constexpr (DST_G) {
            const int64_t n0 = ((int64_t)i0 << SBG_ROW_LG) + c0 + g0;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int64_t n = n0 + ((int64_t)(ST * t) << SBG_ROW_LG);
                *reinterpret_cast<uint2*>(Y + n) = make_uint2(x[t], y[t]);
            }
        } else {
            uint32_t* s0 = sm + g0 * LD;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int a = padded_at<LGST>(i0, t);
                s0[a] = x[t];
                s0[LD + a] = y[t];
            }
        }
    }
    }
}

// K1: limbs -> residues -> column DIF (bit-reversed rows) for one operand,
// one prime, one tile.
template <int LGN1>
__device__ __forceinline__ void col_fwd_body(int q, int tile, int op,
                                             const uint64_t* __restrict__ a, int64_t an,
                                             const uint64_t* __restrict__ b, int64_t bn,
                                             const uint2* __restrict__ twf,
                                             uint32_t* __restrict__ YA,
                                             uint32_t* __restrict__ YB) {
    extern __shared__ uint32_t sm[];
    constexpr int NP = col_np(LGN1);
    constexpr int LGW = col_lgw(LGN1);
    const uint64_t* X = op ? b : a;
    const int64_t xn = op ? bn : an;
    uint32_t* Y = (op ? YB : YA) + ((size_t)q << (LGN1 + SBG_ROW_LG));
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twf + (size_t)q * SBG_TW_N;
    const int c0 = tile << LGW;
    col_pass_t<LGN1, 0, true>(sm, X, xn, Y, c0, tw, pc);
    if constexpr (NP > 1) {
        __syncthreads();
        col_pass_t<LGN1, (NP > 1 ? 1 : 0), true>(sm, X, xn, Y, c0, tw, pc);
    }
    if constexpr (NP > 2) {
        __syncthreads();
        col_pass_t<LGN1, (NP > 2 ? 2 : 0), true>(sm, X, xn, Y, c0, tw, pc);
    }
    if constexpr (NP > 3) {
        __syncthreads();
        col_pass_t<LGN1, (NP > 3 ? 3 : 0), true>(sm, X, xn, Y, c0, tw, pc);
    }
}

// K1: limbs -> residues -> column DIF (bit-reversed rows) for one operand,
// one prime, one tile.  Block order: prime slowest, so the CTAs resident on an
// SM share one prime's twiddles.
template <int LGN1>
__global__ void __launch_bounds__(512, 2) k_col_fwd(const uint64_t* __restrict__ a, int64_t an,
                                                    const uint64_t* __restrict__ b, int64_t bn,
                                                    const uint2* __restrict__ twf,
                                                    uint32_t* __restrict__ YA,
                                                    uint32_t* __restrict__ YB, int nops) {
    constexpr int NTILES = 1 << (SBG_ROW_LG - col_lgw(LGN1));
    const int per_q = NTILES * nops;
    const int q = blockIdx.x / per_q;
    const int rest = blockIdx.x - q * per_q;
    col_fwd_body<LGN1>(q, rest % NTILES, rest / NTILES, a, an, b, bn, twf, YA, YB);
}

// batched: blocks (job, prime, operand, tile), job slowest; the second
// operand's blocks of a squaring exit at once
template <int LGN1>
__global__ void __launch_bounds__(512, 2) k_col_fwd_b(const JobDesc* __restrict__ jobs,
                                                      const uint2* __restrict__ twf) {
    constexpr int NTILES = 1 << (SBG_ROW_LG - col_lgw(LGN1));
    constexpr int PER_JOB = SBG_NP * 2 * NTILES;
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    const int q = r / (2 * NTILES);
    const int r2 = r % (2 * NTILES);
    const int op = r2 / NTILES;
    if (op && J.sq) return;
    uint32_t* YB = J.ws + ((size_t)SBG_NP << (LGN1 + SBG_ROW_LG));
    col_fwd_body<LGN1>(q, r2 % NTILES, op, J.a, J.an, J.b, J.bn, twf, J.ws, YB);
}

// K3: column DIT (reverse of K1), in place, natural row order out.
template <int LGN1>
__device__ __forceinline__ void col_inv_body(int q, int tile, uint32_t* __restrict__ YA,
                                             const uint2* __restrict__ twi) {
    extern __shared__ uint32_t sm[];
    constexpr int NP = col_np(LGN1);
    constexpr int LGW = col_lgw(LGN1);
    uint32_t* Y = YA + ((size_t)q << (LGN1 + SBG_ROW_LG));
    const PrimeConst pc = c_pr[q];
    const uint2* tw = twi + (size_t)q * SBG_TW_N;
    const int c0 = tile << LGW;
    if constexpr (NP > 3) {
        col_pass_t<LGN1, (NP > 3 ? 3 : 0), false>(sm, nullptr, 0, Y, c0, tw, pc);
        __syncthreads();
    }
    if constexpr (NP > 2) {
        col_pass_t<LGN1, (NP > 2 ? 2 : 0), false>(sm, nullptr, 0, Y, c0, tw, pc);
        __syncthreads();
    }
    if constexpr (NP > 1) {
        col_pass_t<LGN1, (NP > 1 ? 1 : 0), false>(sm, nullptr, 0, Y, c0, tw, pc);
        __syncthreads();
    }
    col_pass_t<LGN1, 0, false>(sm, nullptr, 0, Y, c0, tw, pc);
}

template <int LGN1>
__global__ void __launch_bounds__(512, 2) k_col_inv(uint32_t* __restrict__ YA,
                                                    const uint2* __restrict__ twi) {
    constexpr int NTILES = 1 << (SBG_ROW_LG - col_lgw(LGN1));
    col_inv_body<LGN1>(blockIdx.x / NTILES, blockIdx.x % NTILES, YA, twi);
}

template <int LGN1>
__global__ void __launch_bounds__(512, 2) k_col_inv_b(const JobDesc* __restrict__ jobs,
                                                      const uint2* __restrict__ twi) {
    constexpr int NTILES = 1 << (SBG_ROW_LG - col_lgw(LGN1));
    constexpr int PER_JOB = SBG_NP * NTILES;
    const JobDesc& J = jobs[blockIdx.x / PER_JOB];
    const int r = blockIdx.x % PER_JOB;
    col_inv_body<LGN1>(r / NTILES, r % NTILES, J.ws, twi);
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
__device__ __forceinline__ void row_body(int q, int row, uint32_t* __restrict__ YA,
                                         const uint32_t* __restrict__ YB, int sq, int lgN1,
                                         const FsTables& fsf, const FsTables& fsi,
                                         const ScaleArg& sc, const uint2* __restrict__ twf,
                                         const uint2* __restrict__ twi) {
    __shared__ uint32_t smA[padded_len(ROW_N)];
    __shared__ uint32_t smB[padded_len(ROW_N)];
    __shared__ uint2 s_f[16];
    __shared__ uint2 s_i[16];
    const int tid = threadIdx.x;
    const PrimeConst pc = c_pr[q];
    const uint32_t p = pc.p;
    const uint32_t Lmask = (1u << (lgN1 + ROW_LG)) - 1u;
    const size_t base = ((size_t)q << (lgN1 + ROW_LG)) + ((size_t)row << ROW_LG);
    const uint2* tf = twf + (size_t)q * SBG_TW_N;
    const uint2* ti = twi + (size_t)q * SBG_TW_N;
    const uint32_t k1 = bitrev((uint32_t)row, lgN1);
    // four-step twiddles: w_L^(k1 (tid + 256 t)) = b * s^t
    if (tid < 16) {
        uint32_t e = (k1 * 256u * (uint32_t)tid) & Lmask;
        uint32_t v = fs_value(fsf, q, e, p);
        s_f[tid] = make_uint2(v, shoup_fast(v, pc));
        uint32_t vi = mul_shoup(fs_value(fsi, q, e, p), sc.w[q], sc.ws[q], p);
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
            xa[t] = mul_shoup(mul_shoup(Ar[tid + 256 * t], s.x, s.y, p), bf, bfs, p);
            if (!sq) xb[t] = mul_shoup(mul_shoup(__ldg(&Br[tid + 256 * t]), s.x, s.y, p), bf, bfs, p);
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
            dif_regs<16>(xa, tf, 0, 1, 4, p);
#pragma unroll
            for (int t = 0; t < 16; ++t) xa[t] = mont_mul(xa[t], xa[t], p, pc.pinv);
        } else {
            dif_regs2<16>(xa, xb, tf, 0, 1, 4, p);
#pragma unroll
            for (int t = 0; t < 16; ++t) xa[t] = mont_mul(xa[t], xb[t], p, pc.pinv);
        }
        dit_regs<16>(xa, ti, 0, 1, 4, p);
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

__global__ void __launch_bounds__(256, 4) k_row12(uint32_t* __restrict__ YA,
                                                  const uint32_t* __restrict__ YB, int sq,
                                                  int lgN1, FsTables fsf, FsTables fsi, ScaleArg sc,
                                                  const uint2* __restrict__ twf,
                                                  const uint2* __restrict__ twi) {
    row_body(blockIdx.x >> lgN1, blockIdx.x & ((1 << lgN1) - 1), YA, YB, sq, lgN1, fsf, fsi, sc,
             twf, twi);
}

// batched: blocks (job, prime, row), job slowest
__global__ void __launch_bounds__(256, 4) k_row12_b(const JobDesc* __restrict__ jobs, int lgN1,
                                                    FsTables fsf, FsTables fsi, ScaleArg sc,
                                                    const uint2* __restrict__ twf,
                                                    const uint2* __restrict__ twi) {
    const int per_job = SBG_NP << lgN1;
    const JobDesc& J = jobs[blockIdx.x / per_job];
    const int r = blockIdx.x % per_job;
    uint32_t* YB = J.ws + ((size_t)SBG_NP << (lgN1 + ROW_LG));
    row_body(r >> lgN1, r & ((1 << lgN1) - 1), J.ws, YB, J.sq, lgN1, fsf, fsi, sc, twf, twi);
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
// Each thread owns CRT_PER consecutive limbs, resolves the carries inside
// them assuming carry-in 0 and writes them; the carry-in of every thread is
// then found by a block scan plus a decoupled look-back across blocks (block
// order from an atomic ticket, so every predecessor is already resident),
// and threads whose carry-in is 1 ripple the +1 into their limbs.
// ------------------------------------------------------------------------
#define CRT_T 256
#define CRT_PER 16
#define CRT_BLK (CRT_T * CRT_PER)
#define LB_SPIN_LIMIT (1 << 22)
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

__device__ __forceinline__ void crt_body(uint32_t bid, const uint32_t* __restrict__ R, int lgL,
                                         int64_t cmin, int64_t cmax, int64_t off,
                                         uint64_t* __restrict__ out, int64_t nout,
                                         uint32_t* flags, uint32_t* err) {
    __shared__ uint32_t s_warp[CRT_T / 32];
    __shared__ uint32_t s_cin;
    const int64_t L = (int64_t)1 << lgL;
    const int64_t m0 = (int64_t)bid * CRT_BLK + (int64_t)threadIdx.x * CRT_PER;
    const int64_t j0 = m0 + off;
    // residues of coefficients j0-4 .. j0+15 arrive in 5 chunks of 4: one
    // 16-byte load per prime when aligned and in range, else guarded scalars
    const bool vec = ((j0 & 3) == 0) && (j0 >= 4) && (j0 + CRT_PER <= L);
    uint32_t rr[SBG_NP][4];
    auto fetch = [&](int c) {
        const int64_t jb = j0 - 4 + 4 * c;
        if (vec) {
#pragma unroll
            for (int q = 0; q < SBG_NP; ++q) {
                uint4 v = __ldg(reinterpret_cast<const uint4*>(R + (size_t)q * L + jb));
                rr[q][0] = v.x; rr[q][1] = v.y; rr[q][2] = v.z; rr[q][3] = v.w;
            }
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t j = jb + u;
                const bool in = j >= cmin && j <= cmax;
#pragma unroll
                for (int q = 0; q < SBG_NP; ++q) rr[q][u] = in ? __ldg(&R[(size_t)q * L + j]) : 0u;
            }
        }
    };
    auto coeff = [&](int u, int64_t j, uint64_t& lo, uint64_t& mid, uint32_t& hi) {
        if (j >= cmin && j <= cmax) {
            uint32_t r[SBG_NP];
#pragma unroll
            for (int q = 0; q < SBG_NP; ++q) r[q] = rr[q][u];
            garner(r, lo, mid, hi);
        } else {
            lo = 0; mid = 0; hi = 0;
        }
    };
    uint64_t lo_a, mid_a, lo_b, mid_b, lo_c, mid_c;   // a = j-2, b = j-1, c = j
    uint32_t hi_a, hi_b, hi_c;
    fetch(0);
    coeff(1, j0 - 3, lo_a, mid_a, hi_a);
    coeff(2, j0 - 2, lo_b, mid_b, hi_b);
    coeff(3, j0 - 1, lo_c, mid_c, hi_c);
    // kk of limb m0 - 1: S = lo_{j0-1} + mid_{j0-2} + hi_{j0-3}
    uint32_t kk_prev;
    {
        uint64_t s1 = lo_c + mid_b;
        uint32_t c1 = s1 < lo_c;
        uint64_t s2 = s1 + hi_a;
        c1 += s2 < s1;
        kk_prev = (m0 - 1 >= 0) ? c1 : 0u;
    }
    uint32_t carry = 0;         // in-thread carry, assuming thread carry-in 0
    uint32_t pmask = 0;         // bit k: z0_k == ~0
    int nreal = 0;              // limbs < nout owned and written
    bool has_v = false;         // owns limb nout (the spill limb, never stored)
    uint64_t zv = 0;
    uint32_t kv = 0;
#pragma unroll
    for (int k = 0; k < CRT_PER; ++k) {
        const int64_t m = m0 + k;
        if (m > nout) break;
        if ((k & 3) == 0) fetch(1 + (k >> 2));
        lo_a = lo_b; mid_a = mid_b; hi_a = hi_b;
        lo_b = lo_c; mid_b = mid_c; hi_b = hi_c;
        coeff(k & 3, j0 + k, lo_c, mid_c, hi_c);
        uint64_t s1 = lo_c + mid_b;
        uint32_t c1 = s1 < lo_c;
        uint64_t t = s1 + hi_a;
        c1 += t < s1;
        uint64_t y = t + kk_prev;
        uint32_t g = y < t;
        uint64_t z = y + carry;
        uint32_t g2 = z < y;
        kk_prev = c1;
        if (m == nout) {
            has_v = true;
            zv = z;
            kv = c1;
            break;
        }
        carry = g | g2;
        out[m] = z;
        if (z == ~0ull) pmask |= 1u << k;
        nreal = k + 1;
    }
    uint32_t P = (pmask == ((nreal == 32) ? ~0u : ((1u << nreal) - 1u))) ? 1u : 0u;
    uint32_t G = nreal > 0 ? carry : 0u;
    uint32_t gp = G | (P << 1);

    // block scan (exclusive) of gp
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = gp;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc = gp_compose(o, inc);
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
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
                while (true) {
                    uint32_t f = vf[jb];
                    if (f == 0) {
                        if (++spins > LB_SPIN_LIMIT) {
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
            atomicExch(&flags[1 + bid], FLAG_INC | (cout << 2));
            s_cin = cin;
        }
    }
    __syncthreads();
    // thread carry-in = exclusive prefix applied to the block carry-in
    uint32_t excl;
    {
        uint32_t prev_in_warp = __shfl_up_sync(0xffffffffu, inc, 1);
        uint32_t wpre = (wid > 0) ? s_warp[wid - 1] : 2u;
        excl = (lane > 0) ? gp_compose(wpre, prev_in_warp) : wpre;
    }
    uint32_t tcin = (excl & 1u) | (((excl >> 1) & 1u) & s_cin);
    for (int k = 0; k < nreal && tcin; ++k) {
        const int64_t m = m0 + k;
        if ((pmask >> k) & 1u) {
            out[m] = 0;
        } else {
            out[m] = out[m] + 1;
            tcin = 0;
        }
    }
    // limb nout must come out zero, with no carry beyond it
    if (has_v && ((zv | (uint64_t)tcin | (uint64_t)kv) != 0)) atomicOr(err, 2u);
}

// Block order comes from an atomic ticket (flags[0]), not blockIdx, so every
// block's look-back predecessors were scheduled before it.
__global__ void __launch_bounds__(CRT_T) k_crt_carry(const uint32_t* __restrict__ R, int lgL,
                                                     int64_t cmin, int64_t cmax, int64_t off,
                                                     uint64_t* __restrict__ out, int64_t nout,
                                                     uint32_t* flags, uint32_t* err) {
    __shared__ uint32_t s_bid;
    if (threadIdx.x == 0) s_bid = atomicAdd(&flags[0], 1u);
    __syncthreads();
    crt_body(s_bid, R, lgL, cmin, cmax, off, out, nout, flags, err);
}

// batched: blocks_per_job CTAs per job (enough for the longest output of the
// launch); each takes a ticket on its own job's counter, surplus ones exit.
__global__ void __launch_bounds__(CRT_T) k_crt_carry_b(const JobDesc* __restrict__ jobs, int lgL,
                                                       int blocks_per_job, uint32_t* err) {
    __shared__ uint32_t s_bid;
    const JobDesc& J = jobs[blockIdx.x / blocks_per_job];
    if (threadIdx.x == 0) s_bid = atomicAdd(&J.flags[0], 1u);
    __syncthreads();
    const int64_t need = (J.nout + 1 + CRT_BLK - 1) / CRT_BLK;
    if ((int64_t)s_bid >= need) return;
    crt_body(s_bid, J.ws, lgL, J.cmin, J.cmax, J.off, J.out, J.nout, J.flags, err);
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
    return e;
}

#define SBG_COL_CASES(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13)

cudaError_t set_kernel_attributes() {
    const int big = 200 * 1024;
    cudaError_t e = cudaSuccess;
#define SBG_ATTR(n) if (e == cudaSuccess) e = col_attr<n>();
    SBG_COL_CASES(SBG_ATTR)
#undef SBG_ATTR
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

static cudaError_t gen_table(uint2* out, int n, int lgRoot, bool inverse, uint32_t stride,
                             cudaStream_t st, bool per_resolution = false) {
    uint32_t roots[SBG_NP];
    for (int q = 0; q < SBG_NP; ++q) {
        uint32_t p = kPrimes[q];
        uint32_t w = host_powmod(kGenerators[q], (p - 1) >> lgRoot, p);
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
    cudaError_t e = gen_table(tw_f, SBG_TW_N, SBG_TW_LG, false, 1, st, true);
    if (e != cudaSuccess) return e;
    return gen_table(tw_i, SBG_TW_N, SBG_TW_LG, true, 1, st, true);
}

cudaError_t gen_len_tables(LenPlan* lp, cudaStream_t st) {
    // lo: w_L^e for e < 2^13; hi: w_L^(e * 2^13) for e < L / 2^13
    cudaError_t e = gen_table(lp->fs_lo_f, SBG_FS_LO_N, lp->lgL, false, 1, st);
    if (e == cudaSuccess) e = gen_table(lp->fs_lo_i, SBG_FS_LO_N, lp->lgL, true, 1, st);
    if (e == cudaSuccess)
        e = gen_table(lp->fs_hi_f, lp->hi_n, lp->lgL, false, SBG_FS_LO_N, st);
    if (e == cudaSuccess)
        e = gen_table(lp->fs_hi_i, lp->hi_n, lp->lgL, true, SBG_FS_LO_N, st);
    return e;
}

size_t ws_words(int lgL, int sq) {
    size_t L = (size_t)1 << lgL;
    return (sq ? 1 : 2) * SBG_NP * L;
}

cudaError_t launch_conv(const uint64_t* a, int64_t an, const uint64_t* b, int64_t bn, int sq,
                        int lgL, const LenPlan* lp, const uint2* tw_f, const uint2* tw_i,
                        uint32_t* ws, cudaStream_t st, KTimer* kt) {
    const size_t L = (size_t)1 << lgL;
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
    const int lgN1 = lp->lgN1;   // rows: 2^lgN1, columns: 2^12
    FsTables fsf{lp->fs_lo_f, lp->fs_hi_f, lp->hi_n};
    FsTables fsi{lp->fs_lo_i, lp->fs_hi_i, lp->hi_n};
    const int nops = sq ? 1 : 2;
    const int ntiles = 1 << (SBG_ROW_LG - col_lgw(lgN1));
    const size_t col_smem = (size_t)col_smem_bytes(lgN1);
    KT_BEGIN(kt, KID_COL_FWD, st);
    switch (lgN1) {
#define SBG_LAUNCH_F(n)                                                                  \
    case n:                                                                              \
        k_col_fwd<n><<<nops * ntiles * SBG_NP, 512, col_smem, st>>>(a, an, b, bn, tw_f, YA, \
                                                                    YB, nops);           \
        break;
        SBG_COL_CASES(SBG_LAUNCH_F)
#undef SBG_LAUNCH_F
        default: return cudaErrorInvalidValue;
    }
    KT_END(kt, KID_COL_FWD, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_ROW, st);
    k_row12<<<(1 << lgN1) * SBG_NP, 256, 0, st>>>(YA, YB, sq, lgN1, fsf, fsi, sc, tw_f, tw_i);
    KT_END(kt, KID_ROW, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_COL_INV, st);
    switch (lgN1) {
#define SBG_LAUNCH_I(n)                                                          \
    case n: k_col_inv<n><<<ntiles * SBG_NP, 512, col_smem, st>>>(YA, tw_i); break;
        SBG_COL_CASES(SBG_LAUNCH_I)
#undef SBG_LAUNCH_I
        default: return cudaErrorInvalidValue;
    }
    KT_END(kt, KID_COL_INV, st);
    return cudaGetLastError();
}

int64_t crt_blocks(int64_t nout) { return (nout + 1 + CRT_BLK - 1) / CRT_BLK; }

cudaError_t launch_batch_class(const JobDesc* djobs, int njobs, int lgL, const LenPlan* lp,
                               const uint2* tw_f, const uint2* tw_i, int64_t max_nout,
                               uint32_t* flags, size_t flag_words, uint32_t* err,
                               cudaStream_t st, KTimer* kt) {
    if (njobs <= 0) return cudaSuccess;
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
    } else {
        const int lgN1 = lp->lgN1;
        FsTables fsf{lp->fs_lo_f, lp->fs_hi_f, lp->hi_n};
        FsTables fsi{lp->fs_lo_i, lp->fs_hi_i, lp->hi_n};
        const int ntiles = 1 << (SBG_ROW_LG - col_lgw(lgN1));
        const size_t col_smem = (size_t)col_smem_bytes(lgN1);
        switch (lgN1) {
#define SBG_LAUNCH_FB(n)                                                              \
    case n:                                                                           \
        k_col_fwd_b<n><<<njobs * SBG_NP * 2 * ntiles, 512, col_smem, st>>>(djobs, tw_f); \
        break;
            SBG_COL_CASES(SBG_LAUNCH_FB)
#undef SBG_LAUNCH_FB
            default: return cudaErrorInvalidValue;
        }
        k_row12_b<<<(njobs * SBG_NP) << lgN1, 256, 0, st>>>(djobs, lgN1, fsf, fsi, sc, tw_f, tw_i);
        switch (lgN1) {
#define SBG_LAUNCH_IB(n)                                                           \
    case n: k_col_inv_b<n><<<njobs * SBG_NP * ntiles, 512, col_smem, st>>>(djobs, tw_i); break;
            SBG_COL_CASES(SBG_LAUNCH_IB)
#undef SBG_LAUNCH_IB
            default: return cudaErrorInvalidValue;
        }
    }
    const int bpj = (int)crt_blocks(max_nout);
    k_crt_carry_b<<<njobs * bpj, CRT_T, 0, st>>>(djobs, lgL, bpj, err);
    KT_END(kt, KID_BATCH, st);
    return cudaGetLastError();
}

size_t carry_flag_words(int64_t nout) { return 1 + (size_t)((nout + CRT_BLK) / CRT_BLK) + 1; }

cudaError_t launch_crt_carry(const uint32_t* R, int lgL, const LenPlan* lp, int64_t cmin,
                             int64_t cmax, int64_t off, uint64_t* out, int64_t nout,
                             uint32_t* flags, uint32_t* err, cudaStream_t st,
                             KTimer* kt) {
    (void)lp;
    // blocks cover limbs [0, nout] (limb nout is the spill check)
    int64_t nblk = (nout + 1 + CRT_BLK - 1) / CRT_BLK;
    cudaError_t e = cudaMemsetAsync(flags, 0, (1 + nblk) * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_CRT, st);
    k_crt_carry<<<(unsigned)nblk, CRT_T, 0, st>>>(R, lgL, cmin, cmax, off, out, nout, flags, err);
    KT_END(kt, KID_CRT, st);
    return cudaGetLastError();
}

}  // namespace sbg
