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

#define SBG_SMALL_MAX_LG 12
#define SBG_ROW_LG 12
#define SBG_COL_POINTS_LG 14     // points per column-pass CTA
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

// ------------------------------------------------------------------------
// K0: single-CTA product for L <= 2^12 (one CTA per prime)
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_small(const uint64_t* __restrict__ a, int64_t an,
                                               const uint64_t* __restrict__ b, int64_t bn, int sq,
                                               int lgL, const uint2* __restrict__ twf,
                                               const uint2* __restrict__ twi,
                                               uint32_t* __restrict__ R) {
    extern __shared__ uint32_t sm[];
    const int q = blockIdx.x;
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
        A[pad_idx(i)] = mont_mul(x, y, pc.p, pc.pinv);
    }
    __syncthreads();
    ntt_inverse(sm, ld, 1, lgL, twi + q * SBG_TW_N, pc.p);
    for (int i = threadIdx.x; i < L; i += blockDim.x) R[(size_t)q * L + i] = A[pad_idx(i)];
}

// ------------------------------------------------------------------------
// K1: limb unpack + column DIF + four-step twiddle.
// The length-L sequence is an N1 x N2 row-major matrix (n = n1*N2 + n2).
// A CTA owns w adjacent columns of one operand for one prime.
// ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t fs_twiddle(uint32_t v, uint32_t e, const uint2* lo,
                                               const uint2* hi, uint32_t p) {
    uint2 a = __ldg(&lo[e & (SBG_FS_LO_N - 1)]);
    uint2 b = __ldg(&hi[e >> SBG_FS_LO_LG]);
    return mul_shoup(mul_shoup(v, a.x, a.y, p), b.x, b.y, p);
}

__global__ void __launch_bounds__(512) k_col_fwd(const uint64_t* __restrict__ a, int64_t an,
                                                 const uint64_t* __restrict__ b, int64_t bn,
                                                 int lgN1, int lgN2, int lgw, FsTables fs,
                                                 const uint2* __restrict__ twf,
                                                 uint32_t* __restrict__ YA,
                                                 uint32_t* __restrict__ YB) {
    extern __shared__ uint32_t sm[];
    const int q = blockIdx.x % SBG_NP;
    const int rest = blockIdx.x / SBG_NP;
    const int ntiles = 1 << (lgN2 - lgw);
    const int tile = rest % ntiles;
    const int op = rest / ntiles;
    const uint64_t* X = op ? b : a;
    const int64_t xn = op ? bn : an;
    uint32_t* Y = (op ? YB : YA) + ((size_t)q << (lgN1 + lgN2));
    const PrimeConst pc = c_pr[q];
    const int w = 1 << lgw;
    const int ld = padded_len(1 << lgN1) + 1;
    const int c0 = tile << lgw;
    const int npts = 1 << (lgN1 + lgw);
    for (int idx = threadIdx.x; idx < npts; idx += blockDim.x) {
        int g = idx & (w - 1), i = idx >> lgw;
        int64_t n = ((int64_t)i << lgN2) + c0 + g;
        sm[g * ld + pad_idx(i)] = n < xn ? limb_residue(__ldg(&X[n]), pc) : 0u;
    }
    __syncthreads();
    ntt_forward(sm, ld, w, lgN1, twf + q * SBG_TW_N, pc.p);
    const uint2* lo = fs.lo + (size_t)q * SBG_FS_LO_N;
    const uint2* hi = fs.hi + (size_t)q * fs.hi_n;
    for (int idx = threadIdx.x; idx < npts; idx += blockDim.x) {
        int g = idx & (w - 1), i = idx >> lgw;
        uint32_t k1 = bitrev((uint32_t)i, lgN1);
        uint32_t n2 = (uint32_t)(c0 + g);
        uint32_t v = fs_twiddle(sm[g * ld + pad_idx(i)], k1 * n2, lo, hi, pc.p);
        Y[((size_t)i << lgN2) + n2] = v;
    }
}

// ------------------------------------------------------------------------
// K2: one row (N2 points) of one prime: forward DIF of A's and B's rows,
// pointwise Montgomery product, inverse DIT, written back over A.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_row(uint32_t* __restrict__ YA,
                                             const uint32_t* __restrict__ YB, int sq, int lgN1,
                                             int lgN2, const uint2* __restrict__ twf,
                                             const uint2* __restrict__ twi) {
    extern __shared__ uint32_t sm[];
    const int q = blockIdx.x % SBG_NP;
    const int row = blockIdx.x / SBG_NP;
    const PrimeConst pc = c_pr[q];
    const int N2 = 1 << lgN2;
    const int ld = padded_len(N2);
    const size_t base = ((size_t)q << (lgN1 + lgN2)) + ((size_t)row << lgN2);
    uint32_t* Ar = YA + base;
    const uint32_t* Br = YB + base;
    for (int i = threadIdx.x; i < N2; i += blockDim.x) {
        sm[pad_idx(i)] = Ar[i];
        if (!sq) sm[ld + pad_idx(i)] = __ldg(&Br[i]);
    }
    __syncthreads();
    ntt_forward(sm, ld, sq ? 1 : 2, lgN2, twf + q * SBG_TW_N, pc.p);
    for (int i = threadIdx.x; i < N2; i += blockDim.x) {
        uint32_t x = sm[pad_idx(i)];
        uint32_t y = sq ? x : sm[ld + pad_idx(i)];
        sm[pad_idx(i)] = mont_mul(x, y, pc.p, pc.pinv);
    }
    __syncthreads();
    ntt_inverse(sm, ld, 1, lgN2, twi + q * SBG_TW_N, pc.p);
    for (int i = threadIdx.x; i < N2; i += blockDim.x) Ar[i] = sm[pad_idx(i)];
}

// ------------------------------------------------------------------------
// K3: inverse four-step twiddle + column DIT, in place; natural order out.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_col_inv(uint32_t* __restrict__ YA, int lgN1, int lgN2,
                                                 int lgw, FsTables fs,
                                                 const uint2* __restrict__ twi) {
    extern __shared__ uint32_t sm[];
    const int q = blockIdx.x % SBG_NP;
    const int tile = blockIdx.x / SBG_NP;
    uint32_t* Y = YA + ((size_t)q << (lgN1 + lgN2));
    const PrimeConst pc = c_pr[q];
    const int w = 1 << lgw;
    const int ld = padded_len(1 << lgN1) + 1;
    const int c0 = tile << lgw;
    const int npts = 1 << (lgN1 + lgw);
    const uint2* lo = fs.lo + (size_t)q * SBG_FS_LO_N;
    const uint2* hi = fs.hi + (size_t)q * fs.hi_n;
    for (int idx = threadIdx.x; idx < npts; idx += blockDim.x) {
        int g = idx & (w - 1), i = idx >> lgw;
        uint32_t k1 = bitrev((uint32_t)i, lgN1);
        uint32_t n2 = (uint32_t)(c0 + g);
        uint32_t v = Y[((size_t)i << lgN2) + n2];
        sm[g * ld + pad_idx(i)] = fs_twiddle(v, k1 * n2, lo, hi, pc.p);
    }
    __syncthreads();
    ntt_inverse(sm, ld, w, lgN1, twi + q * SBG_TW_N, pc.p);
    for (int idx = threadIdx.x; idx < npts; idx += blockDim.x) {
        int g = idx & (w - 1), i = idx >> lgw;
        Y[((size_t)i << lgN2) + c0 + g] = sm[g * ld + pad_idx(i)];
    }
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

__device__ __forceinline__ void crt_coeff(const uint32_t* __restrict__ R, size_t L, int64_t j,
                                          const ScaleArg& sc, uint64_t& lo, uint64_t& mid,
                                          uint32_t& hi) {
    uint32_t v[SBG_NP];
#pragma unroll
    for (int q = 0; q < SBG_NP; ++q) {
        uint32_t p = c_pr[q].p;
        uint32_t r = __ldg(&R[(size_t)q * L + (size_t)j]);
        v[q] = mul_shoup(r, sc.w[q], sc.ws[q], p);
    }
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

__global__ void __launch_bounds__(CRT_T) k_crt_carry(const uint32_t* __restrict__ R, int lgL,
                                                     int64_t cmin, int64_t cmax, int64_t off,
                                                     uint64_t* __restrict__ out, int64_t nout,
                                                     ScaleArg sc, uint32_t* flags,
                                                     uint32_t* err) {
    __shared__ uint32_t s_bid;
    __shared__ uint32_t s_warp[CRT_T / 32];
    __shared__ uint32_t s_cin;
    const size_t L = (size_t)1 << lgL;
    if (threadIdx.x == 0) s_bid = atomicAdd(&flags[0], 1u);
    __syncthreads();
    const uint32_t bid = s_bid;
    const int64_t m0 = (int64_t)bid * CRT_BLK + (int64_t)threadIdx.x * CRT_PER;

    // sliding window over coefficients j = m + off - 2 .. m + off
    auto coeff = [&](int64_t j, uint64_t& lo, uint64_t& mid, uint32_t& hi) {
        if (j >= cmin && j <= cmax) {
            crt_coeff(R, L, j, sc, lo, mid, hi);
        } else {
            lo = 0; mid = 0; hi = 0;
        }
    };
    uint64_t lo_a, mid_a, lo_b, mid_b, lo_c, mid_c;   // a = j-2, b = j-1, c = j
    uint32_t hi_a, hi_b, hi_c;
    int64_t j0 = m0 + off;
    coeff(j0 - 3, lo_a, mid_a, hi_a);   // slot j-3 -> becomes "a" after shift below
    coeff(j0 - 2, lo_b, mid_b, hi_b);
    coeff(j0 - 1, lo_c, mid_c, hi_c);
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
#pragma unroll 1
    for (int k = 0; k < CRT_PER; ++k) {
        const int64_t m = m0 + k;
        if (m > nout) break;
        lo_a = lo_b; mid_a = mid_b; hi_a = hi_b;
        lo_b = lo_c; mid_b = mid_c; hi_b = hi_c;
        coeff(j0 + k, lo_c, mid_c, hi_c);
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

// ------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------
// per-device kernel attributes (called once per context, device current)
cudaError_t set_kernel_attributes() {
    const int big = 200 * 1024;
    cudaError_t e = cudaFuncSetAttribute(k_col_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_col_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_row, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_small, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
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
                             cudaStream_t st) {
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
        k_gen_pow<<<grid, 256, 0, st>>>(out, n, droots, stride);
        e = cudaGetLastError();
    }
    cudaFreeAsync(droots, st);
    return e;
}

cudaError_t gen_master_tables(uint2* tw_f, uint2* tw_i, cudaStream_t st) {
    cudaError_t e = gen_table(tw_f, SBG_TW_N, SBG_TW_LG, false, 1, st);
    if (e != cudaSuccess) return e;
    return gen_table(tw_i, SBG_TW_N, SBG_TW_LG, true, 1, st);
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
    if (lgL <= SBG_SMALL_MAX_LG) {
        size_t smem = (size_t)2 * padded_len((int)L) * 4;
        KT_BEGIN(kt, KID_SMALL, st);
        k_small<<<SBG_NP, 256, smem, st>>>(a, an, b, bn, sq, lgL, tw_f, tw_i, YA);
        KT_END(kt, KID_SMALL, st);
        return cudaGetLastError();
    }
    const int lgN2 = lp->lgN2, lgN1 = lp->lgN1;
    int lgw = SBG_COL_POINTS_LG - lgN1;
    if (lgw > lgN2) lgw = lgN2;
    if (lgw < 0) lgw = 0;
    const int ntiles = 1 << (lgN2 - lgw);
    FsTables fsf{lp->fs_lo_f, lp->fs_hi_f, lp->hi_n};
    FsTables fsi{lp->fs_lo_i, lp->fs_hi_i, lp->hi_n};
    size_t col_smem = (size_t)(1 << lgw) * (padded_len(1 << lgN1) + 1) * 4;
    int nops = sq ? 1 : 2;
    KT_BEGIN(kt, KID_COL_FWD, st);
    k_col_fwd<<<nops * ntiles * SBG_NP, 512, col_smem, st>>>(a, an, b, bn, lgN1, lgN2, lgw, fsf,
                                                             tw_f, YA, YB);
    KT_END(kt, KID_COL_FWD, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t row_smem = (size_t)2 * padded_len(1 << lgN2) * 4;
    KT_BEGIN(kt, KID_ROW, st);
    k_row<<<(1 << lgN1) * SBG_NP, 256, row_smem, st>>>(YA, YB, sq, lgN1, lgN2, tw_f, tw_i);
    KT_END(kt, KID_ROW, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_COL_INV, st);
    k_col_inv<<<ntiles * SBG_NP, 512, col_smem, st>>>(YA, lgN1, lgN2, lgw, fsi, tw_i);
    KT_END(kt, KID_COL_INV, st);
    return cudaGetLastError();
}

size_t carry_flag_words(int64_t nout) { return 1 + (size_t)((nout + CRT_BLK) / CRT_BLK) + 1; }

cudaError_t launch_crt_carry(const uint32_t* R, int lgL, const LenPlan* lp, int64_t cmin,
                             int64_t cmax, int64_t off, uint64_t* out, int64_t nout,
                             uint32_t* flags, uint32_t* err, cudaStream_t st,
                             KTimer* kt) {
    ScaleArg sc;
    for (int q = 0; q < SBG_NP; ++q) {
        sc.w[q] = lp->scale[q].w;
        sc.ws[q] = lp->scale[q].ws;
    }
    // blocks cover limbs [0, nout] (limb nout is the spill check)
    int64_t nblk = (nout + 1 + CRT_BLK - 1) / CRT_BLK;
    cudaError_t e = cudaMemsetAsync(flags, 0, (1 + nblk) * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    KT_BEGIN(kt, KID_CRT, st);
    k_crt_carry<<<(unsigned)nblk, CRT_T, 0, st>>>(R, lgL, cmin, cmax, off, out, nout, sc, flags,
                                                  err);
    KT_END(kt, KID_CRT, st);
    return cudaGetLastError();
}

}  // namespace sbg
