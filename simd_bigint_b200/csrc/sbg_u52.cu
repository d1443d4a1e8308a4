// sbg_u52.cu -- the u52 redundant-digit boundary: conversions between u64
// limbs and radix-2^52 digits held in 64-bit lanes, and a product whose
// operands and result are such digit arrays.
//
// The reference keeps its numbers inside the multiply and division code as
// radix-2^52 digits (the IFMA-friendly form) and converts at the boundary
// (include/u64cvt.h:1-58: decode u64 -> u52; include/canon.h:303-324: encode
// a redundant u52 array -- unsigned lanes, or signed lanes -- canonicalised
// and packed into u64 limbs).  Here the same boundary is a set of device
// kernels, so that code holding u52 digits (the reference's division layer)
// can call the GPU multiply without converting on the host:
//   * decode: digit i is bits [52 i, 52 i + 52) of the number -- a gather
//     of two limbs per digit, one thread per digit;
//   * encode: the value sum_i d_i 2^(52 i) of redundant digits is split into
//     three numbers whose bit fields do not overlap -- L (the low 52 bits of
//     every lane), H+ and H- (the positive and negative high parts
//     d_i >> 52, at bit 52 (i + 1)) -- each of which packs into u64 limbs
//     with shifts only; limb m of L + H+ - H- then takes a carry or borrow
//     k in {-1, 0, 1} from limb m - 1, and the ripple that k can start is
//     resolved by a scan whose elements are the maps {-1, 0, 1} -> {-1, 0, 1}
//     each limb applies to an incoming ripple (composition is associative):
//     per-block aggregates, one block scanning the aggregates, then every
//     block applies its carry-in.  Three launches, no inter-block waits.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/simd_bigint_b200.h"
#include "sbg_internal.h"

namespace sbg {

#define U52_T 256                           // threads per block
#define U52_V 4                             // consecutive limbs per thread
#define U52_BLK (U52_T * U52_V)             // limbs per block
#define U52_MASK ((1ull << 52) - 1)

// ---- decode ------------------------------------------------------------------
__global__ void k_u52_decode(uint64_t* __restrict__ d, int64_t n52, const uint64_t* __restrict__ a,
                             int64_t an) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n52;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t bit = 52 * i;
        const int64_t w = bit >> 6;
        const int s = (int)(bit & 63);
        const uint64_t lo = w < an ? a[w] : 0ull;
        const uint64_t hi = (s > 12 && w + 1 < an) ? a[w + 1] : 0ull;
        d[i] = ((lo >> s) | (s > 12 ? hi << (64 - s) : 0ull)) & U52_MASK;
    }
}

// ---- encode ------------------------------------------------------------------
// A ripple map f: {-1, 0, 1} -> {-1, 0, 1} as three 2-bit fields holding
// f(x) + 1 for x = -1, 0, 1.
#define MAP_ID (0u | (1u << 2) | (2u << 4))
__device__ __forceinline__ int map_apply(uint32_t f, int x) { return (int)((f >> (2 * (x + 1))) & 3u) - 1; }
// (g after f)(x) = g(f(x))
__device__ __forceinline__ uint32_t map_then(uint32_t f, uint32_t g) {
    uint32_t h = 0;
#pragma unroll
    for (int x = -1; x <= 1; ++x) h |= (uint32_t)(map_apply(g, map_apply(f, x)) + 1) << (2 * (x + 1));
    return h;
}

// The bits of limb m of a number whose fields of `width` bits start at bit
// `pos0 + 52 i` with values v_i (i < n): fields i0 .. i1 can touch the limb.
__device__ __forceinline__ uint64_t place(uint64_t v, int64_t pos, int64_t m) {
    const int64_t sh = pos - 64 * m;
    if (sh >= 64 || sh <= -64) return 0ull;
    return sh >= 0 ? v << sh : v >> (-sh);
}

// L_m, H+_m, H-_m of limb m, then t_m = L + H+ - H- (mod 2^64) and the carry
// k_m in {-1, 0, 1} it hands to limb m + 1
__device__ __forceinline__ void limb_parts(const uint64_t* __restrict__ d, int64_t n52, int sgn,
                                           int64_t m, uint64_t& t, int& k) {
    uint64_t L = 0, Hp = 0, Hn = 0;
    if (m >= 0) {
        // lo fields [52 i, 52 i + 52) touching [64 m, 64 m + 64): i from
        // floor((64 m - 51) / 52) to floor((64 m + 63) / 52); high fields
        // start at 52 (i + 1), so one digit further down reaches the limb
        const int64_t i0 = max((int64_t)0, (64 * m - 51 - 52) / 52);
        const int64_t i1 = min(n52 - 1, (64 * m + 63) / 52);
        for (int64_t i = i0; i <= i1; ++i) {
            const uint64_t x = d[i];
            L |= place(x & U52_MASK, 52 * i, m);
            if (sgn) {
                const int64_t h = (int64_t)x >> 52;            // [-2^11, 2^11)
                if (h > 0) Hp |= place((uint64_t)h, 52 * (i + 1), m);
                if (h < 0) Hn |= place((uint64_t)(-h), 52 * (i + 1), m);
            } else {
                Hp |= place(x >> 52, 52 * (i + 1), m);
            }
        }
    }
    const uint64_t s = L + Hp;
    const int c1 = s < L;
    t = s - Hn;
    const int b1 = s < Hn;
    k = c1 - b1;
}

// z_m = t_m + k_{m-1} and the map limb m applies to an incoming ripple r:
// out = g + (z + r overflow: +1 / underflow: -1), g the carry of t + k
__device__ __forceinline__ uint32_t limb_map(uint64_t t, int kprev, uint64_t& z) {
    z = t + (uint64_t)(int64_t)kprev;
    int g = 0;
    if (kprev > 0 && z == 0) g = 1;
    if (kprev < 0 && z == ~0ull) g = -1;
    uint32_t f = 0;
#pragma unroll
    for (int r = -1; r <= 1; ++r) {
        int o = g;
        if (r > 0 && z == ~0ull) o += 1;
        if (r < 0 && z == 0) o -= 1;
        f |= (uint32_t)(o + 1) << (2 * (r + 1));
    }
    return f;
}

// a thread's U52_V limbs: values z and the composed map
__device__ __forceinline__ uint32_t thread_limbs(const uint64_t* __restrict__ d, int64_t n52, int sgn,
                                                 int64_t m0, uint64_t (&z)[U52_V], uint32_t (&fm)[U52_V]) {
    uint64_t t;
    int kprev;
    limb_parts(d, n52, sgn, m0 - 1, t, kprev);
    uint32_t f = MAP_ID;
#pragma unroll
    for (int v = 0; v < U52_V; ++v) {
        int k;
        limb_parts(d, n52, sgn, m0 + v, t, k);
        fm[v] = limb_map(t, kprev, z[v]);
        f = map_then(f, fm[v]);
        kprev = k;
    }
    return f;
}

// inclusive scan of maps over the block's threads (thread order = limb order)
__device__ __forceinline__ uint32_t block_scan_maps(uint32_t f, uint32_t* s_w, uint32_t& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t g = __shfl_up_sync(0xffffffffu, f, o);
        if (lane >= o) f = map_then(g, f);
    }
    if (lane == 31) s_w[wid] = f;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < U52_T / 32 ? s_w[lane] : MAP_ID;
#pragma unroll
        for (int o = 1; o < U52_T / 32; o <<= 1) {
            const uint32_t g = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w = map_then(g, w);
        }
        if (lane < U52_T / 32) s_w[lane] = w;
    }
    __syncthreads();
    if (wid > 0) f = map_then(s_w[wid - 1], f);
    total = s_w[U52_T / 32 - 1];
    return f;
}

__global__ void __launch_bounds__(U52_T) k_u52_encode_agg(const uint64_t* __restrict__ d, int64_t n52,
                                                         int sgn, int64_t rn, uint32_t* __restrict__ agg) {
    __shared__ uint32_t s_w[U52_T / 32];
    const int64_t m0 = (int64_t)blockIdx.x * U52_BLK + (int64_t)threadIdx.x * U52_V;
    uint64_t z[U52_V];
    uint32_t fm[U52_V];
    uint32_t f = m0 < rn ? thread_limbs(d, n52, sgn, m0, z, fm) : MAP_ID;
    uint32_t total;
    block_scan_maps(f, s_w, total);
    if (threadIdx.x == 0) agg[blockIdx.x] = total;
}

// one block: the ripple carry into every block from the block aggregates
// (in place: agg[i] becomes carry-in + 1), 1024 aggregates per round
__global__ void __launch_bounds__(1024) k_u52_encode_scan(uint32_t* __restrict__ agg, int64_t nblk) {
    __shared__ uint32_t s_w[32];
    __shared__ int s_carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nblk; base += 1024) {
        const int64_t i = base + threadIdx.x;
        uint32_t x = i < nblk ? agg[i] : MAP_ID;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t g = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x = map_then(g, x);
        }
        if (lane == 31) s_w[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint32_t w = s_w[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t g = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w = map_then(g, w);
            }
            s_w[lane] = w;
        }
        __syncthreads();
        // inclusive map through block i; the carry into block i is the
        // carry out of block i - 1
        const uint32_t incl = wid > 0 ? map_then(s_w[wid - 1], x) : x;
        const int cin = s_carry;
        const int out_incl = map_apply(incl, cin);
        int into = __shfl_up_sync(0xffffffffu, out_incl, 1);
        if (lane == 0) into = wid > 0 ? map_apply(s_w[wid - 1], cin) : cin;
        if (i < nblk) agg[i] = (uint32_t)(into + 1);
        __syncthreads();
        if (threadIdx.x == 0) s_carry = map_apply(s_w[31], cin);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(U52_T) k_u52_encode_out(const uint64_t* __restrict__ d, int64_t n52,
                                                         int sgn, uint64_t* __restrict__ r, int64_t rn,
                                                         const uint32_t* __restrict__ cin_blk) {
    __shared__ uint32_t s_w[U52_T / 32];
    const int64_t m0 = (int64_t)blockIdx.x * U52_BLK + (int64_t)threadIdx.x * U52_V;
    uint64_t z[U52_V] = {};
    uint32_t fm[U52_V] = {};
    uint32_t f = m0 < rn ? thread_limbs(d, n52, sgn, m0, z, fm) : MAP_ID;
    uint32_t total;
    const uint32_t incl = block_scan_maps(f, s_w, total);
    const int bc = (int)cin_blk[blockIdx.x] - 1;
    // carry into this thread's first limb: the block's carry-in through the
    // maps of the threads before it
    const uint32_t excl_prev = __shfl_up_sync(0xffffffffu, incl, 1);
    int c;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane > 0)
        c = map_apply(excl_prev, bc);
    else
        c = wid > 0 ? map_apply(s_w[wid - 1], bc) : bc;
    if (m0 >= rn) return;
#pragma unroll
    for (int v = 0; v < U52_V; ++v) {
        if (m0 + v < rn) r[m0 + v] = z[v] + (uint64_t)(int64_t)c;
        c = map_apply(fm[v], c);
    }
}

cudaError_t launch_u52_decode(uint64_t* d, int64_t n52, const uint64_t* a, int64_t an, cudaStream_t st) {
    if (n52 <= 0) return cudaSuccess;
    const int64_t blocks = std::min<int64_t>((n52 + 255) / 256, 148 * 16);
    k_u52_decode<<<(unsigned)blocks, 256, 0, st>>>(d, n52, a, an);
    return cudaGetLastError();
}

size_t u52_encode_scratch_words(int64_t rn) { return (size_t)((rn + U52_BLK - 1) / U52_BLK) + 1; }

cudaError_t launch_u52_encode(uint64_t* r, int64_t rn, const uint64_t* d, int64_t n52, int sgn,
                              uint32_t* scratch, cudaStream_t st) {
    if (rn <= 0) return cudaSuccess;
    const int64_t nblk = (rn + U52_BLK - 1) / U52_BLK;
    k_u52_encode_agg<<<(unsigned)nblk, U52_T, 0, st>>>(d, n52, sgn, rn, scratch);
    k_u52_encode_scan<<<1, 1024, 0, st>>>(scratch, nblk);
    k_u52_encode_out<<<(unsigned)nblk, U52_T, 0, st>>>(d, n52, sgn, r, rn, scratch);
    return cudaGetLastError();
}

}  // namespace sbg

// ---- C ABI ---------------------------------------------------------------------
using namespace sbg;

static int u52_fail(cudaError_t e) {
    if (e == cudaSuccess) return SBG_OK;
    return e == cudaErrorMemoryAllocation ? SBG_EALLOC : SBG_ECUDA;
}

// the context's grow-only boundary scratch, at least `words` u64
static int u52_scratch(sbg_ctx* c, size_t words, uint64_t** out) {
    if (words > c->u52cap) {
        cudaError_t e = cudaStreamSynchronize(c->stream);     // earlier calls may still use it
        if (e != cudaSuccess) return SBG_ECUDA;
        cudaFree(c->u52buf);
        c->u52buf = nullptr;
        c->u52cap = 0;
        const size_t nw = words + words / 4;
        e = dev_alloc((void**)&c->u52buf, nw * sizeof(uint64_t));
        if (e != cudaSuccess) return u52_fail(e);
        c->u52cap = nw;
    }
    *out = c->u52buf;
    return SBG_OK;
}

extern "C" int sbg_u52_from_u64(sbg_ctx* c, uint64_t* dp, int64_t n52, const uint64_t* ap, int64_t an) {
    if (!c || !dp || n52 <= 0 || an < 0 || (an > 0 && !ap)) return SBG_EINVAL;
    if (cudaSetDevice(c->device) != cudaSuccess) return SBG_ECUDA;
    int st = u52_fail(launch_u52_decode(dp, n52, ap, an, c->stream));
    if (!st) c->launches += 1;
    return st;
}

extern "C" int sbg_u64_from_u52(sbg_ctx* c, uint64_t* rp, int64_t rn, const uint64_t* dp, int64_t n52,
                                int is_signed) {
    if (!c || !rp || rn <= 0 || n52 < 0 || (n52 > 0 && !dp)) return SBG_EINVAL;
    if (cudaSetDevice(c->device) != cudaSuccess) return SBG_ECUDA;
    uint64_t* scr = nullptr;
    int st = u52_scratch(c, u52_encode_scratch_words(rn) / 2 + 1, &scr);
    if (st) return st;
    st = u52_fail(launch_u52_encode(rp, rn, dp, n52, is_signed ? 1 : 0, (uint32_t*)scr, c->stream));
    if (!st) c->launches += 3;
    return st;
}

extern "C" int sbg_mul_u52(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an52, const uint64_t* bp,
                           int64_t bn52) {
    if (!c || !rp || !ap || !bp || an52 <= 0 || bn52 <= 0) return SBG_EINVAL;
    const int64_t an = (52 * an52 + 63) / 64, bn = (52 * bn52 + 63) / 64;
    if (an + bn - 1 > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
    if (cudaSetDevice(c->device) != cudaSuccess) return SBG_ECUDA;
    const size_t scan = u52_encode_scratch_words(std::max(an, bn)) / 2 + 1;
    uint64_t* buf = nullptr;
    int st = u52_scratch(c, (size_t)2 * (an + bn) + scan, &buf);
    if (st) return st;
    uint64_t* A = buf;
    uint64_t* B = A + an;
    uint64_t* P = B + bn;
    uint32_t* sc = (uint32_t*)(P + an + bn);
    st = u52_fail(launch_u52_encode(A, an, ap, an52, 0, sc, c->stream));
    if (!st) st = u52_fail(launch_u52_encode(B, bn, bp, bn52, 0, sc, c->stream));
    if (st) return st;
    c->launches += 6;
    st = sbg_mul(c, P, A, an, B, bn);
    if (st) return st;
    st = u52_fail(launch_u52_decode(rp, an52 + bn52, P, an + bn, c->stream));
    if (!st) c->launches += 1;
    return st;
}
