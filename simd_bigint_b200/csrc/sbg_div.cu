// sbg_div.cu -- Newton reciprocal and division on top of the GPU products.
//
// Reciprocal: the Newton iteration for an n-limb normalised divisor D
// (B = 2^64, B^n/2 <= D < B^n), as the reference's division prototypes
// specify it (bench/recip_mulmid_ref.c:51-116, bench/mpinv_mulmid_verify.c:
// 27-45: X_h from the top h limbs, residual of D * X_h, correction
// x_hi * residual / B^k, h -> n = 2h).  We follow the "approximate
// reciprocal" formulation of Brent and Zimmermann (Modern Computer
// Arithmetic, Algorithm 3.5): with l = floor((n-1)/2), h = n - l,
//     X_h = R(top h limbs of D)
//     T   = D * X_h;   while T >= B^(n+h): X_h -= 1, T -= D   (at most 4 times)
//     T_m = floor((B^(n+h) - T) / B^l)
//     U   = T_m * X_h
//     X   = X_h * B^l + floor(U / B^(2h-l))
// which keeps D X < B^2n <= D (X + 2) at every level.  The base case (at
// most SBG_DIV_BASE limbs) is an exact long division, one warp per divisor
// (block division with 3-by-2 quotient estimates; divisions whose divisor is
// that short skip the Newton path altogether).  Every product runs on the batch engine, so all divisions of a
// batch advance one recursion level per round.
//
// Division of a 2n-limb N by D: Q0 = N_hi + floor(N_hi * (X - B^n) / B^n)
// (within 5 of floor(N / D)), R = N - Q0 D, then at most five (R -= D, Q += 1)
// steps.  The linear steps (borrow/carry chains, compares) run one CTA per
// division with a block-wide carry scan.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/simd_bigint_b200.h"
#include "sbg_internal.h"

namespace sbg {
namespace cg = cooperative_groups;

#define DIV_T 1024           // threads of the per-division linear kernels
#define DIV_PER 8            // limbs per thread per tile
#define DIV_TILE (DIV_T * DIV_PER)
// Divisions with n >= DIV_CL_MIN_N run their linear steps on a thread-block
// cluster of DIV_CL CTAs (one CTA otherwise): limb tiles go to the CTAs in
// turn, and the cluster-wide carries and decisions are combined through
// distributed shared memory, so the largest divisions -- the last Newton
// rounds, where few divisions remain -- spread over DIV_CL SMs.
#define DIV_CL 8
#define DIV_CL_MIN_N 32768

// The CTA group of one division: its rank, a barrier over all of its
// threads (release / acquire: global and shared memory written before it
// are visible after it), and cross-CTA exchange slots.  Every CTA of a
// group takes the same path through a kernel, so the slots' parity stays in
// step; a slot is rewritten only two exchanges later, after a barrier that
// follows every CTA's reads of it.
template <int CL>
struct Grp {
    long long* slot;        // two words of the kernel's shared memory
    int par = 0;
    unsigned rank = 0;
    __device__ explicit Grp(long long* s) : slot(s) {
        if constexpr (CL > 1) rank = cg::this_cluster().block_rank();
    }
    __device__ void sync() {
        if constexpr (CL == 1) {
            __syncthreads();
        } else {
            asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
            asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
        }
    }
    // publish this CTA's value (uniform in the CTA), then value k of CTA k
    __device__ const long long* publish(long long v) {
        long long* s = slot + par;
        if (threadIdx.x == 0) *s = v;
        sync();
        par ^= 1;
        return s;
    }
    __device__ long long peer(const long long* s, int k) const {
        if constexpr (CL == 1) {
            return *s;
        } else {
            return *cg::this_cluster().map_shared_rank(s, k);
        }
    }
    __device__ long long max_all(long long v) {
        if constexpr (CL == 1) return v;
        const long long* s = publish(v);
        long long r = peer(s, 0);
        for (int k = 1; k < CL; ++k) r = max(r, peer(s, k));
        return r;
    }
    __device__ long long min_all(long long v) {
        if constexpr (CL == 1) return v;
        const long long* s = publish(v);
        long long r = peer(s, 0);
        for (int k = 1; k < CL; ++k) r = min(r, peer(s, k));
        return r;
    }
};

// ---------------------------------------------------------------------------
// group-wide multi-limb add / sub with carry scan
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t gp2(uint32_t left, uint32_t right) {
    uint32_t gl = left & 1, pl = (left >> 1) & 1, gr = right & 1, pr = (right >> 1) & 1;
    return (gr | (pr & gl)) | ((pr & pl) << 1);
}

// Carries of one tile: the rows' generate / propagate masks g[k], p[k]
// (lane l = limb k * 32 + l of this warp's rows) and the group's carry into
// the tile give cm[k], the carries into every limb as a lane mask; returns
// the carry out of the tile (group-uniform).  Per row, with carry-in c, the
// carries into the 32 limbs are (p + (g << 1 | c)) ^ p and the row passes on
// (p + (g << 1 | c)) >> 32 | g >> 31.  The rows' (G, P) compose to the
// warp's, a block scan of the warps' gives the CTA's, and the CTAs'
// aggregates, composed in rank order, give each CTA its carry-in.
template <int CL, int R>
__device__ uint32_t tile_carries(Grp<CL>& grp, const uint32_t (&g)[R], const uint32_t (&p)[R],
                                 uint32_t carry, uint32_t (&cm)[R]) {
    __shared__ uint32_t s_w[DIV_T / 32];
    __shared__ uint32_t s_tot;
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t wG = 0, wP = 1;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t rG = (uint32_t)(((uint64_t)p[k] + (g[k] << 1)) >> 32) | (g[k] >> 31);
        const uint32_t rP = p[k] == FULL;
        wG = rG | (rP & wG);
        wP = rP & wP;
    }
    if (lane == 0) s_w[wid] = wG | (wP << 1);
    __syncthreads();
    if (wid == 0) {
        uint32_t iv = lane < DIV_T / 32 ? s_w[lane] : 2u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(FULL, iv, d);
            if (lane >= d) iv = gp2(o, iv);
        }
        if (lane < DIV_T / 32) s_w[lane] = iv;     // inclusive warp prefixes
        if (lane == 31) s_tot = iv;
    }
    __syncthreads();
    uint32_t cta_cin = carry, next;
    if constexpr (CL == 1) {
        const uint32_t tot = s_tot;
        next = (tot & 1u) | ((tot >> 1) & carry);
    } else {
        const long long* sl = grp.publish(s_tot);
        uint32_t pre = 2u, all = 2u;
        for (int k = 0; k < CL; ++k) {
            const uint32_t v = (uint32_t)grp.peer(sl, k);
            if (k < (int)grp.rank) pre = gp2(pre, v);
            all = gp2(all, v);
        }
        cta_cin = (pre & 1u) | ((pre >> 1) & carry);
        next = (all & 1u) | ((all >> 1) & carry);
    }
    const uint32_t wpre = wid > 0 ? s_w[wid - 1] : 2u;
    uint32_t c = (wpre & 1u) | ((wpre >> 1) & cta_cin);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint64_t sum = (uint64_t)p[k] + ((g[k] << 1) | c);
        cm[k] = (uint32_t)sum ^ p[k];
        c = (uint32_t)(sum >> 32) | (g[k] >> 31);
    }
    __syncthreads();                 // s_w, s_tot reused by the next tile
    return next;
}

// One row of an add (sub = false) or subtract chain: d = a +/- b, its
// generate / propagate masks over the warp; limbs past the length (!in)
// propagate, so a chain's carry out is that of its last limb.
__device__ __forceinline__ void chain_row(uint64_t a, uint64_t b, bool in, bool sub, uint64_t& d,
                                          uint32_t& g, uint32_t& p) {
    constexpr unsigned FULL = 0xffffffffu;
    bool G, P;
    if (sub) {
        d = a - b;
        G = a < b;                     // borrow generated
        P = !in || d == 0;             // borrow propagates
    } else {
        d = a + b;
        G = d < a;
        P = !in || d == ~0ull;
    }
    g = __ballot_sync(FULL, G);
    p = __ballot_sync(FULL, P);
}

// z[0..len) = x +/- y (+ cin / - bin), x(i), y(i) limb accessors (0 beyond
// their length); returns the carry / borrow out.  z may alias x or y limb
// for limb (limb i is read and written by the same thread).  A tile holds
// CL * DIV_TILE limbs, DIV_TILE per CTA; a warp takes 32 * DIV_PER
// consecutive limbs as DIV_PER rows of 32, lane l on limb row * 32 + l, so
// every load and store is coalesced.
template <int CL, class FX, class FY>
__device__ uint32_t block_addsub(Grp<CL>& grp, uint64_t* z, int64_t len, FX x, FY y, bool sub,
                                 uint32_t cin) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t carry = cin;
    for (int64_t base = 0; base < len; base += (int64_t)CL * DIV_TILE) {
        const int64_t w0 = base + (int64_t)grp.rank * DIV_TILE + (int64_t)wid * (32 * DIV_PER) + lane;
        uint64_t s[DIV_PER];
        uint32_t g[DIV_PER], p[DIV_PER], cm[DIV_PER];
#pragma unroll
        for (int k = 0; k < DIV_PER; ++k) {
            const int64_t i = w0 + 32 * k;
            const bool in = i < len;
            chain_row(in ? x(i) : 0, in ? y(i) : 0, in, sub, s[k], g[k], p[k]);
        }
        carry = tile_carries(grp, g, p, carry, cm);
#pragma unroll
        for (int k = 0; k < DIV_PER; ++k) {
            const int64_t i = w0 + 32 * k;
            const uint64_t cl = (cm[k] >> lane) & 1u;
            if (i < len) z[i] = sub ? s[k] - cl : s[k] + cl;
        }
    }
    return carry;
}

// The three chains of the division's end-around remainder in one pass:
// F = C_lo + C_hi (C_hi = P[L .. L+3) at limbs 0..2), G = N_lo - F,
// H = G + N_hi (N_hi = N[L .. n2)), H into P[0 .. L).  Returns the carry
// outs c, b, c2 in bits 0, 1, 2: the value N - C = H + (c2 - b - c) B^L.
// Each row's limbs go through the chains in order, every chain's carries
// resolved per tile before the next chain reads its digits.
#define FOLD_PER 4
template <int CL>
__device__ uint32_t block_fold3(Grp<CL>& grp, uint64_t* P, int64_t L, const uint64_t* N, int64_t n2) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int64_t TILE = (int64_t)DIV_T * FOLD_PER;
    uint32_t ca = 0, cb = 0, cc = 0;
    for (int64_t base = 0; base < L; base += (int64_t)CL * TILE) {
        const int64_t w0 = base + (int64_t)grp.rank * TILE + (int64_t)wid * (32 * FOLD_PER) + lane;
        uint64_t v[FOLD_PER], nl[FOLD_PER], nh[FOLD_PER];
        uint32_t g[FOLD_PER], p[FOLD_PER], cm[FOLD_PER];
#pragma unroll
        for (int k = 0; k < FOLD_PER; ++k) {
            const int64_t i = w0 + 32 * k;
            const bool in = i < L;
            nl[k] = in ? N[i] : 0;
            nh[k] = (in && L + i < n2) ? N[L + i] : 0;
            chain_row(in ? P[i] : 0, (in && i < 3) ? P[L + i] : 0, in, false, v[k], g[k], p[k]);
        }
        ca = tile_carries(grp, g, p, ca, cm);
#pragma unroll
        for (int k = 0; k < FOLD_PER; ++k) {
            const int64_t i = w0 + 32 * k;
            const bool in = i < L;          // limbs past L hold 0 in every chain
            chain_row(nl[k], in ? v[k] + ((cm[k] >> lane) & 1u) : 0, in, true, v[k], g[k], p[k]);
        }
        cb = tile_carries(grp, g, p, cb, cm);
#pragma unroll
        for (int k = 0; k < FOLD_PER; ++k) {
            const int64_t i = w0 + 32 * k;
            const bool in = i < L;
            chain_row(in ? v[k] - ((cm[k] >> lane) & 1u) : 0, nh[k], in, false, v[k], g[k], p[k]);
        }
        cc = tile_carries(grp, g, p, cc, cm);
#pragma unroll
        for (int k = 0; k < FOLD_PER; ++k) {
            const int64_t i = w0 + 32 * k;
            if (i < L) P[i] = v[k] + ((cm[k] >> lane) & 1u);
        }
    }
    return ca | (cb << 1) | (cc << 2);
}

// sign of x - y over len limbs: -1, 0, 1 (group-uniform).  Walks down from
// the top CL * DIV_T limbs at a time and stops at the first window holding a
// difference (the top one, unless the operands agree there).
template <int CL, class FX, class FY>
__device__ int block_cmp(Grp<CL>& grp, int64_t len, FX x, FY y) {
    __shared__ long long s_hi;
    for (int64_t top = len; top > 0; top -= (int64_t)CL * DIV_T) {
        if (threadIdx.x == 0) s_hi = -1;
        __syncthreads();
        const int64_t i = top - 1 - (int64_t)grp.rank * DIV_T - threadIdx.x;
        if (i >= 0 && x(i) != y(i)) atomicMax(&s_hi, (long long)i);
        __syncthreads();
        const long long hi = grp.max_all(s_hi);
        __syncthreads();
        if (hi >= 0) return x(hi) > y(hi) ? 1 : -1;
    }
    return 0;
}

// z[0..len) += 1 (inc) or -= 1 in place: the carry / borrow ripples only
// through the low limbs equal to ~0 / 0, so the pass stops at the first
// limb that absorbs it (found CL * DIV_T limbs at a time).  The caller puts
// a group barrier between this and any read of z by another CTA.
template <int CL>
__device__ bool block_step1(Grp<CL>& grp, uint64_t* z, int64_t len, bool inc) {
    __shared__ long long s_lo;
    const uint64_t ripple = inc ? ~0ull : 0ull;
    for (int64_t base = 0; base < len; base += (int64_t)CL * DIV_T) {
        if (threadIdx.x == 0) s_lo = len;
        __syncthreads();
        const int64_t i = base + (int64_t)grp.rank * DIV_T + threadIdx.x;
        const bool stop = i < len && z[i] != ripple;
        if (stop) atomicMin(&s_lo, (long long)i);
        __syncthreads();
        const long long lo = grp.min_all(s_lo);
        // limbs below lo (within this window) ripple; limb lo absorbs
        if (i < len && i < lo) z[i] = inc ? 0ull : ~0ull;
        if (i == lo) z[i] = inc ? z[i] + 1 : z[i] - 1;
        __syncthreads();
        if (lo < len) return false;
    }
    return true;                        // rippled out of the top limb
}

// a flag over the group: any (OR) or every (AND) CTA's
template <int CL>
__device__ bool grp_any(Grp<CL>& grp, bool v) { return grp.max_all(v ? 1 : 0) != 0; }

// ---------------------------------------------------------------------------
// per-division descriptors
// ---------------------------------------------------------------------------
struct RecipStep {
    const uint64_t* A;      // top n limbs of D
    uint64_t* Xh;           // h+1 limbs (in/out: corrected in place)
    uint64_t* T;            // n+h+1 limbs: D*Xh on entry (rebuilt from C when L > 0)
    uint64_t* C;            // L > 0: A*Xh mod (B^L - 1) as L+3 unfolded limbs
    int64_t L;
    uint64_t* TM;           // out: h+1 limbs
    const uint64_t* U;      // n/a in step 1; 2h+2 limbs in step 2
    uint64_t* X;            // out of step 2: n+1 limbs
    int64_t n, h;
};

struct DivFix {
    const uint64_t* N;      // 2n limbs
    const uint64_t* D;      // n limbs
    uint64_t* P;            // step q0: N_hi * V (2n limbs); step fix: Q0 * D (2n+1), or
    int64_t L;              //   with L > 0 Q0 * D mod (B^L - 1) as L+3 unfolded limbs
    uint64_t* Q;            // n+1 limbs
    uint64_t* R;            // n limbs (remainder out)
    uint64_t* Rw;           // n+1 limbs of scratch
    int64_t n;
};

// ---- block division for small divisors -----------------------------------
// Schoolbook division of an nn-limb N by a normalised m-limb D (m <= 127),
// one warp per division: the reference's block division (divrem_core,
// include/divrem.h:117-160, with its 3-by-2 reciprocal seed) restated for a
// warp.  Each quotient limb is estimated from the remainder's top three limbs
// and the divisor's top two by the 3-by-2 division of Moeller and Granlund
// ("Improved division by invariant integers", IEEE Trans. Computers 60(2),
// 2011: Algorithm 5 div3by2 with the reciprocal of Algorithm 6); the estimate
// is exact or one too large, so the multiply-subtract of q D is followed by
// at most one add-back.  Lane l holds limbs 4l .. 4l+3 of the running
// remainder and of D; the borrow and carry chains of a step are resolved in
// one go from the lanes' generate / propagate ballots.
#define SBG_DIV_BASE 127            // largest divisor of the warp division (limbs)

// floor((B^3 - 1) / (d1 B + d0)) - B for d1 >= B/2 (Algorithm 6; its first
// line, floor((B^2 - 1) / d1) - B, by a 128-by-64 division)
__device__ __forceinline__ uint64_t recip_3by2(uint64_t d1, uint64_t d0) {
    const unsigned __int128 num = ((unsigned __int128)(~d1) << 64) | ~0ull;
    uint64_t v = (uint64_t)(num / d1);
    uint64_t p = d1 * v;
    p += d0;
    if (p < d0) {
        --v;
        if (p >= d1) {
            --v;
            p -= d1;
        }
        p -= d1;
    }
    const unsigned __int128 t = (unsigned __int128)v * d0;
    const uint64_t t1 = (uint64_t)(t >> 64), t0 = (uint64_t)t;
    p += t1;
    if (p < t1) {
        --v;
        if (p > d1 || (p == d1 && t0 >= d0)) --v;
    }
    return v;
}

// floor((u2 B^2 + u1 B + u0) / (d1 B + d0)) for (u2, u1) < (d1, d0) (Algorithm 5)
__device__ __forceinline__ uint64_t div3by2(uint64_t u2, uint64_t u1, uint64_t u0, uint64_t d1, uint64_t d0,
                                            uint64_t v) {
    const unsigned __int128 qq = (unsigned __int128)v * u2 + (((unsigned __int128)u2 << 64) | u1);
    uint64_t q1 = (uint64_t)(qq >> 64);
    const uint64_t q0 = (uint64_t)qq;
    uint64_t r1 = u1 - q1 * d1;
    const unsigned __int128 t = (unsigned __int128)d0 * q1;
    unsigned __int128 r = (((unsigned __int128)r1 << 64) | u0) - t - (((unsigned __int128)d1 << 64) | d0);
    r1 = (uint64_t)(r >> 64);
    q1 += 1;
    const unsigned __int128 dd = ((unsigned __int128)d1 << 64) | d0;
    if (r1 >= q0) {
        q1 -= 1;
        r += dd;
    }
    if (r >= dd) q1 += 1;
    return q1;
}

#define WFULL 0xffffffffu

// limb i (warp-uniform) of a warp-held array
__device__ __forceinline__ uint64_t wget(const uint64_t (&w)[4], int i) {
    const int k = i & 3;
    const uint64_t x = k == 0 ? w[0] : (k == 1 ? w[1] : (k == 2 ? w[2] : w[3]));
    return __shfl_sync(WFULL, x, i >> 2);
}

// ripple resolution of a 1-bit chain over the warp's 128 positions: per lane
// the generate / propagate bits of its 4 limbs; returns the chain's input
// into this lane's first limb and sets `out` to the chain's output
__device__ __forceinline__ uint32_t warp_chain(uint32_t gb, uint32_t pb, uint32_t& out) {
    const int lane = threadIdx.x & 31;
    const uint32_t lG = (pb + (gb << 1)) >> 4, lP = pb == 15u;
    const uint32_t g = __ballot_sync(WFULL, lG), p = __ballot_sync(WFULL, lP);
    const uint64_t sum = (uint64_t)p + (g << 1);
    out = (uint32_t)(sum >> 32) | (g >> 31);
    return (((uint32_t)sum ^ p) >> lane) & 1u;
}

// w -= q d over the warp's limbs; true when the result is negative (borrow
// out of the top).  Limbs above the used range are zero before and are left
// for the caller to clear.
__device__ __forceinline__ bool warp_submul(uint64_t (&w)[4], const uint64_t (&d)[4], uint64_t q) {
    const int lane = threadIdx.x & 31;
    uint64_t lo[4], hi[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        lo[k] = q * d[k];
        hi[k] = __umul64hi(q, d[k]);
    }
    uint64_t hin = __shfl_up_sync(WFULL, hi[3], 1);
    if (lane == 0) hin = 0;
    uint64_t t[4];
    uint32_t kb[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint64_t hp = k ? hi[k - 1] : hin;
        const uint64_t s1 = w[k] - lo[k];
        const uint32_t b1 = w[k] < lo[k];
        t[k] = s1 - hp;
        kb[k] = b1 + (s1 < hp);
    }
    uint32_t kin = __shfl_up_sync(WFULL, kb[3], 1);
    if (lane == 0) kin = 0;
    uint32_t gb = 0, pb = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t kp = k ? kb[k - 1] : kin;
        const uint64_t z = t[k] - kp;
        gb |= (uint32_t)(t[k] < kp) << k;
        pb |= (uint32_t)(z == 0) << k;
        t[k] = z;
    }
    uint32_t neg;
    uint32_t r = warp_chain(gb, pb, neg);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        w[k] = t[k] - r;
        r = ((gb >> k) & 1u) | (((pb >> k) & 1u) & r);
    }
    return neg != 0;
}

// w += d over the warp's limbs; the carry out of the top
__device__ __forceinline__ bool warp_add(uint64_t (&w)[4], const uint64_t (&d)[4]) {
    uint32_t gb = 0, pb = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint64_t s = w[k] + d[k];
        gb |= (uint32_t)(s < w[k]) << k;
        pb |= (uint32_t)(s == ~0ull) << k;
        w[k] = s;
    }
    uint32_t cout;
    uint32_t c = warp_chain(gb, pb, cout);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint64_t s = w[k];
        w[k] = s + c;
        c = ((gb >> k) & 1u) | (((pb >> k) & 1u) & c);
    }
    return cout != 0;
}

// zero the limbs at index > top
__device__ __forceinline__ void warp_clip(uint64_t (&w)[4], int top) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (4 * lane + k > top) w[k] = 0;
}

// Q[0 .. nn-m] = floor(N / D), R[0 .. m) = N mod D (R may be null); numerator
// limb i is nlimb(i) (i < nn).  D normalised, 1 <= m <= SBG_DIV_BASE, nn >= m.
// Returns false when an estimate needed more than one add-back (cannot
// happen for a normalised D; reported as an error).
template <class NF>
__device__ bool warp_divrem(const uint64_t* __restrict__ D, int m, NF nlimb, int64_t nn, uint64_t* __restrict__ Q,
                            uint64_t* __restrict__ R) {
    const int lane = threadIdx.x & 31;
    uint64_t d[4], w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int i = 4 * lane + k;
        d[k] = i < m ? D[i] : 0ull;
        w[k] = i < m ? nlimb(nn - m + i) : 0ull;
    }
    const uint64_t d1 = wget(d, m - 1), d0 = m >= 2 ? wget(d, m - 2) : 0ull;
    const uint64_t v = recip_3by2(d1, d0);
    bool ok = true;
    // top quotient limb: 0 or 1 (the top m limbs of N are below 2 D)
    {
        uint64_t qt = 1;
        if (warp_submul(w, d, 1)) {
            warp_add(w, d);
            qt = 0;
        }
        warp_clip(w, m);
        if (lane == 0) Q[nn - m] = qt;
    }
    uint64_t nbuf = 0;
    for (int64_t j = nn - m - 1, s = 0; j >= 0; --j, ++s) {
        if ((s & 31) == 0) {                       // the next 32 numerator limbs, one per lane
            const int64_t i = j - lane;
            nbuf = i >= 0 ? nlimb(i) : 0ull;
        }
        // shift the remainder up one limb and bring in N[j]
        const uint64_t inl = __shfl_sync(WFULL, nbuf, (int)(s & 31));
        const uint64_t up = __shfl_up_sync(WFULL, w[3], 1);
        w[3] = w[2];
        w[2] = w[1];
        w[1] = w[0];
        w[0] = lane == 0 ? inl : up;
        const uint64_t u2 = wget(w, m), u1 = wget(w, m - 1), u0 = m >= 2 ? wget(w, m - 2) : 0ull;
        uint64_t q = (u2 == d1 && u1 == d0) ? ~0ull : div3by2(u2, u1, u0, d1, d0, v);
        if (warp_submul(w, d, q)) {
            q -= 1;
            if (!warp_add(w, d)) {              // still negative: a second add-back
                q -= 1;
                if (!warp_add(w, d)) ok = false;
            }
        }
        warp_clip(w, m);
        if (lane == 0) Q[j] = q;
    }
    if (R) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = 4 * lane + k;
            if (i < m) R[i] = w[k];
        }
    }
    return ok;
}

#define WDIV_WARPS 4            // divisions (warps) per CTA

// exact base case of the Newton recursion: X = floor((B^2m - 1) / A), m+1
// limbs (top limb 1), m <= SBG_DIV_BASE; one warp per divisor
__global__ void __launch_bounds__(32 * WDIV_WARPS) k_recip_base(const uint64_t* const* A, const int64_t* m,
                                                              uint64_t* const* X, int count, uint32_t* err) {
    const int idx = blockIdx.x * WDIV_WARPS + (threadIdx.x >> 5);
    if (idx >= count) return;
    const int n = (int)m[idx];
    uint64_t* q = X[idx];
    const bool ok = warp_divrem(A[idx], n, [](int64_t) { return ~0ull; }, 2 * (int64_t)n, q, nullptr);
    __syncwarp();
    if ((threadIdx.x & 31) == 0 && (!ok || q[n] != 1)) atomicOr(err, 8u);
}

// a division of the batch that runs entirely as one warp
struct WarpDiv {
    const uint64_t* N;
    const uint64_t* D;
    uint64_t* Q;            // nn - dn + 1 limbs
    uint64_t* R;            // dn limbs
    int64_t nn;
    int64_t dn;
};

__global__ void __launch_bounds__(32 * WDIV_WARPS) k_divrem_warp(const WarpDiv* jobs, int count, uint32_t* err) {
    const int idx = blockIdx.x * WDIV_WARPS + (threadIdx.x >> 5);
    if (idx >= count) return;
    const WarpDiv J = jobs[idx];
    const uint64_t* N = J.N;
    const bool ok = warp_divrem(J.D, (int)J.dn, [N](int64_t i) { return N[i]; }, J.nn, J.Q, J.R);
    if ((threadIdx.x & 31) == 0 && !ok) atomicOr(err, 8u);
}

// step 0 (wrapped first product): T = A X_h lies within 2 B^n of B^(n+h)
// (A X_h = A_h X_h B^l + A_l X_h with B^2h - 2 A_h <= A_h X_h < B^2h and
// 0 <= A_l X_h < 2 B^n), so it is known from T mod (B^L - 1) for any
// L >= n + 2: with E' = (T - B^(n+h)) mod (B^L - 1) in [0, B^L - 1),
// T = B^(n+h) + E' if E' < B^L / 2, else B^(n+h) - (B^L - 1 - E').  The
// product itself is the cyclic convolution of length L (the FFT form of the
// middle product), carried into L + 3 limbs and folded here.
//
// Every linear kernel runs CL CTAs per division (descriptor blockIdx.x / CL);
// limb-parallel loops spread over the group, and a group barrier separates
// phases that read what another CTA wrote.
#define GRP_LOOP(i, n) for (int64_t i = (int64_t)grp.rank * DIV_T + threadIdx.x; i < (n); i += (int64_t)CL * DIV_T)

template <int CL>
__global__ void __launch_bounds__(DIV_T) k_recip_wrap(const RecipStep* st, uint32_t* err) {
    __shared__ long long s_slot[2];
    Grp<CL> grp(s_slot);
    const RecipStep S = st[blockIdx.x / CL];
    if (S.L == 0) return;                   // the whole group returns
    const int64_t n = S.n, h = S.h, L = S.L, sft = n + h - L;   // 0 <= sft < L
    uint64_t* C = S.C;
    // fold: C mod (B^L - 1) = C[0..L) + C[L..L+3), end-around carry
    const uint32_t c = block_addsub(grp, C, L, [&](int64_t i) { return C[i]; },
                                    [&](int64_t i) { return i < 3 ? C[L + i] : 0ull; }, false, 0);
    grp.sync();
    if (c && block_step1(grp, C, L, true)) {    // B^L = 1 again: the value is 1
        if (grp.rank == 0 && threadIdx.x == 0) C[0] = 1;
    }
    grp.sync();
    // E' = C - B^sft: a borrow rippling up from limb sft, over the zero limbs
    // only (a borrow out of the top means C < B^sft: E' = C - B^sft + B^L - 1)
    const bool b = block_step1(grp, C + sft, L - sft, false);
    grp.sync();
    if (b) block_step1(grp, C, L, false);
    grp.sync();
    const bool neg = (C[L - 1] >> 63) != 0;
    // |E| < 2 B^n: limbs n+1 .. L-1 of E' are 0 (E >= 0) or ~0 (E < 0)
    if (threadIdx.x == 0 && L - 1 > n && C[L - 1] != (neg ? ~0ull : 0ull)) atomicOr(err, 128u);
    uint64_t* T = S.T;
    const int64_t tl = n + h + 1;
    if (!neg) {
        GRP_LOOP(i, tl) T[i] = i < L ? C[i] : (i == n + h ? 1ull : 0ull);
    } else {
        // T = B^(n+h) - |E| = (E' + 1) on the low L limbs, ~0 up to n+h-1, 0 on
        // top: a copy, then the +1 ripple (E' < B^L - 1, so it stops inside)
        GRP_LOOP(i, L) T[i] = C[i];
        grp.sync();
        block_step1(grp, T, L, true);
        for (int64_t i = L + (int64_t)grp.rank * DIV_T + threadIdx.x; i < tl; i += (int64_t)CL * DIV_T)
            T[i] = i == n + h ? 0ull : ~0ull;
    }
    if constexpr (CL > 1) grp.sync();       // peers may still read this CTA's slots
}

// step 1: correct X_h while T >= B^(n+h); T_m = limbs l..n of B^(n+h) - T
template <int CL>
__global__ void __launch_bounds__(DIV_T) k_recip_step1(const RecipStep* st, uint32_t* err) {
    __shared__ long long s_slot[2];
    Grp<CL> grp(s_slot);
    const RecipStep S = st[blockIdx.x / CL];
    const int64_t n = S.n, h = S.h, l = n - h, tl = n + h + 1;
    grp.sync();
    if (S.T[n + h] != 0) {
        // T >= B^(n+h): E = T - B^(n+h) < 2 B^n <= 4 A sits in T's low n+1
        // limbs.  With k the number of corrections (the least k with
        // k A > E), B^(n+h) - (T - k A) = W = k A - E in (0, A], so T_m is
        // limbs l..n of W: W = A - E, then + A while W <= 0 -- n-limb passes
        // instead of k passes over T's n+h+1 limbs.
        const uint64_t* A = S.A;
        uint64_t* T = S.T;
        uint32_t neg = block_addsub(grp, T, n + 1, [&](int64_t i) { return i < n ? A[i] : 0ull; },
                                    [&](int64_t i) { return T[i]; }, true, 0);
        int k = 1;
        for (;;) {
            grp.sync();
            // W > 0: no borrow left and some limb nonzero
            if (!neg && block_cmp(grp, n + 1, [&](int64_t i) { return T[i]; },
                                  [&](int64_t i) { return 0ull; }) > 0)
                break;
            if (k == 4) {
                if (threadIdx.x == 0) atomicOr(err, 16u);
                break;
            }
            const uint32_t c = block_addsub(grp, T, n + 1, [&](int64_t i) { return T[i]; },
                                            [&](int64_t i) { return i < n ? A[i] : 0ull; }, false, 0);
            neg = neg & (c ^ 1u);       // a carry out of the n+1 limbs ends the wrap
            ++k;
        }
        for (int j = 0; j < k; ++j) {
            block_step1(grp, S.Xh, h + 1, false);
            grp.sync();
        }
        uint64_t* TM = S.TM;
        GRP_LOOP(i, h + 1) TM[i] = T[l + i];
        if constexpr (CL > 1) grp.sync();
        return;
    }
    // T < B^(n+h) (the loop below keeps its correction path as a guard)
    for (int it = 0; it < 6; ++it) {
        grp.sync();
        if (S.T[n + h] == 0) break;
        if (it == 5) {
            if (threadIdx.x == 0) atomicOr(err, 16u);
            break;
        }
        const uint64_t* A = S.A;
        uint64_t* T = S.T;
        block_addsub(grp, T, tl, [&](int64_t i) { return T[i]; },
                     [&](int64_t i) { return i < n ? A[i] : 0ull; }, true, 0);
        block_step1(grp, S.Xh, h + 1, false);
    }
    grp.sync();
    // B^(n+h) - T = (~T + 1) on the low n+1 limbs; the +1 reaches limb l only
    // when the limbs below l are all zero
    const uint64_t* T = S.T;
    __shared__ int s_nz;
    if (threadIdx.x == 0) s_nz = 0;
    __syncthreads();
    GRP_LOOP(i, l) if (T[i] != 0) s_nz = 1;
    __syncthreads();
    const uint32_t cin = grp_any(grp, s_nz != 0) ? 0u : 1u;
    uint64_t* TM = S.TM;
    block_addsub(grp, TM, h + 1, [&](int64_t i) { return ~T[l + i]; },
                 [&](int64_t i) { return 0ull; }, false, cin);
    if constexpr (CL > 1) grp.sync();
}

// step 2: X = X_h * B^l + floor(U / B^(2h-l))
template <int CL>
__global__ void __launch_bounds__(DIV_T) k_recip_step2(const RecipStep* st) {
    __shared__ long long s_slot[2];
    Grp<CL> grp(s_slot);
    const RecipStep S = st[blockIdx.x / CL];
    const int64_t n = S.n, h = S.h, l = n - h, sh = 2 * h - l;
    const uint64_t* U = S.U;
    const uint64_t* Xh = S.Xh;
    uint64_t* X = S.X;
    // U' = U >> sh limbs has l + 2 limbs (U has 2h + 2)
    block_addsub(grp, X, n + 1,
                 [&](int64_t i) {
                     const int64_t k = sh + i;
                     return k < 2 * h + 2 ? U[k] : 0ull;
                 },
                 [&](int64_t i) { return i >= l ? Xh[i - l] : 0ull; }, false, 0);
    if constexpr (CL > 1) grp.sync();
}

// Q0 = N_hi + floor(P / B^n), P = N_hi * V (2n limbs)
template <int CL>
__global__ void __launch_bounds__(DIV_T) k_div_q0(const DivFix* df) {
    __shared__ long long s_slot[2];
    Grp<CL> grp(s_slot);
    const DivFix F = df[blockIdx.x / CL];
    const int64_t n = F.n;
    const uint64_t* Nh = F.N + n;
    const uint64_t* P = F.P;
    block_addsub(grp, F.Q, n + 1, [&](int64_t i) { return i < n ? Nh[i] : 0ull; },
                 [&](int64_t i) { return i < n ? P[n + i] : 0ull; }, false, 0);
    if constexpr (CL > 1) grp.sync();
}

// R = (N - Q0 D) on n+1 limbs, then while R >= D: R -= D, Q += 1.  With a
// wrapped product (L >= n + 3): 0 <= R < 6 D < B^(n+1) is the residue of
// N - C mod (B^L - 1), N folded to L limbs, C = Q0 D mod (B^L - 1).
template <int CL>
__global__ void __launch_bounds__(DIV_T) k_div_fix(const DivFix* df, uint32_t* err) {
    __shared__ long long s_slot[2];
    Grp<CL> grp(s_slot);
    const DivFix F = df[blockIdx.x / CL];
    const int64_t n = F.n;
    const uint64_t* N = F.N;
    uint64_t* P = F.P;
    const uint64_t* D = F.D;
    uint64_t* Rw = F.Rw;
    if (F.L == 0) {
        block_addsub(grp, Rw, n + 1, [&](int64_t i) { return N[i]; }, [&](int64_t i) { return P[i]; },
                     true, 0);
    } else {
        const int64_t L = F.L;
        // H = (N_lo - (C_lo + C_hi)) + N_hi in one pass; N - C = H + d B^L
        // with d = c2 - b - c, and B^L = 1 modulo B^L - 1
        const uint32_t cs = block_fold3(grp, P, L, N, 2 * n);
        const int d = (int)((cs >> 2) & 1u) - (int)((cs >> 1) & 1u) - (int)(cs & 1u);
        grp.sync();
        if (d > 0) {
            // H + 1; wrapping past B^L - 1 leaves B^L = 1
            if (block_step1(grp, P, L, true) && grp.rank == 0 && threadIdx.x == 0) P[0] = 1;
            grp.sync();
        }
        for (int k = 0; k < -d; ++k) {
            // H - 1; wrapping below 0 leaves B^L - 1, which is one more than -1
            if (block_step1(grp, P, L, false)) {
                grp.sync();
                block_step1(grp, P, L, false);
            }
            grp.sync();
        }
        // the value is R, or R + (B^L - 1) when R = 0 and the sum came out all ones
        __shared__ int s_hi, s_ones;
        if (threadIdx.x == 0) {
            s_hi = 0;
            s_ones = 1;
        }
        __syncthreads();
        for (int64_t i = n + 1 + (int64_t)grp.rank * DIV_T + threadIdx.x; i < L; i += (int64_t)CL * DIV_T)
            if (P[i] != 0) s_hi = 1;
        __syncthreads();
        if (grp_any(grp, s_hi != 0)) {
            GRP_LOOP(i, L) if (P[i] != ~0ull) s_ones = 0;
            __syncthreads();
            if (grp_any(grp, s_ones == 0) && threadIdx.x == 0) atomicOr(err, 256u);
            GRP_LOOP(i, n + 1) Rw[i] = 0;
        } else {
            GRP_LOOP(i, n + 1) Rw[i] = P[i];
        }
    }
    for (int it = 0; it < 8; ++it) {
        grp.sync();
        int c = block_cmp(grp, n + 1, [&](int64_t i) { return Rw[i]; },
                          [&](int64_t i) { return i < n ? D[i] : 0ull; });
        if (c < 0) break;
        if (it == 7) {
            if (threadIdx.x == 0) atomicOr(err, 32u);
            break;
        }
        block_addsub(grp, Rw, n + 1, [&](int64_t i) { return Rw[i]; },
                     [&](int64_t i) { return i < n ? D[i] : 0ull; }, true, 0);
        block_step1(grp, F.Q, n + 1, true);
    }
    grp.sync();
    GRP_LOOP(i, n) F.R[i] = Rw[i];
    if constexpr (CL > 1) grp.sync();
}

// recip output: V = X - B^n, +1 when B^2n - 1 - D X >= D (X exact in {V, V+1}),
// computed from P = D * X (2n+1 limbs): R = complement of P's low n+1 limbs
template <int CL>
__global__ void __launch_bounds__(DIV_T) k_recip_final(const DivFix* df, uint32_t* err) {
    __shared__ long long s_slot[2];
    Grp<CL> grp(s_slot);
    const DivFix F = df[blockIdx.x / CL];
    const int64_t n = F.n;
    const uint64_t* P = F.P;
    const uint64_t* D = F.D;
    uint64_t* Rw = F.Rw;
    GRP_LOOP(i, n + 1) Rw[i] = ~P[i];
    grp.sync();
    int c = block_cmp(grp, n + 1, [&](int64_t i) { return Rw[i]; },
                      [&](int64_t i) { return i < n ? D[i] : 0ull; });
    // Q holds X (n+1 limbs); V = X (+1) low n limbs
    uint64_t* Q = F.Q;
    if (c >= 0) block_step1(grp, Q, n + 1, true);
    grp.sync();
    if (threadIdx.x == 0 && Q[n] != 1) atomicOr(err, 64u);
    GRP_LOOP(i, n) F.R[i] = Q[i];
    if constexpr (CL > 1) grp.sync();
}
#undef GRP_LOOP

}  // namespace sbg

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
namespace sbg {

struct DivInst {
    const uint64_t* D;      // normalised divisor, n limbs (device)
    const uint64_t* N;      // numerator padded to 2n limbs (device), or null (recip only)
    uint64_t* Qout;         // quotient out (qlen limbs) or reciprocal out (n limbs)
    uint64_t* Rout;         // remainder out (n limbs) or null
    int64_t n;
    int64_t qlen;
    // scratch (device)
    uint64_t* X[2];
    uint64_t* T;
    uint64_t* TM;
    uint64_t* U;
    uint64_t* P;
    uint64_t* Q;
    uint64_t* Rw;
    std::vector<int64_t> sz;   // recursion sizes, sz[0] = n
    int wrapq = -1;            // length code of the wrapped Q0 * D, or -1 (full product)
};

static int64_t h_of(int64_t n) { return n - (n - 1) / 2; }

size_t div_scratch_limbs(int64_t n) { return (size_t)(14 * n + 64); }

}  // namespace sbg

using namespace sbg;

// Every transfer below is stream-ordered on the context stream: descriptor
// arrays go through the context's upload ring, products through its product
// queue; the only synchronisation is the one at the end of a call.
template <class T>
static int upload(sbg_ctx* c, const std::vector<T>& host, T** dev) {
    void* d = nullptr;
    int st = c->ring.push(host.data(), host.size() * sizeof(T), c->stream, &d);
    *dev = (T*)d;
    return st;
}

// Batched limb copies, dst[0..n_dst) = src[0..n_src) zero-extended: the
// padded numerators in, the quotients or reciprocals out -- one launch for a
// whole batch instead of a copy (and a fill) per division.
struct CopyDesc {
    const uint64_t* src;
    uint64_t* dst;
    int64_t n_src, n_dst;
};
#define COPY_BPD 8          // blocks per descriptor
__global__ void __launch_bounds__(256) k_copy_pad(const CopyDesc* d) {
    const CopyDesc D = d[blockIdx.x / COPY_BPD];
    const int64_t stride = (int64_t)COPY_BPD * blockDim.x;
    for (int64_t i = (int64_t)(blockIdx.x % COPY_BPD) * blockDim.x + threadIdx.x; i < D.n_dst; i += stride)
        D.dst[i] = i < D.n_src ? D.src[i] : 0ull;
}
static int copy_batch(sbg_ctx* c, const std::vector<CopyDesc>& cp) {
    for (size_t first = 0; first < cp.size(); first += 4096) {
        const size_t cnt = std::min<size_t>(4096, cp.size() - first);
        std::vector<CopyDesc> part(cp.begin() + first, cp.begin() + first + cnt);
        CopyDesc* dd = nullptr;
        int rc = upload(c, part, &dd);
        if (rc) return rc;
        k_copy_pad<<<(unsigned)(cnt * COPY_BPD), 256, 0, c->stream>>>(dd);
        c->launches += 1;
        if (cudaGetLastError() != cudaSuccess) return SBG_ECUDA;
    }
    return SBG_OK;
}

// One linear step over a descriptor list ordered single-CTA divisions
// first ([0, ns)), clustered ones after ([ns, ns + nb)): a launch per part.
template <class D, class... KA, class... A>
static int launch_lin(sbg_ctx* c, void (*k1)(const D*, KA...), void (*kc)(const D*, KA...), const D* d,
                      int ns, int nb, A... a) {
    if (ns > 0) {
        k1<<<ns, DIV_T, 0, c->stream>>>(d, a...);
        c->launches += 1;
    }
    if (nb > 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)nb * DIV_CL);
        cfg.blockDim = dim3(DIV_T);
        cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = DIV_CL;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (cudaLaunchKernelEx(&cfg, kc, d + ns, a...) != cudaSuccess) return SBG_ECUDA;
        c->launches += 1;
    }
    return cudaGetLastError() == cudaSuccess ? SBG_OK : SBG_ECUDA;
}

// Reciprocals (and optionally quotients) of every instance; all scratch set.
static int div_core(sbg_ctx* c, std::vector<DivInst>& v, uint32_t* err, bool quotient) {
    cudaStream_t st = c->stream;
    int maxd = 0;
    for (auto& d : v) {
        d.sz.clear();
        d.sz.push_back(d.n);
        while (d.sz.back() > SBG_DIV_BASE) d.sz.push_back(h_of(d.sz.back()));
        maxd = std::max(maxd, (int)d.sz.size() - 1);
    }
    int rc = SBG_OK;
    // base case: X[cur] of every instance
    {
        std::vector<const uint64_t*> A;
        std::vector<int64_t> m;
        std::vector<uint64_t*> X;
        for (auto& d : v) {
            const int64_t mb = d.sz.back();
            A.push_back(d.D + (d.n - mb));
            m.push_back(mb);
            X.push_back(d.X[(d.sz.size() - 1) & 1]);
        }
        const uint64_t** dA = nullptr;
        int64_t* dm = nullptr;
        uint64_t** dX = nullptr;
        if ((rc = upload(c, A, &dA)) || (rc = upload(c, m, &dm)) || (rc = upload(c, X, &dX))) return rc;
        k_recip_base<<<((int)v.size() + WDIV_WARPS - 1) / WDIV_WARPS, 32 * WDIV_WARPS, 0, st>>>(
            dA, dm, dX, (int)v.size(), err);
        c->launches += 1;
        if (cudaGetLastError() != cudaSuccess) return SBG_ECUDA;
    }
    for (int r = 1; r <= maxd && !rc; ++r) {
        std::vector<sbg_job> jt, ju;
        std::vector<RecipStep> steps, big;       // single-CTA divisions, clustered ones
        for (auto& d : v) {
            const int depth = (int)d.sz.size() - 1;
            if (depth < r) continue;
            const int k = depth - r;               // level: n = sz[k], h = sz[k+1]
            const int64_t n = d.sz[k], h = d.sz[k + 1];
            RecipStep S{};
            S.A = d.D + (d.n - n);
            S.Xh = d.X[(k + 1) & 1];
            S.X = d.X[k & 1];
            S.T = d.T;
            S.TM = d.TM;
            S.U = d.U;
            S.n = n;
            S.h = h;
            // the first product wrapped at a shorter length when one exists
            // (result into U, which the second product overwrites later)
            const int cfull = conv_lg(n + h, c->len3_mask), cwrap = conv_lg(n + 2, c->len3_mask);
            if (code_len(cwrap) < code_len(cfull)) {
                S.L = code_len(cwrap);
                S.C = d.U;
                jt.push_back(sbg_job{S.C, S.A, S.Xh, n, h + 1, SBG_JOB_CYCLIC, cwrap});
            } else {
                jt.push_back(sbg_job{S.T, S.A, S.Xh, n, h + 1, SBG_JOB_MUL, 0});
            }
            (n >= DIV_CL_MIN_N ? big : steps).push_back(S);
            ju.push_back(sbg_job{d.U, S.TM, S.Xh, h + 1, h + 1, SBG_JOB_MUL, 0});
        }
        const int ns = (int)steps.size(), nb = (int)big.size();
        if (ns + nb == 0) continue;
        steps.insert(steps.end(), big.begin(), big.end());
        RecipStep* dsteps = nullptr;
        if ((rc = upload(c, steps, &dsteps))) break;
        if ((rc = enqueue_products(c, jt.data(), (int64_t)jt.size(), err))) break;
        if ((rc = launch_lin(c, k_recip_wrap<1>, k_recip_wrap<DIV_CL>, (const RecipStep*)dsteps, ns, nb, err)))
            break;
        if ((rc = launch_lin(c, k_recip_step1<1>, k_recip_step1<DIV_CL>, (const RecipStep*)dsteps, ns, nb, err)))
            break;
        if ((rc = enqueue_products(c, ju.data(), (int64_t)ju.size(), err))) break;
        if ((rc = launch_lin(c, k_recip_step2<1>, k_recip_step2<DIV_CL>, (const RecipStep*)dsteps, ns, nb)))
            break;
    }
    if (rc) return rc;
    // final stage: exact reciprocal, or quotient and remainder
    std::vector<DivFix> fx, fxb;             // single-CTA divisions, clustered ones
    std::vector<sbg_job> jp;
    std::vector<CopyDesc> cpx;
    for (auto& d : v) {
        DivFix F{};
        F.N = d.N;
        F.D = d.D;
        F.P = d.P;
        if (quotient) {             // Q0 D wrapped at a shorter length when there is one
            const int cfull = conv_lg(2 * d.n, c->len3_mask), cwrap = conv_lg(d.n + 3, c->len3_mask);
            if (code_len(cwrap) < code_len(cfull)) {
                F.L = code_len(cwrap);
                d.wrapq = cwrap;
            }
        }
        F.Q = d.Q;
        F.R = quotient ? d.Rout : d.Qout;
        F.Rw = d.Rw;
        F.n = d.n;
        (d.n >= DIV_CL_MIN_N ? fxb : fx).push_back(F);
        uint64_t* X = d.X[0];
        if (quotient) {
            // P = N_hi * V, V = low n limbs of X
            jp.push_back(sbg_job{d.P, d.N + d.n, X, d.n, d.n, SBG_JOB_MUL, 0});
        } else {
            cpx.push_back(CopyDesc{X, d.Q, d.n + 1, d.n + 1});
            jp.push_back(sbg_job{d.P, d.D, X, d.n, d.n + 1, SBG_JOB_MUL, 0});
        }
    }
    if (!cpx.empty() && (rc = copy_batch(c, cpx))) return rc;
    const int fs = (int)fx.size(), fb = (int)fxb.size();
    fx.insert(fx.end(), fxb.begin(), fxb.end());
    DivFix* dfx = nullptr;
    if ((rc = upload(c, fx, &dfx))) return rc;
    if ((rc = enqueue_products(c, jp.data(), (int64_t)jp.size(), err))) return rc;
    if (!quotient) {
        if ((rc = launch_lin(c, k_recip_final<1>, k_recip_final<DIV_CL>, (const DivFix*)dfx, fs, fb, err)))
            return rc;
    } else {
        if ((rc = launch_lin(c, k_div_q0<1>, k_div_q0<DIV_CL>, (const DivFix*)dfx, fs, fb))) return rc;
        std::vector<sbg_job> jq;
        for (auto& d : v)
            jq.push_back(d.wrapq >= 0 ? sbg_job{d.P, d.Q, d.D, d.n + 1, d.n, SBG_JOB_CYCLIC, d.wrapq}
                                      : sbg_job{d.P, d.Q, d.D, d.n + 1, d.n, SBG_JOB_MUL, 0});
        if ((rc = enqueue_products(c, jq.data(), (int64_t)jq.size(), err))) return rc;
        if ((rc = launch_lin(c, k_div_fix<1>, k_div_fix<DIV_CL>, (const DivFix*)dfx, fs, fb, err))) return rc;
        std::vector<CopyDesc> cq;
        cq.reserve(v.size());
        for (auto& d : v) cq.push_back(CopyDesc{d.Q, d.Qout, d.qlen, d.qlen});
        if ((rc = copy_batch(c, cq))) return rc;
    }
    return SBG_OK;
}

// grow-only division scratch of the context (and its error word, cleared)
static int div_scratch(sbg_ctx* c, size_t limbs, uint64_t** scratch, bool clear_err = true) {
    if (limbs > c->dscr_cap) {
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) return SBG_ECUDA;
        cudaFree(c->dscr);
        c->dscr = nullptr;
        c->dscr_cap = 0;
        const size_t nl = limbs + limbs / 4;
        if (cudaMalloc(&c->dscr, nl * 8) != cudaSuccess) return SBG_EALLOC;
        c->dscr_cap = nl;
    }
    if (!c->derr) {
        if (cudaMalloc(&c->derr, 4) != cudaSuccess) return SBG_EALLOC;
        clear_err = true;               // a fresh word starts at zero
    }
    if (clear_err && cudaMemsetAsync(c->derr, 0, 4, c->stream) != cudaSuccess) return SBG_ECUDA;
    *scratch = c->dscr;
    return SBG_OK;
}

// wait for the call's work and turn its error word into a status
static int div_finish(sbg_ctx* c, int rc) {
    if (cudaStreamSynchronize(c->stream) != cudaSuccess && !rc) rc = SBG_ECUDA;
    uint32_t h = 0;
    if (!rc && cudaMemcpy(&h, c->derr, 4, cudaMemcpyDeviceToHost) != cudaSuccess) rc = SBG_ECUDA;
    if (!rc && h) rc = (h & 1u) ? SBG_ETIMEOUT : ((h & 2u) ? SBG_ESPILL : SBG_ECUDA);
    return rc;
}

static void carve(DivInst& d, uint64_t*& p) {
    const int64_t n = d.n;
    d.X[0] = p; p += n + 2;
    d.X[1] = p; p += n + 2;
    d.T = p; p += 2 * n + 4;
    d.TM = p; p += n + 2;
    d.U = p; p += 2 * n + 6;
    d.P = p; p += 2 * n + 4;
    d.Q = p; p += n + 2;
    d.Rw = p; p += n + 2;
}

int sbg::recip_batch(sbg_ctx* c, const uint64_t* const* D, uint64_t* const* V, const int64_t* n,
                     int count) {
    if (count <= 0) return SBG_OK;
    size_t total = 0;
    for (int i = 0; i < count; ++i) {
        if (!D[i] || !V[i] || n[i] <= 0) return SBG_EINVAL;
        if (2 * n[i] + 2 > ((int64_t)1 << 25)) return SBG_EBAND;
        total += div_scratch_limbs(n[i]);
    }
    if (cudaSetDevice(c->device) != cudaSuccess) return SBG_ECUDA;
    uint64_t* scratch = nullptr;
    int rc = div_scratch(c, total, &scratch);
    if (rc) return rc;
    std::vector<DivInst> v((size_t)count);
    uint64_t* p = scratch;
    for (int i = 0; i < count; ++i) {
        v[i].D = D[i];
        v[i].N = nullptr;
        v[i].Qout = V[i];
        v[i].Rout = nullptr;
        v[i].n = n[i];
        v[i].qlen = n[i];
        carve(v[i], p);
    }
    return div_finish(c, div_core(c, v, c->derr, false));
}

extern "C" int sbg_recip(sbg_ctx* c, uint64_t* ip, const uint64_t* dp, int64_t n) {
    if (!c || !ip || !dp || n <= 0) return SBG_EINVAL;
    return sbg::recip_batch(c, &dp, &ip, &n, 1);
}

// Batched division: every job has a normalised divisor (top bit set) and
// nn <= 2 dn (the configurations of the reference's Newton division); other
// shapes go through sbg_divrem, which normalises and splits them.  Queues the
// whole batch on the context's stream; keep_err leaves the error word of
// earlier queued batches in place (the asynchronous entry).
static int divrem_enqueue(sbg_ctx* c, const sbg_div_job* jobs, int64_t count, bool keep_err,
                          bool* queued) {
    *queued = false;
    if (!c || (count > 0 && !jobs) || count < 0) return SBG_EINVAL;
    size_t total = 0;
    for (int64_t i = 0; i < count; ++i) {
        const sbg_div_job& j = jobs[i];
        if (!j.qp || !j.rp || !j.np || !j.dp || j.dn <= 0 || j.nn < j.dn || j.nn > 2 * j.dn)
            return SBG_EINVAL;
        if (2 * j.dn + 2 > ((int64_t)1 << 25)) return SBG_EBAND;
        total += div_scratch_limbs(j.dn) + 2 * j.dn + 8;
    }
    if (cudaSetDevice(c->device) != cudaSuccess) return SBG_ECUDA;
    uint64_t* scratch = nullptr;
    int rc = div_scratch(c, total, &scratch, !keep_err);
    if (rc) return rc;
    *queued = true;
    // divisors of at most SBG_DIV_BASE limbs: block division, one warp each
    std::vector<WarpDiv> wd;
    for (int64_t i = 0; i < count; ++i) {
        const sbg_div_job& j = jobs[i];
        if (j.dn <= SBG_DIV_BASE) wd.push_back(WarpDiv{j.np, j.dp, j.qp, j.rp, j.nn, j.dn});
    }
    if (!wd.empty()) {
        WarpDiv* dw = nullptr;
        if ((rc = upload(c, wd, &dw))) return rc;
        k_divrem_warp<<<((int)wd.size() + WDIV_WARPS - 1) / WDIV_WARPS, 32 * WDIV_WARPS, 0, c->stream>>>(
            dw, (int)wd.size(), c->derr);
        c->launches += 1;
        if (cudaGetLastError() != cudaSuccess) return SBG_ECUDA;
        if ((int64_t)wd.size() == count) return SBG_OK;
    }
    std::vector<DivInst> v;
    std::vector<CopyDesc> cn;
    v.reserve((size_t)count);
    cn.reserve((size_t)count);
    uint64_t* p = scratch;
    for (int64_t i = 0; i < count; ++i) {
        const sbg_div_job& j = jobs[i];
        if (j.dn <= SBG_DIV_BASE) continue;
        v.emplace_back();
        cn.emplace_back();
        DivInst& d = v.back();
        d.D = j.dp;
        d.n = j.dn;
        d.Qout = j.qp;
        d.Rout = j.rp;
        d.qlen = j.nn - j.dn + 1;
        // numerator zero-padded to 2n limbs (one batched copy below)
        uint64_t* Np = p;
        p += 2 * j.dn + 8;
        cn.back() = CopyDesc{j.np, Np, j.nn, 2 * j.dn};
        d.N = Np;
        carve(d, p);
    }
    rc = copy_batch(c, cn);
    if (!rc) rc = div_core(c, v, c->derr, true);
    return rc;
}

extern "C" int sbg_divrem_batch(sbg_ctx* c, const sbg_div_job* jobs, int64_t count) {
    bool queued = false;
    int rc = divrem_enqueue(c, jobs, count, false, &queued);
    if (!queued) return rc;             // argument errors: nothing was queued
    rc = div_finish(c, rc);
    if (getenv("SBG_DEBUG") && rc)
        fprintf(stderr, "sbg_divrem_batch: status %d (count %lld, first dn %lld nn %lld)\n", rc,
                (long long)count, count ? (long long)jobs[0].dn : 0LL,
                count ? (long long)jobs[0].nn : 0LL);
    return rc;
}

// The same batch queued without waiting: consecutive batches on one context
// follow each other on its stream (scratch, descriptor ring and padded
// numerators are reused in stream order), so the host prepares the next
// batch while the device runs this one.  Device errors accumulate until
// sbg_divrem_wait.
extern "C" int sbg_divrem_batch_async(sbg_ctx* c, const sbg_div_job* jobs, int64_t count) {
    bool queued = false;
    return divrem_enqueue(c, jobs, count, true, &queued);
}

extern "C" int sbg_divrem_wait(sbg_ctx* c) {
    if (!c) return SBG_EINVAL;
    if (cudaSetDevice(c->device) != cudaSuccess) return SBG_ECUDA;
    if (!c->derr) return cudaStreamSynchronize(c->stream) == cudaSuccess ? SBG_OK : SBG_ECUDA;
    const int rc = div_finish(c, SBG_OK);
    if (cudaMemsetAsync(c->derr, 0, 4, c->stream) != cudaSuccess) return rc ? rc : SBG_ECUDA;
    return rc;
}

extern "C" int sbg_divrem(sbg_ctx* c, uint64_t* qp, uint64_t* rp, const uint64_t* np, int64_t nn,
                          const uint64_t* dp, int64_t dn) {
    sbg_div_job j{qp, rp, np, dp, nn, dn};
    return sbg_divrem_batch(c, &j, 1);
}

// ---------------------------------------------------------------------------
// reference-signature division (include/divrem.h:218, include/dc_div.h:154)
// ---------------------------------------------------------------------------
namespace sbg {

// out[0..n) = (in[0..n) << s) | (carry-in from below); out[n] = spill (if out_n > n)
__global__ void k_shl(uint64_t* out, const uint64_t* in, int64_t n, int64_t out_n, int s) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < out_n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t cur = i < n ? in[i] : 0, prev = (i >= 1 && i - 1 < n) ? in[i - 1] : 0;
        out[i] = s ? ((cur << s) | (prev >> (64 - s))) : cur;
    }
}
__global__ void k_shr(uint64_t* out, const uint64_t* in, int64_t n, int s) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t cur = in[i], next = i + 1 < n ? in[i + 1] : 0;
        out[i] = s ? ((cur >> s) | (next << (64 - s))) : cur;
    }
}

}  // namespace sbg

static bool dev_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

extern "C" sbg_ctx* sbg_default_ctx_internal(void);

// Q = floor(N / D), R = N mod D for any dn >= 1 with dp[dn-1] != 0 and
// nn >= dn (the reference's contract, include/divrem.h:212-217); writes the
// trimmed lengths.  Host or device pointers; synchronous.  Returns 1 on
// success, 0 on failure (the reference returns nothing and aborts on OOM).
extern "C" int sbg_divrem_u64(uint64_t* qp, uint64_t* rp, const uint64_t* np, uint64_t nn64,
                              const uint64_t* dp, uint64_t dn64, uint64_t* qn_out,
                              uint64_t* rn_out) {
    if (!qp || !rp || !np || !dp || dn64 == 0 || nn64 < dn64) return 0;
    sbg_ctx* c = sbg_default_ctx_internal();
    if (!c) return 0;
    cudaStream_t st = (cudaStream_t)sbg_ctx_get_stream(c);
    const int64_t nn = (int64_t)nn64, dn = (int64_t)dn64;
    uint64_t dtop = 0;
    const bool ddev = dev_ptr(dp);
    if (cudaMemcpy(&dtop, dp + dn - 1, 8, ddev ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost) !=
            cudaSuccess || dtop == 0)
        return 0;
    const int s = __builtin_clzll(dtop);
    // device copies: D' (dn), N' (nn+1 limbs), Q (nn-dn+2), R work
    const int64_t nn1 = nn + 1;
    size_t limbs = (size_t)(2 * dn + 2 * nn1 + 4 * dn + 16);
    uint64_t* buf = nullptr;
    if (cudaMalloc(&buf, limbs * 8) != cudaSuccess) return 0;
    uint64_t* dD = buf;                 // dn (raw then normalised in place via tmp)
    uint64_t* dN = dD + dn;             // nn1
    uint64_t* dQ = dN + nn1;            // nn1
    uint64_t* chunk = dQ + nn1;         // 2dn
    uint64_t* cq = chunk + 2 * dn;      // dn + 1
    uint64_t* cr = cq + dn + 1;         // dn
    uint64_t* tmp = cr + dn;            // max(dn, nn) staging
    int ok = 1;
    auto cp = [&](void* d, const void* sp, size_t bytes, cudaMemcpyKind k) {
        if (ok && cudaMemcpyAsync(d, sp, bytes, k, st) != cudaSuccess) ok = 0;
    };
    uint64_t* stage = nullptr;
    if (cudaMalloc(&stage, (size_t)std::max(dn, nn) * 8) != cudaSuccess) {
        cudaFree(buf);
        return 0;
    }
    cp(stage, dp, dn * 8, cudaMemcpyDefault);
    k_shl<<<64, 256, 0, st>>>(dD, stage, dn, dn, s);
    cp(stage, np, nn * 8, cudaMemcpyDefault);
    k_shl<<<256, 256, 0, st>>>(dN, stage, nn, nn1, s);
    if (cudaGetLastError() != cudaSuccess) ok = 0;
    // schoolbook over dn-limb chunks of N' from the top: R < D' always
    int64_t top = nn1;                      // limbs of N' not yet consumed
    int64_t first = nn1 % dn;               // a short leading chunk, if any
    if (first == 0) first = dn;
    // R = the leading chunk (first limbs, < B^first) -- if first < dn it is < D'
    // trivially; if first == dn compare is folded into the first 2dn step by
    // prefixing a zero chunk.
    cudaMemsetAsync(cr, 0, dn * 8, st);
    cudaMemsetAsync(dQ, 0, nn1 * 8, st);
    int64_t qpos = top;                     // quotient limbs are written below qpos
    bool started = false;
    while (ok && top > 0) {
        const int64_t take = started ? dn : first;
        top -= take;
        // chunk = R * B^take + N'[top .. top+take)   (take + dn limbs <= 2dn)
        cp(chunk, dN + top, take * 8, cudaMemcpyDeviceToDevice);
        cp(chunk + take, cr, dn * 8, cudaMemcpyDeviceToDevice);
        sbg_div_job j{cq, cr, chunk, dD, take + dn, dn};
        if (ok && sbg_divrem_batch(c, &j, 1) != SBG_OK) ok = 0;
        // quotient chunk: take+1 limbs, the top one is zero since R < D'
        qpos -= take;
        cp(dQ + qpos, cq, take * 8, cudaMemcpyDeviceToDevice);
        started = true;
    }
    // Q = dQ[0 .. nn-dn+1), R = cr >> s
    const int64_t qlen = nn - dn + 1;
    k_shr<<<64, 256, 0, st>>>(tmp, cr, dn, s);
    if (cudaGetLastError() != cudaSuccess) ok = 0;
    cp(qp, dQ, qlen * 8, cudaMemcpyDefault);
    cp(rp, tmp, dn * 8, cudaMemcpyDefault);
    if (ok && cudaStreamSynchronize(st) != cudaSuccess) ok = 0;
    if (ok) {
        // trimmed lengths (at least 1), as the reference reports them
        std::vector<uint64_t> hq((size_t)qlen), hr((size_t)dn);
        cudaMemcpy(hq.data(), dQ, qlen * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(hr.data(), tmp, dn * 8, cudaMemcpyDeviceToHost);
        int64_t a = qlen;
        while (a > 1 && hq[a - 1] == 0) --a;
        int64_t b = dn;
        while (b > 1 && hr[b - 1] == 0) --b;
        if (qn_out) *qn_out = (uint64_t)a;
        if (rn_out) *rn_out = (uint64_t)b;
    }
    cudaFree(stage);
    cudaFree(buf);
    return ok;
}
