// sbg_arith.cuh -- 31-bit prime-field arithmetic for the NTT multiplier.
//
// Five primes p_q = k_q * 2^25 + 1 (all < 2^31, ascending: the Garner CRT
// consumes them in this order, as the reference's p30 Garner does,
// include/p30.h:70-71 "ascending order is load-bearing for Garner").  Every
// p_q - 1 is divisible by 3 * 2^25, so transforms of length up to 2^25 (and
// 3 * 2^25) exist mod every prime.  Their product is 2^153.36, which bounds a
// convolution coefficient min(an, bn) * (2^64 - 1)^2 for min(an, bn) up to
// 42,941,745 limbs -- beyond any operand a 2^25-point transform can hold.
//
// Range discipline: every stored residue is canonical, [0, p).  Because p is
// above 2^30, 4p does not fit a u32, so the lazy [0, 4p) ranges the reference
// uses (p30.h:33-38, p < 2^30) are not available; each add/sub reduces with a
// single unsigned min().
#pragma once
#include <cstdint>

#define SBG_NP 5
#define SBG_MAX_LG 25

namespace sbg {

struct PrimeConst {
    uint32_t p;        // the prime
    uint32_t pinv;     // -p^-1 mod 2^32 (Montgomery REDC)
    uint32_t c32;      // 2^32 mod p
    uint32_t c32s;     // Shoup companion of c32: floor(c32 * 2^32 / p)
    uint32_t ones;     // Shoup companion of 1: floor(2^32 / p)
    uint32_t g;        // a generator of (Z/p)^*
    uint32_t mu_lo;    // floor(2^64 / p), low and high words: division-free
    uint32_t mu_hi;    //   Shoup companions (shoup_fast)
};

// host-side copy of the primes (ascending)
static const uint32_t kPrimes[SBG_NP] = {
    1107296257u,   // 33 * 2^25 + 1
    1711276033u,   // 51 * 2^25 + 1
    1811939329u,   // 27 * 2^26 + 1
    2013265921u,   // 15 * 2^27 + 1
    2113929217u,   // 63 * 2^25 + 1
};
static const uint32_t kGenerators[SBG_NP] = { 10u, 29u, 13u, 31u, 5u };

// x in [0, 2p) -> [0, p)
__device__ __forceinline__ uint32_t red1(uint32_t x, uint32_t p) {
    return min(x, x - p);
}

// Shoup multiply by a constant w with companion ws = floor(w * 2^32 / p):
// result in [0, 2p) for ANY u32 x.
__device__ __forceinline__ uint32_t mul_shoup_lazy(uint32_t x, uint32_t w, uint32_t ws,
                                                   uint32_t p) {
    uint32_t q = __umulhi(x, ws);
    return x * w - q * p;
}
__device__ __forceinline__ uint32_t mul_shoup(uint32_t x, uint32_t w, uint32_t ws, uint32_t p) {
    return red1(mul_shoup_lazy(x, w, ws, p), p);
}

// floor(w * 2^32 / p) for w < p without a division: w * floor(2^64 / p) / 2^32
// underestimates by at most one, which the remainder test corrects.
__device__ __forceinline__ uint32_t shoup_fast(uint32_t w, const PrimeConst& c) {
    uint32_t est = __umulhi(w, c.mu_lo) + w * c.mu_hi;
    uint32_t r = 0u - est * c.p;                // (w * 2^32 - est * p) mod 2^32, in [0, 2p)
    return est + (r >= c.p ? 1u : 0u);
}

// Montgomery product a * b * 2^-32 mod p for a, b < p; result in [0, p).
__device__ __forceinline__ uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    uint64_t t = (uint64_t)a * b;               // < p^2 < 2^62
    uint32_t m = (uint32_t)t * pinv;
    uint64_t u = t + (uint64_t)m * p;           // < 2^62 + 2^63
    return red1((uint32_t)(u >> 32), p);
}

__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
    return red1(a + b, p);
}
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
    return red1(a - b + p, p);
}

// u64 limb -> residue in [0, p):  hi * (2^32 mod p) + lo, each Shoup-reduced.
__device__ __forceinline__ uint32_t limb_residue(uint64_t x, const PrimeConst& c) {
    uint32_t hi = (uint32_t)(x >> 32), lo = (uint32_t)x;
    uint32_t a = mul_shoup(hi, c.c32, c.c32s, c.p);
    uint32_t b = mul_shoup(lo, 1u, c.ones, c.p);
    return add_mod(a, b, c.p);
}

// Gentleman-Sande (DIF) butterfly: (u, v) -> (u + v, (u - v) * w).
__device__ __forceinline__ void bfly_gs(uint32_t& u, uint32_t& v, uint32_t w, uint32_t ws,
                                        uint32_t p) {
    uint32_t s = u + v;
    uint32_t d = u - v + p;                     // [1, 2p)
    u = red1(s, p);
    v = mul_shoup(d, w, ws, p);
}
// Either butterfly with the twiddle 1: (u, v) -> (u + v, u - v), no multiply.
__device__ __forceinline__ void bfly_triv(uint32_t& u, uint32_t& v, uint32_t p) {
    uint32_t s = u + v;
    uint32_t d = u - v + p;                     // [1, 2p)
    u = red1(s, p);
    v = red1(d, p);
}
// Cooley-Tukey (DIT) butterfly: (u, v) -> (u + v * w, u - v * w).  Exact
// inverse of bfly_gs with w^-1, up to the factor 2.
__device__ __forceinline__ void bfly_ct(uint32_t& u, uint32_t& v, uint32_t w, uint32_t ws,
                                        uint32_t p) {
    uint32_t t = mul_shoup(v, w, ws, p);
    uint32_t s = u + t;
    uint32_t d = u - t + p;
    u = red1(s, p);
    v = red1(d, p);
}

}  // namespace sbg
