// sbg_plan.cu -- host-side constants of the prime set: Montgomery and Shoup
// companions, Garner mixed-radix constants, per-length CRT scale.
//
// Mirrors the reference's plan set-up (include/p30.h:200-358 p30_pset_init /
// p30_pset_ensure; include/p50.h:236-269 p50_plan_ensure), which computes its
// constants with scalar u128 arithmetic on first use.  Here only the O(1)
// constants are computed on the host; the O(L) twiddle tables are generated on
// the device (sbg_kernels.cu k_gen_pow), which takes milliseconds instead of
// the reference's tens of seconds at 2^22-2^24 limbs.
#include "sbg_internal.h"

namespace sbg {

uint32_t host_powmod(uint64_t a, uint64_t e, uint32_t p) {
    uint64_t r = 1;
    a %= p;
    while (e) {
        if (e & 1) r = r * a % p;
        a = a * a % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

uint32_t host_shoup(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }

static uint32_t host_inv(uint32_t a, uint32_t p) { return host_powmod(a, p - 2, p); }

void host_prime_consts(PrimeConst out[SBG_NP]) {
    for (int q = 0; q < SBG_NP; ++q) {
        uint32_t p = kPrimes[q];
        uint32_t inv = p;                       // p^-1 mod 2^32 by Newton (5 steps)
        for (int i = 0; i < 5; ++i) inv *= 2u - p * inv;
        PrimeConst c;
        c.p = p;
        c.pinv = 0u - inv;
        c.c32 = (uint32_t)((1ull << 32) % p);
        c.c32s = host_shoup(c.c32, p);
        c.ones = host_shoup(1u, p);
        c.g = kGenerators[q];
        unsigned __int128 mu = (((unsigned __int128)1) << 64) / p;
        c.mu_lo = (uint32_t)(uint64_t)mu;
        c.mu_hi = (uint32_t)((uint64_t)mu >> 32);
        out[q] = c;
    }
}

void host_crt_consts(CrtConst* out) {
    CrtConst c;
    for (int i = 0; i < SBG_NP; ++i) {
        for (int k = 0; k < SBG_NP; ++k) {
            c.ppm[i][k] = 0;
            c.ppms[i][k] = 0;
        }
        c.inv[i] = 0;
        c.invs[i] = 0;
    }
    for (int i = 1; i < SBG_NP; ++i) {
        uint32_t pi = kPrimes[i];
        uint64_t prod = 1;                      // prod_{j<k} p_j mod p_i
        for (int k = 1; k <= i; ++k) {
            prod = prod * (kPrimes[k - 1] % pi) % pi;
            if (k < i) {
                c.ppm[i][k] = (uint32_t)prod;
                c.ppms[i][k] = host_shoup((uint32_t)prod, pi);
            } else {
                c.inv[i] = host_inv((uint32_t)prod, pi);
                c.invs[i] = host_shoup(c.inv[i], pi);
            }
        }
    }
    *out = c;
}

// 2^32 * L^-1 mod p_q: cancels the Montgomery factor of the pointwise
// product and the factor L of the unnormalised forward/inverse pair.
ShoupPair host_scale(int64_t L, int q) {
    uint32_t p = kPrimes[q];
    uint32_t linv = host_inv((uint32_t)((uint64_t)L % p), p);
    uint32_t s = (uint32_t)((((1ull << 32) % p) * linv) % p);
    return ShoupPair{s, host_shoup(s, p)};
}

}  // namespace sbg
