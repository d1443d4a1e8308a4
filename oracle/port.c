/* port.c -- CPU restatement of the reference's large-operand multiply path.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY.  The product library never links, loads
 * or calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, as the checker.  Its results are pinned against the
 * reference itself (oracle/_ref/libsbref.so, built by oracle/Makefile from the
 * reference's own sources) by tests/test_oracle.py, and against the golden
 * vectors in tests/golden/.
 *
 * What it restates (scalar C, one limb = one coefficient, as the reference's
 * p30 engine does -- include/p30.h:1-56):
 *   sbo_ntt_mul / sbo_ntt_sqr   p30_mul_r / p30_sqr_r (include/p30.h:1847-1938,
 *                               1950-2020): residues -> forward NTT -> pointwise
 *                               -> inverse NTT -> scale -> Garner (ascending
 *                               primes) -> lo/mid/hi compose -> carry
 *                               (p30_output, include/p30.h:1742-1842).  Five
 *                               primes k*2^25+1 < 2^31 instead of p30's
 *                               k*2^22+1 < 2^30 so the band reaches 2^25 limbs.
 *   sbo_mul_school              u128 schoolbook (the reference tests' ground
 *                               truth shape, tests/mpn_mul_u64_test.cpp).
 *   sbo_mulmid                  the middle product by its definition
 *                               (bench/recip_mulmid_ref.c:11-16, the
 *                               parallelogram cross-check at :73-77).
 *   sbo_divrem                  Knuth algorithm D on u64 limbs (the family of
 *                               include/divrem.h:117 divrem_core, scalar).
 *   sbo_recip                   floor((B^2n - 1) / D) - B^n for a normalised
 *                               n-limb D (B = 2^64): the reciprocal the Newton
 *                               iteration of bench/recip_mulmid_ref.c:63-116
 *                               approximates.
 *   sbo_mod_u64                 value mod q, for the random-prime spot check.
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ---------------------------------------------------------------- PRNG --- */
/* xorshift64, the reference tests' generator (tests/p30_test.c:14-15) */
uint64_t sbo_xorshift_fill(uint64_t *p, int64_t n, uint64_t state){
    for(int64_t i = 0; i < n; ++i){
        state ^= state << 13; state ^= state >> 7; state ^= state << 17;
        p[i] = state;
    }
    return state;
}

/* --------------------------------------------------------- schoolbook --- */
void sbo_mul_school(uint64_t *rp, const uint64_t *ap, int64_t an,
                    const uint64_t *bp, int64_t bn){
    memset(rp, 0, (size_t)(an + bn) * 8);
    for(int64_t i = 0; i < an; ++i){
        uint64_t cy = 0, ai = ap[i];
        for(int64_t j = 0; j < bn; ++j){
            u128 t = (u128)ai * bp[j] + rp[i + j] + cy;
            rp[i + j] = (uint64_t)t;
            cy = (uint64_t)(t >> 64);
        }
        rp[i + bn] = cy;
    }
}

/* middle product (GMP mpn_mulmid convention), an >= bn >= 1, an-bn+3 limbs:
 * sum_{bn-1 <= i+j <= an-1} a_i b_j B^(i+j-(bn-1)), carried. */
void sbo_mulmid(uint64_t *rp, const uint64_t *ap, int64_t an,
                const uint64_t *bp, int64_t bn){
    int64_t wl = an - bn + 1;                  /* coefficients in the window */
    int64_t nout = wl + 2;
    /* three-word accumulator per output position */
    uint64_t *acc = calloc((size_t)(nout + 2) * 3, 8);
    for(int64_t k = 0; k < wl; ++k){
        int64_t pos = k + bn - 1;                /* coefficient index i + j */
        u128 lo = 0; uint64_t hi = 0;
        int64_t i0 = pos - (bn - 1); if(i0 < 0) i0 = 0;
        int64_t i1 = pos < an - 1 ? pos : an - 1;
        for(int64_t i = i0; i <= i1; ++i){
            int64_t j = pos - i;
            if(j < 0 || j >= bn) continue;
            u128 p = (u128)ap[i] * bp[j];
            u128 s = lo + p;
            if(s < lo) hi++;
            lo = s;
        }
        /* add (hi:lo) at position k */
        u128 t = (u128)acc[3 * k] + (uint64_t)lo;
        acc[3 * k] = (uint64_t)t;
        u128 t2 = (u128)acc[3 * k + 1] + (uint64_t)(lo >> 64) + (uint64_t)(t >> 64);
        acc[3 * k + 1] = (uint64_t)t2;
        acc[3 * k + 2] += hi + (uint64_t)(t2 >> 64);
    }
    /* resolve: value = sum_k (acc0 + acc1 B + acc2 B^2) B^k */
    u128 carry = 0;
    for(int64_t m = 0; m < nout; ++m){
        u128 s = carry + acc[3 * m];
        if(m >= 1) s += acc[3 * (m - 1) + 1];
        uint64_t extra = 0;
        if(m >= 2){ u128 s2 = s + acc[3 * (m - 2) + 2]; if(s2 < s) extra = 1; s = s2; }
        rp[m] = (uint64_t)s;
        carry = (s >> 64) + ((u128)extra << 64);
    }
    free(acc);
}

/* ------------------------------------------------- five-prime NTT ------- */
#define NP 5
static const uint32_t PR[NP] = { 1107296257u, 1711276033u, 1811939329u,
                                 2013265921u, 2113929217u };
static const uint32_t GEN[NP] = { 10u, 29u, 13u, 31u, 5u };

static uint32_t powm(uint64_t a, uint64_t e, uint32_t p){
    uint64_t r = 1; a %= p;
    for(; e; e >>= 1, a = a * a % p) if(e & 1) r = r * a % p;
    return (uint32_t)r;
}
static inline uint32_t shoup_c(uint32_t w, uint32_t p){ return (uint32_t)(((uint64_t)w << 32) / p); }
static inline uint32_t mulsh(uint32_t x, uint32_t w, uint32_t ws, uint32_t p){
    uint32_t q = (uint32_t)(((uint64_t)x * ws) >> 32);
    uint32_t r = x * w - q * p;
    return r >= p ? r - p : r;
}

/* twiddles w^e (e < L/2) with Shoup companions */
static void tw_table(uint32_t *w, uint32_t *ws, int64_t half, uint32_t root, uint32_t p){
    uint64_t x = 1;
    for(int64_t e = 0; e < half; ++e){
        w[e] = (uint32_t)x; ws[e] = shoup_c((uint32_t)x, p);
        x = x * root % p;
    }
}

/* DIF, natural in -> bit-reversed out (the network of p30's forward) */
static void ntt_dif(uint32_t *x, int64_t L, const uint32_t *w, const uint32_t *ws, uint32_t p){
    for(int64_t m = L >> 1, tstep = 1; m >= 1; m >>= 1, tstep <<= 1)
        for(int64_t b = 0; b < L; b += 2 * m)
            for(int64_t j = 0; j < m; ++j){
                uint32_t u = x[b + j], v = x[b + j + m];
                uint32_t s = u + v; if(s >= p) s -= p;
                uint32_t d = u + p - v; if(d >= p) d -= p;
                x[b + j] = s;
                x[b + j + m] = mulsh(d, w[j * tstep], ws[j * tstep], p);
            }
}
/* DIT, bit-reversed in -> natural out, inverse twiddles; returns L * x */
static void ntt_dit(uint32_t *x, int64_t L, const uint32_t *w, const uint32_t *ws, uint32_t p){
    for(int64_t m = 1, tstep = L >> 1; m < L; m <<= 1, tstep >>= 1)
        for(int64_t b = 0; b < L; b += 2 * m)
            for(int64_t j = 0; j < m; ++j){
                uint32_t u = x[b + j];
                uint32_t t = mulsh(x[b + j + m], w[j * tstep], ws[j * tstep], p);
                uint32_t s = u + t; if(s >= p) s -= p;
                uint32_t d = u + p - t; if(d >= p) d -= p;
                x[b + j] = s; x[b + j + m] = d;
            }
}

/* cyclic convolution of a and b (or a with itself) into r[q][0..L), scaled
 * to the true coefficient residues. */
static int conv5(uint32_t *r[NP], const uint64_t *ap, int64_t an,
                 const uint64_t *bp, int64_t bn, int sq, int64_t L){
    uint32_t *ta = malloc((size_t)L * 4), *tb = sq ? NULL : malloc((size_t)L * 4);
    uint32_t *w = malloc((size_t)(L / 2 + 1) * 4), *ws = malloc((size_t)(L / 2 + 1) * 4);
    if(!ta || (!sq && !tb) || !w || !ws){ free(ta); free(tb); free(w); free(ws); return 0; }
    for(int q = 0; q < NP; ++q){
        uint32_t p = PR[q];
        uint32_t root = powm(GEN[q], (p - 1) / (uint64_t)L, p);
        uint64_t two32 = (1ull << 32) % p;
        for(int64_t i = 0; i < L; ++i){
            ta[i] = i < an ? (uint32_t)(((ap[i] >> 32) * two32 + (ap[i] & 0xffffffffu)) % p) : 0;
            if(!sq) tb[i] = i < bn ? (uint32_t)(((bp[i] >> 32) * two32 + (bp[i] & 0xffffffffu)) % p) : 0;
        }
        tw_table(w, ws, L / 2 > 0 ? L / 2 : 1, root, p);
        ntt_dif(ta, L, w, ws, p);
        if(!sq) ntt_dif(tb, L, w, ws, p);
        for(int64_t i = 0; i < L; ++i)
            ta[i] = (uint32_t)((uint64_t)ta[i] * (sq ? ta[i] : tb[i]) % p);
        tw_table(w, ws, L / 2 > 0 ? L / 2 : 1, powm(root, p - 2, p), p);
        ntt_dit(ta, L, w, ws, p);
        uint32_t linv = powm((uint64_t)L % p, p - 2, p), lis = shoup_c(linv, p);
        for(int64_t i = 0; i < L; ++i) r[q][i] = mulsh(ta[i], linv, lis, p);
    }
    free(ta); free(tb); free(w); free(ws);
    return 1;
}

/* Garner (ascending primes) + compose into 160 bits (lo, mid, hi) */
static void garner(const uint32_t v_in[NP], uint64_t *lo, uint64_t *mid, uint64_t *hi){
    uint64_t v[NP];
    v[0] = v_in[0];
    for(int i = 1; i < NP; ++i){
        uint64_t pi = PR[i], acc = v[0] % pi, prod = 1;
        for(int k = 1; k < i; ++k){
            prod = prod * (PR[k - 1] % pi) % pi;
            acc = (acc + v[k] * prod) % pi;
        }
        prod = prod * (PR[i - 1] % pi) % pi;
        uint64_t inv = powm(prod, pi - 2, (uint32_t)pi);
        v[i] = (v_in[i] % pi + pi - acc) % pi * inv % pi;
    }
    /* c = v0 + p0 (v1 + p1 (v2 + p2 (v3 + p3 v4))) in 32-bit words */
    uint32_t w[6] = { (uint32_t)v[4], 0, 0, 0, 0, 0 };
    int nw = 1;
    for(int i = 3; i >= 0; --i){
        uint64_t c = v[i];
        for(int k = 0; k < nw; ++k){
            uint64_t t = (uint64_t)w[k] * PR[i] + c;
            w[k] = (uint32_t)t; c = t >> 32;
        }
        w[nw++] = (uint32_t)c;
    }
    *lo = ((uint64_t)w[1] << 32) | w[0];
    *mid = ((uint64_t)w[3] << 32) | w[2];
    *hi = w[4];
}

/* windowed carry: out[m] = limb (m + off) of sum_{cmin<=j<=cmax} c_j B^j */
static int crt_window(uint64_t *out, int64_t nout, uint32_t *r[NP], int64_t cmin,
                      int64_t cmax, int64_t off){
    uint64_t lo1 = 0, mid1 = 0, hi1 = 0, hi2 = 0;  /* c_{j-1} mid/hi, c_{j-2} hi */
    u128 carry = 0;
    for(int64_t m = -2; m <= nout; ++m){
        int64_t j = m + off;
        uint64_t lo = 0, mid = 0, hi = 0;
        if(j >= cmin && j <= cmax){
            uint32_t v[NP];
            for(int q = 0; q < NP; ++q) v[q] = r[q][j];
            garner(v, &lo, &mid, &hi);
        }
        u128 s = carry + lo + (u128)mid1 + hi2;
        if(m >= 0 && m < nout) out[m] = (uint64_t)s;
        if(m == nout && (uint64_t)s != 0) return 0;   /* spill */
        carry = m >= 0 ? (s >> 64) : 0;
        hi2 = hi1; hi1 = hi; mid1 = mid; (void)lo1;
    }
    return carry == 0;
}

static int64_t pow2_at_least(int64_t n){ int64_t L = 16; while(L < n) L <<= 1; return L; }

#define SBO_MAX_L ((int64_t)1 << 25)

static int windowed(uint64_t *rp, const uint64_t *ap, int64_t an, const uint64_t *bp,
                    int64_t bn, int sq, int64_t need, int64_t cmin, int64_t cmax,
                    int64_t off, int64_t nout){
    int64_t L = pow2_at_least(need);
    if(L > SBO_MAX_L) return 0;
    uint32_t *r[NP];
    uint32_t *blk = malloc((size_t)L * NP * 4);
    if(!blk) return 0;
    for(int q = 0; q < NP; ++q) r[q] = blk + (size_t)q * L;
    int ok = conv5(r, ap, an, bp, bn, sq, L) && crt_window(rp, nout, r, cmin, cmax, off);
    free(blk);
    return ok;
}

int sbo_ntt_mul(uint64_t *rp, const uint64_t *ap, int64_t an, const uint64_t *bp, int64_t bn){
    if(an <= 0 || bn <= 0) return 0;
    return windowed(rp, ap, an, bp, bn, 0, an + bn - 1, 0, an + bn - 2, 0, an + bn);
}
int sbo_ntt_sqr(uint64_t *rp, const uint64_t *ap, int64_t an){
    if(an <= 0) return 0;
    return windowed(rp, ap, an, ap, an, 1, 2 * an - 1, 0, 2 * an - 2, 0, 2 * an);
}
/* middle product through the wrapped convolution (length >= an) */
int sbo_ntt_mulmid(uint64_t *rp, const uint64_t *ap, int64_t an, const uint64_t *bp, int64_t bn){
    if(bn <= 0 || an < bn) return 0;
    return windowed(rp, ap, an, bp, bn, 0, an, bn - 1, an - 1, bn - 1, an - bn + 3);
}

/* ------------------------------------------------------------- divide --- */
/* Knuth D: q = floor(n / d), r = n mod d.  nn >= dn >= 1, d[dn-1] != 0.
 * q gets nn - dn + 1 limbs, r gets dn limbs. */
void sbo_divrem(uint64_t *qp, uint64_t *rp, const uint64_t *np, int64_t nn,
                const uint64_t *dp, int64_t dn){
    if(dn == 1){
        u128 rem = 0;
        for(int64_t i = nn - 1; i >= 0; --i){
            u128 cur = (rem << 64) | np[i];
            qp[i] = (uint64_t)(cur / dp[0]);
            rem = cur % dp[0];
        }
        rp[0] = (uint64_t)rem;
        return;
    }
    int s = __builtin_clzll(dp[dn - 1]);
    uint64_t *d = malloc((size_t)dn * 8), *u = malloc((size_t)(nn + 1) * 8);
    for(int64_t i = dn - 1; i > 0; --i)
        d[i] = s ? (dp[i] << s) | (dp[i - 1] >> (64 - s)) : dp[i];
    d[0] = dp[0] << s;
    u[nn] = s ? np[nn - 1] >> (64 - s) : 0;
    for(int64_t i = nn - 1; i > 0; --i)
        u[i] = s ? (np[i] << s) | (np[i - 1] >> (64 - s)) : np[i];
    u[0] = np[0] << s;
    uint64_t dh = d[dn - 1], dl = d[dn - 2];
    for(int64_t j = nn - dn; j >= 0; --j){
        u128 num = ((u128)u[j + dn] << 64) | u[j + dn - 1];
        u128 qh = num / dh, rh = num % dh;
        while(qh >> 64 || (u128)(uint64_t)qh * dl > ((rh << 64) | u[j + dn - 2])){
            qh--; rh += dh;
            if(rh >> 64) break;
        }
        /* u[j..j+dn] -= qh * d */
        uint64_t q = (uint64_t)qh, borrow = 0, cy = 0;
        for(int64_t i = 0; i < dn; ++i){
            u128 p = (u128)q * d[i] + cy;
            cy = (uint64_t)(p >> 64);
            uint64_t pl = (uint64_t)p;
            uint64_t t = u[i + j] - pl - borrow;
            borrow = (u[i + j] < pl) || (u[i + j] - pl < borrow);
            u[i + j] = t;
        }
        uint64_t t = u[j + dn] - cy - borrow;
        int neg = (u[j + dn] < cy) || (u[j + dn] - cy < borrow);
        u[j + dn] = t;
        if(neg){                                  /* add back */
            q--;
            uint64_t c = 0;
            for(int64_t i = 0; i < dn; ++i){
                u128 sum = (u128)u[i + j] + d[i] + c;
                u[i + j] = (uint64_t)sum; c = (uint64_t)(sum >> 64);
            }
            u[j + dn] += c;
        }
        qp[j] = q;
    }
    for(int64_t i = 0; i < dn; ++i)
        rp[i] = s ? (u[i] >> s) | (u[i + 1] << (64 - s)) : u[i];
    free(d); free(u);
}

/* I = floor((B^2n - 1) / D) - B^n for normalised D (top bit set), n limbs out. */
void sbo_recip(uint64_t *ip, const uint64_t *dp, int64_t n){
    uint64_t *num = malloc((size_t)(2 * n) * 8), *q = malloc((size_t)(n + 1) * 8),
             *r = malloc((size_t)n * 8);
    for(int64_t i = 0; i < 2 * n; ++i) num[i] = ~0ull;
    sbo_divrem(q, r, num, 2 * n, dp, n);
    memcpy(ip, q, (size_t)n * 8);                /* q[n] == 1 is the implicit B^n */
    free(num); free(q); free(r);
}

/* value of {ap, an} mod q (q < 2^63) */
uint64_t sbo_mod_u64(const uint64_t *ap, int64_t an, uint64_t q){
    u128 r = 0;
    u128 b = ((u128)1 << 64) % q;
    for(int64_t i = an - 1; i >= 0; --i)
        r = (r * b + ap[i] % q) % q;
    return (uint64_t)r;
}

/* ------------------------------------------------- threaded CPU baseline - */
typedef struct {
    int32_t kind;      /* 0 mul, 1 sqr, 2 divrem */
    int32_t pad;
    uint64_t *r, *r2;
    const uint64_t *a, *b;
    uint64_t an, bn;
} sbo_job;

typedef struct { sbo_job *jobs; int64_t njobs; atomic_long next; atomic_int fails; } sbo_pool;

static void *sbo_worker(void *arg){
    sbo_pool *pool = arg;
    for(;;){
        long i = atomic_fetch_add(&pool->next, 1);
        if(i >= pool->njobs) break;
        sbo_job *j = &pool->jobs[i];
        int ok = 1;
        if(j->kind == 0) ok = sbo_ntt_mul(j->r, j->a, (int64_t)j->an, j->b, (int64_t)j->bn);
        else if(j->kind == 1) ok = sbo_ntt_sqr(j->r, j->a, (int64_t)j->an);
        else sbo_divrem(j->r, j->r2, j->a, (int64_t)j->an, j->b, (int64_t)j->bn);
        if(!ok) atomic_fetch_add(&pool->fails, 1);
    }
    return NULL;
}

int sbo_run_threads(sbo_job *jobs, int64_t njobs, int threads){
    sbo_pool pool = { jobs, njobs };
    atomic_init(&pool.next, 0);
    atomic_init(&pool.fails, 0);
    if(threads <= 1){ sbo_worker(&pool); return atomic_load(&pool.fails); }
    if(threads > 256) threads = 256;
    pthread_t tid[256];
    for(int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, sbo_worker, &pool);
    for(int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
    return atomic_load(&pool.fails);
}
