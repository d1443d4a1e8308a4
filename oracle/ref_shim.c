/* ref_shim.c -- exports the reference library's own multiply / divide entry
 * points from a shared object, so the test suite and the CPU baseline can call
 * the UNMODIFIED reference code through ctypes.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY.  Nothing in the product links this file.
 * It is compiled by oracle/Makefile straight against the reference's headers
 * (include/ntmul.h, include/u64cvt.h, include/dc_div.h) where they lie; no
 * reference source is copied into this repository.
 *
 * Exported (all pointers are HOST memory, little-endian uint64 limbs):
 *   sbref_nt_mul / sbref_nt_sqr      -> nt_mul / nt_sqr        (include/ntmul.h:71-80)
 *   sbref_simd_mpn_mul               -> simd_mpn_mul           (include/u64cvt.h:94)
 *   sbref_divrem_u64_dc              -> divrem_u64_dc          (include/dc_div.h:154)
 *   sbref_divrem_u64                 -> divrem_u64             (include/divrem.h:218)
 *   sbref_mul_router                 -> the baseline router: simd_mpn_mul while
 *                                       2(an+bn) <= 2^19 (its FFT band,
 *                                       include/u64cvt.h:84-89), else nt_mul/nt_sqr
 *   sbref_run_threads                -> runs a list of independent jobs on T
 *                                       pthreads (one job at a time per thread),
 *                                       the multi-core CPU baseline.
 *   sbref_u52_from_u64               -> u52_from_u64           (include/u64cvt.h:42)
 *   sbref_u64_from_u52               -> u64_from_u52_canon / u64_from_u52_canonneg
 *                                       (include/canon.h:303-324), the u52
 *                                       redundant-digit boundary; plain arrays
 *                                       are copied into the 64-byte aligned,
 *                                       vector-padded buffers those functions take.
 */
#define SCRATCH_IMPLEMENTATION
#include "ntmul.h"
#include "u64cvt.h"
#include "dc_div.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

int sbref_nt_mul(uint64_t *rp, const uint64_t *ap, int64_t an,
                 const uint64_t *bp, int64_t bn){
    return nt_mul(rp, ap, (ptrdiff_t)an, bp, (ptrdiff_t)bn);
}

int sbref_nt_sqr(uint64_t *rp, const uint64_t *ap, int64_t an){
    return nt_sqr(rp, ap, (ptrdiff_t)an);
}

void sbref_simd_mpn_mul(uint64_t *rp, const uint64_t *ap, uint64_t an,
                        const uint64_t *bp, uint64_t bn){
    simd_mpn_mul(rp, ap, an, bp, bn);
}

void sbref_divrem_u64_dc(uint64_t *qp, uint64_t *rp,
                         const uint64_t *np, uint64_t nn,
                         const uint64_t *dp, uint64_t dn,
                         uint64_t *qn_out, uint64_t *rn_out){
    divrem_u64_dc(qp, rp, np, nn, dp, dn, qn_out, rn_out);
}

void sbref_divrem_u64(uint64_t *qp, uint64_t *rp,
                      const uint64_t *np, uint64_t nn,
                      const uint64_t *dp, uint64_t dn,
                      uint64_t *qn_out, uint64_t *rn_out){
    divrem_u64(qp, rp, np, nn, dp, dn, qn_out, rn_out);
}

/* kind 0 = mul, 1 = sqr (bp ignored).  Returns 1 on success. */
int sbref_mul_router(int kind, uint64_t *rp, const uint64_t *ap, uint64_t an,
                     const uint64_t *bp, uint64_t bn){
    if(kind == 1){ bp = ap; bn = an; }
    if(2u * (an + bn) <= (1u << 19)){
        simd_mpn_mul(rp, ap, an, bp, bn);
        return 1;
    }
    if(kind == 1) return nt_sqr(rp, ap, (ptrdiff_t)an);
    return nt_mul(rp, ap, (ptrdiff_t)an, bp, (ptrdiff_t)bn);
}

/* ---- multi-threaded job runner (CPU baseline) ---------------------------- */
/* job kinds: 0 mul, 1 sqr, 2 divrem_u64_dc.  For divrem: a = N (an limbs),
 * b = D (bn limbs), r = Q (an-bn+1 limbs), r2 = R (bn limbs). */
typedef struct {
    int32_t kind;
    int32_t pad;
    uint64_t *r, *r2;
    const uint64_t *a, *b;
    uint64_t an, bn;
} sbref_job;

typedef struct {
    sbref_job *jobs;
    int64_t njobs;
    atomic_long next;
    atomic_int fails;
} sbref_pool;

static void *sbref_worker(void *arg){
    sbref_pool *pool = (sbref_pool *)arg;
    for(;;){
        long i = atomic_fetch_add(&pool->next, 1);
        if(i >= pool->njobs) break;
        sbref_job *j = &pool->jobs[i];
        if(j->kind == 2){
            uint64_t qn = 0, rn = 0;
            divrem_u64_dc(j->r, j->r2, j->a, j->an, j->b, j->bn, &qn, &rn);
        }else if(!sbref_mul_router(j->kind, j->r, j->a, j->an, j->b, j->bn)){
            atomic_fetch_add(&pool->fails, 1);
        }
    }
    return NULL;
}

/* Runs jobs[0..njobs) on `threads` pthreads.  Returns the number of failed
 * multiplies (0 on success). */
int sbref_run_threads(sbref_job *jobs, int64_t njobs, int threads){
    if(threads < 1) threads = 1;
    sbref_pool pool;
    pool.jobs = jobs;
    pool.njobs = njobs;
    atomic_init(&pool.next, 0);
    atomic_init(&pool.fails, 0);
    if(threads == 1){
        sbref_worker(&pool);
        return atomic_load(&pool.fails);
    }
    pthread_t tid[256];
    if(threads > 256) threads = 256;
    for(int t = 0; t < threads; ++t)
        pthread_create(&tid[t], NULL, sbref_worker, &pool);
    for(int t = 0; t < threads; ++t)
        pthread_join(tid[t], NULL);
    return atomic_load(&pool.fails);
}

/* ---- u52 redundant-digit boundary ----------------------------------------- */
/* n52 canonical u52 digits of {ap, an} into out (room for an*64/52 + 1
 * digits); returns n52. */
uint64_t sbref_u52_from_u64(uint64_t *out, const uint64_t *ap, uint64_t an){
    const uint64_t cap = (an * 64 + 51) / 52 + 16;
    uint64_t *buf = aligned_alloc(64, ((cap * 8 + 63) / 64) * 64);
    if(!buf) return 0;
    memset(buf, 0, ((cap * 8 + 63) / 64) * 64);
    const uint64_t n52 = u52_from_u64((pvec)buf, ap, an);
    memcpy(out, buf, n52 * 8);
    free(buf);
    return n52;
}

/* rp[0 .. out_limbs) = sum_i d[i] 2^(52 i) for n52 redundant digits: each
 * d[i] an unsigned 64-bit lane (is_signed = 0, u64_from_u52_canon) or a
 * two's-complement signed lane (is_signed = 1, u64_from_u52_canonneg). */
void sbref_u64_from_u52(uint64_t *rp, uint64_t out_limbs, const uint64_t *d, uint64_t n52,
                        int is_signed){
    const uint64_t need = (out_limbs * 64 + 51) / 52 + 16;
    const uint64_t cap = (need > n52 ? need : n52) + 16;
    const size_t bytes = ((cap * 8 + 63) / 64) * 64;
    uint64_t *buf = aligned_alloc(64, bytes);
    if(!buf) return;
    memset(buf, 0, bytes);
    memcpy(buf, d, n52 * 8);
    if(is_signed) u64_from_u52_canonneg(rp, (cpvec)buf, out_limbs);
    else u64_from_u52_canon(rp, (cpvec)buf, out_limbs);
    free(buf);
}
