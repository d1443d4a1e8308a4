/* simd_bigint_b200.h -- C ABI of the B200 large-operand multiplication path.
 *
 * Numbers are little-endian arrays of uint64_t limbs passed as pointer plus
 * length, exactly as in the reference library (iamstupid/simd_bigint).
 * Products are bit-exact: they are the integer products, computed by a
 * five-prime number-theoretic transform on the GPU followed by Garner CRT and
 * carry resolution, with no floating point anywhere.
 *
 * Two families of entry points:
 *
 *  1. Context entries (sbg_*): pointers are DEVICE memory; work is queued on
 *     the context's CUDA stream and the call returns without waiting.  They
 *     return a status code: SBG_OK (0) or one of the SBG_E* codes below.
 *     NOTE the inversion against the reference, whose entries return 1 on
 *     success and 0 on failure.  Errors detected on the device (carry scan
 *     timeout, spill check) are sticky and reported by sbg_ctx_sync().
 *
 *  2. Reference-signature drop-ins (sbg_nt_mul, sbg_nt_sqr, ...): same
 *     argument order, meaning and return convention as the reference
 *     (1 = success, 0 = failure / out of band).  Pointers may be host or
 *     device memory (classified with cudaPointerGetAttributes); the call is
 *     synchronous and runs on a per-thread default context of the current
 *     CUDA device.
 *
 * rp must not overlap the inputs (reference include/u64cvt.h:92-93).  Zero
 * high limbs are allowed and are treated as values.  Transform band: one
 * product may have an + bn - 1 <= 2^25 limbs (any shape inside that), which
 * covers 2^24 x 2^24; sizes beyond return SBG_EBAND (drop-ins: 0).
 */
#ifndef SIMD_BIGINT_B200_H
#define SIMD_BIGINT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SBG_OK = 0,
    SBG_EINVAL = 1,    /* bad argument (length <= 0, an < bn for mulmid, NULL) */
    SBG_EBAND = 2,     /* beyond the transform band (an + bn - 1 > 2^25)      */
    SBG_EALLOC = 3,    /* device allocation failed                             */
    SBG_ECUDA = 4,     /* a CUDA runtime call failed                           */
    SBG_ETIMEOUT = 5,  /* a bounded device-side wait expired                   */
    SBG_ESPILL = 6,    /* the product spilled past its top limb (internal)     */
    SBG_EADMIT = 7,    /* serving: request rejected by admission control       */
    SBG_ENODEV = 8,    /* no CUDA device / library built without device code  */
    SBG_ECANCELED = 9  /* serving: request cancelled before it was launched    */
};

typedef struct sbg_ctx sbg_ctx;

/* ---- context ------------------------------------------------------------
 * A context owns one CUDA stream, the twiddle tables of every transform length
 * used so far, and the device workspace (it replaces the reference's
 * scratch* argument: include/ntmul.h:47 nt_mul_r, include/scratch.h:293-324).
 */
int sbg_ctx_create(int device, sbg_ctx **out);
void sbg_ctx_destroy(sbg_ctx *ctx);
/* Use an external cudaStream_t (NULL: the context's own stream). */
int sbg_ctx_set_stream(sbg_ctx *ctx, void *cuda_stream);
void *sbg_ctx_get_stream(sbg_ctx *ctx);
/* Wait for queued work; returns and clears any sticky device-side error. */
int sbg_ctx_sync(sbg_ctx *ctx);
/* Build tables and size the workspace for products up to total_limbs limbs
 * (an + bn), so later calls neither allocate nor generate tables. */
int sbg_ctx_reserve(sbg_ctx *ctx, int64_t total_limbs);
const char *sbg_strerror(int status);
/* Per-launch CUDA-event timing of the library's kernels (off by default).
 * sbg_ctx_kernel_times sums the recorded launches per kernel id since the
 * last call (ids: 0 single-CTA product, 1 column forward, 2 row
 * forward+pointwise+inverse, 3 column inverse, 4 CRT+carry, 5 batch,
 * 6 division helpers), waiting for them; n must be >= 8. */
int sbg_ctx_set_timing(sbg_ctx *ctx, int on);
/* Number of kernel launches this context has queued so far (diagnostics). */
int64_t sbg_ctx_launches(sbg_ctx *ctx);
/* Transform lengths.  A product of N coefficients runs at L = 2^a >= N or,
 * for 2^(k+1) < N <= 3 * 2^k with 16 <= k <= 23, at L = 3 * 2^k when bit k
 * of the context's mask is set.  sbg_ctx_autotune times one product of each
 * such size class at both lengths on this device (about a second; allocates
 * 400 MB temporarily) and sets the mask to the faster; times (optional, 16
 * doubles) receives {ms at 2^(k+2), ms at 3 * 2^k} for k = 16 .. 23.  No
 * counterpart in the reference (its p30 engine picks lengths by its own
 * table, include/p30.h:31-37). */
int sbg_ctx_autotune(sbg_ctx *ctx, double *times);
int sbg_ctx_set_len3_mask(sbg_ctx *ctx, uint32_t mask);
uint32_t sbg_ctx_get_len3_mask(sbg_ctx *ctx);
int sbg_ctx_kernel_times(sbg_ctx *ctx, double *ms, int64_t *counts, int n);
/* Largest an + bn accepted by one product (2^25 + 1). */
int64_t sbg_max_total_limbs(void);

/* ---- device-pointer entries ---------------------------------------------- */

/* rp[0 .. an+bn) = {ap, an} * {bp, bn}.
 * Replaces nt_mul / nt_mul_r (reference include/ntmul.h:47-75, 71). */
int sbg_mul(sbg_ctx *ctx, uint64_t *rp, const uint64_t *ap, int64_t an, const uint64_t *bp,
            int64_t bn);

/* rp[0 .. 2an) = {ap, an}^2.
 * Replaces nt_sqr / nt_sqr_r (reference include/ntmul.h:60-80). */
int sbg_sqr(sbg_ctx *ctx, uint64_t *rp, const uint64_t *ap, int64_t an);

/* Middle product, GMP mpn_mulmid convention: an >= bn >= 1, writes an-bn+3
 * limbs  rp = sum_{bn-1 <= i+j <= an-1} ap[i] * bp[j] * 2^(64 (i+j-(bn-1))).
 * Specification: reference bench/recip_mulmid_ref.c:11-16 and
 * include/mulmid.h:5-18 (the reference has no library implementation). */
int sbg_mulmid(sbg_ctx *ctx, uint64_t *rp, const uint64_t *ap, int64_t an, const uint64_t *bp,
               int64_t bn);

/* ---- u52 redundant-digit boundary -------------------------------------------
 * Radix-2^52 digits in 64-bit lanes, the form the reference keeps inside its
 * multiply and division code, converted on the device so that code holding
 * such digits can use the GPU multiply without converting on the host.  All
 * pointers are device memory; work is queued on the context's stream.
 *
 * sbg_u52_from_u64: dp[i] = bits [52 i, 52 i + 52) of {ap, an}, i < n52
 * (digits beyond the number are zero; the reference's u52_from_u64 writes
 * ceil(bitlength / 52) of them -- include/u64cvt.h:42).
 * sbg_u64_from_u52: rp[0 .. rn) = (sum_i dp[i] 2^(52 i)) mod 2^(64 rn) for
 * redundant digits -- unsigned lanes (is_signed = 0, the reference's
 * u64_from_u52_canon, include/canon.h:324) or two's-complement signed lanes
 * (is_signed = 1, u64_from_u52_canonneg, include/canon.h:303).
 * sbg_mul_u52: rp[0 .. an52 + bn52) = the canonical digits of the product
 * of two canonical digit arrays (each digit < 2^52). */
int sbg_u52_from_u64(sbg_ctx *ctx, uint64_t *dp, int64_t n52, const uint64_t *ap, int64_t an);
int sbg_u64_from_u52(sbg_ctx *ctx, uint64_t *rp, int64_t rn, const uint64_t *dp, int64_t n52,
                     int is_signed);
int sbg_mul_u52(sbg_ctx *ctx, uint64_t *rp, const uint64_t *ap, int64_t an52, const uint64_t *bp,
                int64_t bn52);

/* ---- host-pointer entries, stream-ordered ---------------------------------
 * The product of HOST operands into a HOST result, queued and returned at
 * once: upload, transforms and download run on the context's streams, and
 * consecutive calls alternate two staging slots so one product's download
 * overlaps the next one's upload (use page-locked buffers for the overlap;
 * pageable ones work but copy synchronously).  The buffers must stay valid
 * and rp unread until sbg_ctx_sync returns.  Asynchronous form of nt_mul /
 * nt_sqr (reference include/ntmul.h:71-80), which multiply host arrays one
 * call at a time. */
int sbg_mul_host(sbg_ctx *ctx, uint64_t *rp, const uint64_t *ap, int64_t an, const uint64_t *bp,
                 int64_t bn);
int sbg_sqr_host(sbg_ctx *ctx, uint64_t *rp, const uint64_t *ap, int64_t an);

/* ---- batches ---------------------------------------------------------------
 * Thousands of independent products of uneven sizes in a few launches: jobs
 * are grouped by transform length, each group runs one launch per stage for
 * all its jobs, groups run concurrently.  No counterpart in the reference
 * (which multiplies one pair per call); the per-job semantics are those of
 * sbg_mul / sbg_sqr / sbg_mulmid.  All pointers are device memory. */
enum { SBG_JOB_MUL = 0, SBG_JOB_SQR = 1, SBG_JOB_MULMID = 2 };
typedef struct {
    uint64_t *rp;          /* an+bn limbs (mul), 2an (sqr), an-bn+3 (mulmid) */
    const uint64_t *ap;
    const uint64_t *bp;    /* ignored for SBG_JOB_SQR */
    int64_t an, bn;        /* bn ignored for SBG_JOB_SQR */
    int32_t kind;          /* SBG_JOB_* */
    int32_t reserved;
} sbg_job;
typedef struct sbg_batch sbg_batch;
/* Plan a batch: validates jobs, builds missing twiddle tables, allocates the
 * batch workspace and uploads the job table (synchronous). */
int sbg_batch_create(sbg_ctx *ctx, const sbg_job *jobs, int64_t count, sbg_batch **out);
/* Record the batch's launches into a CUDA graph; later runs replay it. */
int sbg_batch_capture(sbg_batch *batch);
/* Queue the whole batch on the context stream (stream-ordered, async). */
int sbg_batch_run(sbg_batch *batch);
/* Waits for queued runs, then frees. */
void sbg_batch_destroy(sbg_batch *batch);
/* Batch engine.  0: ONE persistent kernel whose CTAs take work items --
 * (job, stage, tile) -- from a queue in device memory, waiting on per-job
 * progress counters between a job's stages; it runs the schoolbook,
 * single-CTA and power-of-two four-step classes up to 2^20 points (longer
 * and 3 * 2^k classes keep per-class launches beside it).  1 (default): one
 * launch per stage per length class for every class, the classes on forked
 * streams.  2: the same queue and kernel as 0, one CTA per item instead of
 * persistent CTAs.  sbg_batch_autotune picks one by timing.  wave_bytes (0: keep the
 * current, default 64 MB) bounds the transform workspace of the jobs whose
 * stages the queue interleaves (L2 blocking).  Drops a captured graph:
 * capture again.  No counterpart in the reference. */
int sbg_batch_set_engine(sbg_batch *batch, int engine, int64_t wave_bytes);
/* Times three runs of the batch on each engine (the queue engines at 16 and
 * 64 MB waves; after two warm-up runs; the products are written each time)
 * and keeps the fastest; ms (optional, 3 doubles) receives the best per-run
 * milliseconds of engines 0, 1, 2.  Capture the graph afterwards.  No
 * counterpart in the reference. */
int sbg_batch_autotune(sbg_batch *batch, double *ms);
/* One-shot batch through the context's reusable product arena (no per-call
 * allocation once it has grown): returns when the products are written. */
int sbg_mul_batch(sbg_ctx *ctx, const sbg_job *jobs, int64_t count);

/* ---- Newton reciprocal and division ----------------------------------------
 * All pointers are device memory; the calls wait for their result.
 *
 * sbg_recip: V = floor((2^(128 n) - 1) / D) - 2^(64 n), n limbs, for an n-limb
 * normalised D (top bit set): the reciprocal the reference's Newton
 * prototypes compute (bench/recip_mulmid_ref.c:51-116), here exact.
 *
 * sbg_divrem: Q = floor(N / D) (nn-dn+1 limbs), R = N mod D (dn limbs) for a
 * normalised D and dn <= nn <= 2 dn, by the Newton reciprocal and GPU
 * products; the results equal the reference's divrem_u64_dc
 * (include/dc_div.h:154) bit for bit.  sbg_divrem_batch runs many such
 * divisions with their recursion levels in lockstep (one batch of products
 * per level). */
int sbg_recip(sbg_ctx *ctx, uint64_t *ip, const uint64_t *dp, int64_t n);
int sbg_divrem(sbg_ctx *ctx, uint64_t *qp, uint64_t *rp, const uint64_t *np, int64_t nn,
               const uint64_t *dp, int64_t dn);
typedef struct {
    uint64_t *qp;          /* nn-dn+1 limbs */
    uint64_t *rp;          /* dn limbs */
    const uint64_t *np;
    const uint64_t *dp;    /* top bit set */
    int64_t nn, dn;        /* dn <= nn <= 2 dn */
} sbg_div_job;
int sbg_divrem_batch(sbg_ctx *ctx, const sbg_div_job *jobs, int64_t count);
/* sbg_divrem_batch_async: the same batch queued on the context's stream
 * without waiting (argument errors are returned at once); the host can
 * prepare the next batch while the device runs this one.  Consecutive
 * batches on one context run in order.  Device errors of every queued batch
 * accumulate until sbg_divrem_wait, which waits for the stream and returns
 * (and clears) them; a synchronous sbg_divrem_batch clears them too, so wait
 * before mixing the two.  Operands and results must stay valid until then. */
int sbg_divrem_batch_async(sbg_ctx *ctx, const sbg_div_job *jobs, int64_t count);
int sbg_divrem_wait(sbg_ctx *ctx);

/* ---- serving loop -------------------------------------------------------------
 * Continuous batching of independent requests with admission by HBM
 * footprint; no counterpart in the reference.  Requests name DEVICE operands
 * (which must stay valid until the request completes); results are written
 * into the server's HBM arena and stay there until sbg_server_release.
 * A scheduler thread forms batches from the head of the request FIFO while
 * their footprint (workspace + result) fits the arena, and runs up to
 * `slots` batches concurrently on their own streams; reciprocal requests are
 * batched by `recip_workers` threads, each with its own context.  Latency is measured from sbg_server_submit to
 * the moment the server observes the result on the device. */
enum { SBG_REQ_MUL = 0, SBG_REQ_SQR = 1, SBG_REQ_RECIP = 2 };
typedef struct {
    int32_t kind;          /* SBG_REQ_*; RECIP: ap = normalised divisor (an limbs) */
    int32_t reserved;
    const uint64_t *ap;
    int64_t an;
    const uint64_t *bp;    /* MUL only */
    int64_t bn;
} sbg_request;
typedef struct {
    uint64_t ticket;
    int32_t status;        /* SBG_OK or an error code */
    int32_t reserved;
    uint64_t *rp;          /* device result: an+bn (mul), 2an (sqr), an (recip) limbs */
    int64_t rn;
    double latency_s;      /* submission -> result observed on the device */
    double queue_s;        /* submission -> launch of its batch (the rest is device time) */
} sbg_completion;
typedef struct {
    size_t arena_bytes;    /* HBM budget (default 8 GiB): 5/8 for transform workspaces,
                              3/8 for results awaiting sbg_server_release */
    int32_t slots;         /* batches in flight (default 4) */
    int32_t max_batch;     /* requests per batch (default 512) */
    int32_t recip_workers; /* reciprocal batches in flight, own context each (default 2) */
    int32_t batch_lg_points; /* log2 of the transform points one multiply batch may hold
                                (default 26): smaller batches turn slots over sooner */
} sbg_server_config;
typedef struct sbg_server sbg_server;
int sbg_server_create(sbg_ctx *ctx, const sbg_server_config *cfg, sbg_server **out);
/* Thread-safe, non-blocking.  SBG_EADMIT: the request can never fit the arena. */
int sbg_server_submit(sbg_server *srv, const sbg_request *req, uint64_t *ticket);
/* A burst of requests under one lock: queues reqs[0..] in order until the
 * first one that fails validation (its status is returned); *accepted = the
 * number queued, tickets[i] their tickets. */
int sbg_server_submit_many(sbg_server *srv, const sbg_request *reqs, int64_t count, uint64_t *tickets,
                           int64_t *accepted);
/* Up to max completions; waits up to wait_ms for the first. */
int sbg_server_poll(sbg_server *srv, sbg_completion *out, int max, int *n, int wait_ms);
/* Frees a completed request's result buffer. */
int sbg_server_release(sbg_server *srv, uint64_t ticket);
/* Cancels a request that is still queued: it completes at once with status
 * SBG_ECANCELED and no result.  SBG_EINVAL when the ticket is unknown or the
 * request has already been launched or completed (it then runs to the end). */
int sbg_server_cancel(sbg_server *srv, uint64_t ticket);
int sbg_server_stats(sbg_server *srv, int64_t *pending, int64_t *completed, int64_t *batches,
                     size_t *arena_used);
/* Kernel launches queued by the server so far (multiply batches and reciprocals). */
int64_t sbg_server_launches(sbg_server *srv);
/* Stops the scheduler (queued requests are dropped) and frees the arena. */
void sbg_server_destroy(sbg_server *srv);

/* ---- reference-signature drop-ins ---------------------------------------- */

/* int nt_mul(uint64_t *rp, const uint64_t *ap, ptrdiff_t an,
 *            const uint64_t *bp, ptrdiff_t bn)   -- reference include/ntmul.h:71 */
int sbg_nt_mul(uint64_t *rp, const uint64_t *ap, ptrdiff_t an, const uint64_t *bp, ptrdiff_t bn);

/* int nt_sqr(uint64_t *rp, const uint64_t *ap, ptrdiff_t an)
 *                                                  -- reference include/ntmul.h:77 */
int sbg_nt_sqr(uint64_t *rp, const uint64_t *ap, ptrdiff_t an);

/* void divrem_u64(uint64_t *qp, uint64_t *rp, const uint64_t *np, uint64_t nn64,
 *                 const uint64_t *dp, uint64_t dn64, uint64_t *qn64_out,
 *                 uint64_t *rn64_out)        -- reference include/divrem.h:218,
 *                                               include/dc_div.h:154 (divrem_u64_dc)
 * Same arguments: qp gets nn-dn+1 limbs, rp gets dn limbs, *qn64_out and
 * *rn64_out the trimmed lengths (>= 1). Any divisor with a nonzero top limb, any
 * nn >= dn (normalised and split into 2dn/dn Newton steps).  Returns 1 on
 * success, 0 on failure (the reference's version returns void). */
int sbg_divrem_u64(uint64_t *qp, uint64_t *rp, const uint64_t *np, uint64_t nn64,
                   const uint64_t *dp, uint64_t dn64, uint64_t *qn64_out, uint64_t *rn64_out);

/* ---- allocation-free multiply -------------------------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory when they multiply -- programs that reserve all GPU memory up front,
 * plug-ins inside a host that owns the device allocator, latency-critical
 * loops that cannot take cudaMalloc's implicit synchronisation.
 * rp[0 .. an+bn) = {ap, an} * {bp, bn} on DEVICE pointers, queued on `stream`
 * (NULL: the default stream), for an + bn <= SBG_NOALLOC_MAX_LIMBS; larger
 * products return SBG_EBAND.  Its scratch and twiddle tables are static
 * device arrays of the library (about 740 KB, held on every GPU that loads it
 * until exit); the first call on a device fills the tables and synchronises
 * `stream`, so make that first call before any stream capture.  All calls
 * share one scratch array: calls that overlap on the GPU race and must be
 * ordered by the caller.  Makes no cudaMalloc / cudaFree call. */
#define SBG_NOALLOC_MAX_LIMBS 4097
int sbg_mul_noalloc(uint64_t *rp, const uint64_t *ap, int64_t an, const uint64_t *bp, int64_t bn,
                    void *stream);
int64_t sbg_noalloc_max_limbs(void);
/* Waits for `stream`, then returns the status of the device-side checks of
 * the sbg_mul_noalloc calls made on the current device since the last
 * sbg_noalloc_status (SBG_OK, SBG_ETIMEOUT: the carry scan's bounded wait
 * expired, SBG_ESPILL: the spill check failed), and clears it.  Errors
 * accumulate until read, so an earlier queued call's error is not hidden by
 * a later clean call.  Allocates nothing.  No counterpart in the reference. */
int sbg_noalloc_status(void *stream);

/* ---- test hooks (error paths) ------------------------------------------------
 * For tests of the failure paths without faulting the GPU; no counterpart in
 * the reference.  sbg_debug_inject sets, for the current device, test hooks
 * of the CRT + carry kernel that change data or withhold a flag (0 = off):
 *   SBG_INJECT_WITHHOLD  the first block of each carry scan never publishes
 *                        its look-back flag, and the look-back's bounded wait
 *                        is shortened, so the next block's wait runs out:
 *                        the product is wrong and the status SBG_ETIMEOUT;
 *   SBG_INJECT_TOP       the top coefficient's first residue is altered
 *                        before Garner: the product spills, SBG_ESPILL;
 *   SBG_INJECT_MID       a middle coefficient's residue is altered: a wrong
 *                        product that no device check sees (for host checks).
 * sbg_debug_fail_allocs(n): the next n device allocations of contexts
 * (workspace, plan tables) fail as an out-of-memory device would (SBG_EALLOC). */
enum { SBG_INJECT_WITHHOLD = 1, SBG_INJECT_TOP = 2, SBG_INJECT_MID = 4 };
int sbg_debug_inject(uint32_t mask);
void sbg_debug_fail_allocs(int n);

/* ---- diagnostics ---------------------------------------------------------- */

/* Register-only throughput of the transform butterfly on `device`
 * (butterflies per second): the integer-pipe ceiling of the NTT kernels.
 * No counterpart in the reference (a measurement helper). */
int sbg_probe_bfly_peak(int device, double *bfly_per_s);

#ifdef __cplusplus
}
#endif

#endif /* SIMD_BIGINT_B200_H */
