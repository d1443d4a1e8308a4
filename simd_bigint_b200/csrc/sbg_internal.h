// sbg_internal.h -- host-side declarations shared by the CUDA translation
// units of the library (kernel launchers, plan tables, constants).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#include <atomic>
#include <vector>

#include "../../include/simd_bigint_b200.h"
#include "sbg_arith.cuh"

namespace sbg {

// Transform lengths are identified by a code: c <= SBG_MAX_LG is L = 2^c,
// c = SBG_CODE3 + k is L = 3 * 2^k (four-step only, k >= SBG_THREE_MIN_LG),
// chosen when it is the smaller of the two lengths that hold a product.
#define SBG_CODE3 32
#define SBG_NCODES (SBG_CODE3 + SBG_MAX_LG)
#define SBG_THREE_MIN_LG 16
// k = 16..19 and 21..23: where 3 * 2^k measured faster than 2^(k+2) on B200
// (at k = 20 the columns of 768 rows need the cross-CTA radix-3 exchange,
// which costs more than the quarter of the points it saves)
#define SBG_LEN3_DEFAULT 0x00EF0000u
// Plain products of at most SBG_SCHOOL_MAX limbs (an + bn) run as one
// schoolbook warp each (sbg_school.cu); in the batch engine they form the
// length class SBG_CODE_SCHOOL (no transform, no workspace).
#define SBG_SCHOOL_MAX 128
#define SBG_CODE_SCHOOL 1
inline bool code_three(int c) { return c >= SBG_CODE3; }
inline int code_lg(int c) { return c >= SBG_CODE3 ? c - SBG_CODE3 : c; }
inline int64_t code_len(int c) { return (int64_t)(c >= SBG_CODE3 ? 3 : 1) << code_lg(c); }

// A (w, shoup) pair as stored in device tables.
struct ShoupPair {
    uint32_t w, ws;
};

// Garner / compose constants (ascending primes).
struct CrtConst {
    // ppm[i][k] = (p_0 * ... * p_{k-1}) mod p_i, k = 1..i-1 (Shoup pairs)
    uint32_t ppm[SBG_NP][SBG_NP];
    uint32_t ppms[SBG_NP][SBG_NP];
    // inv[i] = (p_0 * ... * p_{i-1})^-1 mod p_i
    uint32_t inv[SBG_NP];
    uint32_t invs[SBG_NP];
};

// Per-transform-length plan: the four-step twiddle tables (device) and the
// CRT scale 2^32 * L^-1 mod p (host-side Shoup pairs passed by value).
struct LenPlan {
    int lgL = -1;                 // length code (see code_len)
    int lgN1 = 0, lgN2 = 0;       // column / row sizes (lgN1 = 0: single-CTA); 3 * 2^m3 columns
    int m3 = -1;                  //   rows when m3 >= 0 (L = 3 * 2^(m3 + 12))
    int64_t L = 0;
    uint2* t3_f = nullptr;        // [q][2^(m3+1)] w_N1^j, the radix-3 level's twiddles
    uint2* t3_i = nullptr;
    uint32_t w3f[SBG_NP] = {}, w3fs[SBG_NP] = {};   // cube roots of unity (forward)
    uint32_t w3i[SBG_NP] = {}, w3is[SBG_NP] = {};   // and their inverses
    uint2* fs_lo_f = nullptr;     // [q][8192]      w_L^e, e < 2^13
    uint2* fs_hi_f = nullptr;     // [q][L >> 13]   w_L^(e << 13)
    uint2* fs_lo_i = nullptr;
    uint2* fs_hi_i = nullptr;
    int hi_n = 0;                 // entries in each hi table
    ShoupPair scale[SBG_NP];
};

// Kernel-argument bundle for the four-step twiddles.
struct FsTables {
    const uint2* lo;   // + q * 8192
    const uint2* hi;   // + q * hi_n
    int hi_n;
};

struct ScaleArg {
    uint32_t w[SBG_NP];
    uint32_t ws[SBG_NP];
};

// radix-3 level of a 3 * 2^k transform: twiddle table + cube roots
struct Radix3Arg {
    const uint2* t3;        // + q * 2M
    uint32_t w[SBG_NP];
    uint32_t ws[SBG_NP];
};

// One windowed convolution of the batch engine (device-resident array).
// out[m] = limb (m + off) of sum_{cmin <= j <= cmax} c_j 2^(64 j), m < nout,
// where c = a * b cyclic of the launch's length 2^lgL.
struct JobDesc {
    const uint64_t* a;
    const uint64_t* b;      // == a for squaring
    uint64_t* out;
    int64_t an, bn;
    int64_t cmin, cmax;
    int64_t off;
    int64_t nout;
    uint32_t* ws;           // YA (5 x 2^lgL u32); YB follows it (mul only)
    uint32_t* flags;        // carry look-back: ticket + one word per block
    int32_t sq;
    int32_t pad;
};

// ---- the persistent batch engine ----
// One work item of the persistent batch kernel: a stage of one job (or a
// group of up to 8 schoolbook jobs).  `need` is the value the job's progress
// counter must reach before the item may start (its earlier stages done).
enum PKind : uint16_t { PK_SCHOOL = 0, PK_SMALL = 1, PK_COLF = 2, PK_ROW = 3, PK_COLI = 4, PK_CRT = 5,
                        PK_SMALLJOB = 6 };
struct PItem {
    uint32_t job;           // index into the batch's JobDesc array (first job of a group)
    uint16_t kind;          // PKind
    uint16_t lg;            // the job's length code
    uint32_t idx;           // index within the stage (prime, tile, row, carry block; group size)
    uint32_t need;          // progress-counter value required before starting
};
// per length code: four-step twiddle tables and the CRT scale
struct PClass {
    FsTables fsf, fsi;
    ScaleArg sc;
};
// length codes the persistent kernel runs: schoolbook, single-CTA, and
// power-of-two four-step lengths with columns of at most 2^8 rows
inline bool persist_code(int c) {
    return c == SBG_CODE_SCHOOL || (c >= 4 && c <= 12) || (c >= 13 && c <= 20);
}
#define PERSIST_THREADS 256
// rows per row item and carry blocks per carry item of the persistent queue
// (2 rows and 4 blocks per item measured 17% slower on the mixed batch than
// one of each: finer items balance better)
#ifndef PERSIST_ROWS
#define PERSIST_ROWS 1
#endif
#ifndef PERSIST_CRT
#define PERSIST_CRT 1
#endif

// Kernel ids for the optional per-launch event timing (sbg_ctx_kernel_times).
enum KernelId {
    KID_SMALL = 0,
    KID_COL_FWD = 1,
    KID_ROW = 2,
    KID_COL_INV = 3,
    KID_CRT = 4,
    KID_BATCH = 5,
    KID_DIV = 6,
    KID_COUNT = 8
};

// Records a CUDA event pair around each launch when attached to a context.
struct KTimer {
    virtual void begin(int kid, cudaStream_t st) = 0;
    virtual void end(int kid, cudaStream_t st) = 0;
    virtual ~KTimer() {}
};
#define KT_BEGIN(kt, kid, st) \
    do {                       \
        if (kt) (kt)->begin((kid), (st)); \
    } while (0)
#define KT_END(kt, kid, st) \
    do {                     \
        if (kt) (kt)->end((kid), (st)); \
    } while (0)

// ---- host helpers (sbg_plan.cu) ----
uint32_t host_powmod(uint64_t a, uint64_t e, uint32_t p);
uint32_t host_shoup(uint32_t w, uint32_t p);
void host_prime_consts(PrimeConst out[SBG_NP]);
void host_crt_consts(CrtConst* out);
ShoupPair host_scale(int64_t L, int q);

// ---- launchers (sbg_kernels.cu) ----
cudaError_t upload_constants(cudaStream_t st);
// test hooks of the CRT kernel on the current device (SBG_INJECT_* bits)
cudaError_t set_inject(uint32_t mask);
// device allocation of the context's workspace and plan tables; fails on
// purpose while sbg_debug_fail_allocs has failures pending
cudaError_t dev_alloc(void** p, size_t bytes);
cudaError_t set_kernel_attributes();
size_t master_table_entries();
cudaError_t gen_master_tables(uint2* tw_f, uint2* tw_i, cudaStream_t st);
cudaError_t gen_len_tables(LenPlan* lp, cudaStream_t st);

// Whole product through the transform pipeline.  Workspace `ws` must hold
// ws_words(code) u32.  `err` is a device word that receives sticky error bits.
// Every `lgL` below is a length code.
size_t ws_words(int lgL, int sq);
// b_ready (optional): an event the second operand's arrival is recorded
// on; the first operand's forward transform does not wait for it.
cudaError_t launch_conv(const uint64_t* a, int64_t an, const uint64_t* b, int64_t bn, int sq,
                        int lgL, const LenPlan* lp, const uint2* tw_f, const uint2* tw_i,
                        uint32_t* ws, cudaStream_t st, KTimer* kt = nullptr,
                        cudaEvent_t b_ready = nullptr);
// CRT + carry of residues R (5 x L u32) into out[0..nout): out[m] = limb (m + off)
// of sum_{cmin <= j <= cmax} c_j * 2^(64 j).
cudaError_t launch_crt_carry(const uint32_t* R, int lgL, const LenPlan* lp, int64_t cmin,
                             int64_t cmax, int64_t off, uint64_t* out, int64_t nout,
                             uint32_t* flags, uint32_t* err, cudaStream_t st,
                             KTimer* kt = nullptr);
size_t carry_flag_words(int64_t nout);
// schoolbook products (sbg_school.cu): one, or one warp per job of a list
// (plain products: cmin = off = 0, nout = an + bn <= SBG_SCHOOL_MAX)
cudaError_t launch_school(const uint64_t* a, int64_t an, const uint64_t* b, int64_t bn,
                          uint64_t* out, cudaStream_t st);
cudaError_t launch_school_batch(const JobDesc* djobs, int njobs, cudaStream_t st);
// the persistent batch kernel over a work-item queue (sbg_kernels.cu); state
// = {queue head, one progress counter per job}, zeroed before every run;
// grid > 0: that many persistent CTAs, grid = 0: one CTA per item
cudaError_t launch_persist(const PItem* items, int nitems, const JobDesc* jobs, const PClass* cls,
                           uint32_t* state, const uint2* tw_f, const uint2* tw_i, uint32_t* err,
                           int grid, cudaStream_t st);
int persist_grid(int device);
size_t persist_smem_bytes();
// column tiles of a power-of-two four-step transform with 2^lgN1 rows
int col_tiles(int lgN1);
// u52 boundary (sbg_u52.cu): digits <- limbs; limbs <- redundant digits
// (scratch: u52_encode_scratch_words(rn) u32)
cudaError_t launch_u52_decode(uint64_t* d, int64_t n52, const uint64_t* a, int64_t an, cudaStream_t st);
size_t u52_encode_scratch_words(int64_t rn);
cudaError_t launch_u52_encode(uint64_t* r, int64_t rn, const uint64_t* d, int64_t n52, int sgn,
                              uint32_t* scratch, cudaStream_t st);
int64_t crt_blocks(int64_t nout);
// All stages of one size class of the batch engine (every job of length
// 2^lgL); `flags` holds flag_words zero-initialised words, job regions inside.
cudaError_t launch_batch_class(const JobDesc* djobs, int njobs, int lgL, const LenPlan* lp,
                               const uint2* tw_f, const uint2* tw_i, int64_t max_nout,
                               uint32_t* flags, size_t flag_words, uint32_t* err,
                               cudaStream_t st, KTimer* kt = nullptr);


// ---- the context (C ABI opaque type), shared by the library's TUs ----
// Per-launch CUDA event pairs, summed per kernel id by sbg_ctx_kernel_times.
struct EventTimer : KTimer {
    struct Rec {
        int kid;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int kid, cudaStream_t st) override {
        Rec r{kid, take(), nullptr};
        cudaEventRecord(r.a, st);
        recs.push_back(r);
    }
    void end(int kid, cudaStream_t st) override {
        for (size_t i = recs.size(); i-- > 0;)
            if (recs[i].kid == kid && recs[i].b == nullptr) {
                recs[i].b = take();
                cudaEventRecord(recs[i].b, st);
                return;
            }
    }
    void collect(double* ms, int64_t* cnt) {
        for (auto& r : recs) {
            if (r.b) {
                float t = 0.f;
                if (cudaEventSynchronize(r.b) == cudaSuccess &&
                    cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
                    ms[r.kid] += t;
                    cnt[r.kid] += 1;
                }
                pool.push_back(r.b);
            }
            pool.push_back(r.a);
        }
        recs.clear();
    }
    ~EventTimer() override {
        for (auto& r : recs) {
            cudaEventDestroy(r.a);
            if (r.b) cudaEventDestroy(r.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

// Stream-ordered upload of small descriptor arrays without allocation or
// synchronisation in steady state: bytes are copied into a pinned host ring
// and an asynchronous copy into the matching device ring is enqueued on the
// caller's stream.  Reusing ring bytes (wrap-around) or growing the ring
// first synchronises the streams of earlier pushes, so no copy or kernel
// still reading the reused bytes is in flight.  One host thread at a time.
struct UploadRing {
    uint8_t* h = nullptr;           // page-locked host buffer
    uint8_t* hd = nullptr;          //   its device address
    uint8_t* d = nullptr;
    size_t cap = 0, head = 0;
    int64_t pulls = 0;              // copy kernels launched (k_ring_pull)
    cudaStream_t last = nullptr;
    int push(const void* src, size_t bytes, cudaStream_t st, void** dev);
    void release();
};

// Internal job kind (not in the public header): the cyclic convolution of
// a (an limbs) and b (bn limbs) at the transform length code `reserved`
// (an, bn <= L), its L coefficients carried into rp[0 .. L+3) -- the value
// of which is a * b mod (B^L - 1) after an end-around fold.
#define SBG_JOB_CYCLIC 0x43

#define SBG_AUX_STREAMS 4
// transforms up to 2^12 points run in one CTA per prime (k_small)
#define SBG_SMALL_MAX_LG 12

// kernel launches of one product (or one length class of a batch): the
// fused single-CTA transform or the three four-step transforms, then CRT+carry
inline int class_launches(int lgL) {
    return lgL == SBG_CODE_SCHOOL ? 1 : (lgL <= SBG_SMALL_MAX_LG ? 2 : 4);
}
// codes in the order batches launch them: longest transforms first
inline int64_t code_order_key(int c) { return code_len(c); }

}  // namespace sbg

struct sbg_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    uint2* tw_f = nullptr;          // master tables [q][2^12]
    uint2* tw_i = nullptr;
    sbg::LenPlan plans[SBG_NCODES + 1];
    uint32_t* ws = nullptr;         // transform workspace (u32 words)
    size_t ws_cap = 0;
    uint32_t* flags = nullptr;      // carry look-back flags
    size_t flags_cap = 0;
    uint32_t* err = nullptr;        // sticky device error bits
    // staging for the host-pointer drop-ins, the stream their uploads run on
    // and the events that mark each operand's arrival
    uint64_t* d_stage = nullptr;
    size_t stage_cap = 0;
    cudaStream_t s_stage = nullptr;
    cudaEvent_t stage_a = nullptr, stage_b = nullptr, stage_go = nullptr;
    sbg::EventTimer* timer = nullptr;    // non-null while kernel timing is on
    // queued product lists (Newton division): grow-only arena for the
    // transforms and carry flags, descriptor ring, forked streams
    uint8_t* pw = nullptr;
    size_t pw_cap = 0;
    sbg::UploadRing ring;
    cudaStream_t aux[SBG_AUX_STREAMS] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[SBG_AUX_STREAMS] = {};
    // u52 boundary scratch (grow-only): packed operands, product, scan words
    uint64_t* u52buf = nullptr;
    size_t u52cap = 0;
    // division scratch (grow-only) and its error word
    uint64_t* dscr = nullptr;
    size_t dscr_cap = 0;
    uint32_t* derr = nullptr;
    std::atomic<int64_t> launches{0};   // kernels queued by this context (diagnostics)
    int stream_priority = 0;            // priority of the streams the context creates itself
    // 3 * 2^k transform lengths in use (bit k), by measurement where
    // sbg_ctx_autotune ran, else the default measured on B200
    uint32_t len3_mask = SBG_LEN3_DEFAULT;
    // host-operand products (sbg_mul_host): two staging slots so that one
    // product's download overlaps the next one's upload and compute
    struct HostSlot {
        uint64_t* d = nullptr;          // operands then result
        size_t cap = 0;                 // limbs
        cudaEvent_t in_done = nullptr, comp_done = nullptr, out_done = nullptr;
    };
    HostSlot hslot[2];
    cudaStream_t s_in = nullptr, s_out = nullptr;
    int hnext = 0;
};

namespace sbg {
int cuda_fail(cudaError_t e, const char* where);
int lg_ceil(int64_t n);
int conv_lg(int64_t need, uint32_t mask3);
int ensure_plan(sbg_ctx* c, int lgL);
// Newton reciprocals of `count` normalised divisors (device pointers), all
// recursion levels in lockstep; synchronous on the context stream.
int recip_batch(sbg_ctx* c, const uint64_t* const* D, uint64_t* const* V, const int64_t* n,
                int count);
size_t div_scratch_limbs(int64_t n);
// Enqueue a list of products (sbg_job) on the context stream: one launch
// sequence per transform-length class on forked streams, joined back.  No
// allocation or synchronisation once the context's arena and ring have grown
// to the largest list seen.  Device error bits go to `err` (null: the
// context's own word).
int enqueue_products(sbg_ctx* c, const sbg_job* jobs, int64_t count, uint32_t* err = nullptr);
// host-operand pipeline of a context: wait for its copies / free it
int host_pipe_sync(sbg_ctx* c);
void host_pipe_release(sbg_ctx* c);
}  // namespace sbg

