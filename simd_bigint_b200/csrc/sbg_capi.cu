// sbg_capi.cu -- the C ABI: contexts, plans, workspace, and the mul / sqr /
// mulmid entry points (include/simd_bigint_b200.h).
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "../../include/simd_bigint_b200.h"
#include "sbg_internal.h"

using namespace sbg;

namespace sbg {
int cuda_fail(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return SBG_OK;
    if (getenv("SBG_DEBUG")) fprintf(stderr, "sbg: %s: %s\n", where, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return SBG_EALLOC;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SBG_ENODEV;
    return SBG_ECUDA;
}
#define CK(call)                                            \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

static std::atomic<int> g_fail_allocs{0};

cudaError_t dev_alloc(void** p, size_t bytes) {
    int n = g_fail_allocs.load();
    while (n > 0)
        if (g_fail_allocs.compare_exchange_weak(n, n - 1)) return cudaErrorMemoryAllocation;
    return cudaMalloc(p, bytes);
}

int lg_ceil(int64_t n) {
    int l = 0;
    while (((int64_t)1 << l) < n) ++l;
    return l;
}

// Transform length (code) for a convolution whose wanted coefficients need
// L >= need: 2^a >= need, or 3 * 2^b >= need when that is shorter and bit b
// of `mask3` allows it (the context's choice per size class, sbg_ctx_autotune).
int conv_lg(int64_t need, uint32_t mask3) {
    int l = lg_ceil(need);
    if (l < 4) l = 4;
    int k = lg_ceil((need + 2) / 3);
    if (k >= SBG_THREE_MIN_LG && k <= SBG_MAX_LG - 2 && ((int64_t)3 << k) < ((int64_t)1 << l) &&
        ((mask3 >> k) & 1u))
        return SBG_CODE3 + k;
    return l;
}

int ensure_plan(sbg_ctx* c, int lgL) {
    LenPlan* lp = &c->plans[lgL];
    if (lp->lgL == lgL) return SBG_OK;
    LenPlan np;
    np.lgL = lgL;
    np.L = code_len(lgL);
    if (lgL <= 12) {
        np.lgN1 = 0;
        np.lgN2 = lgL;
    } else {
        np.lgN2 = 12;
        if (code_three(lgL)) {
            np.m3 = code_lg(lgL) - 12;
            np.lgN1 = 0;
        } else {
            np.lgN1 = lgL - 12;
        }
        np.hi_n = (int)(np.L >> 13);
        size_t lo_b = (size_t)SBG_NP * 8192 * sizeof(uint2);
        size_t hi_b = (size_t)SBG_NP * np.hi_n * sizeof(uint2);
        const size_t t3_b = np.m3 >= 0 ? (size_t)SBG_NP * (2 << np.m3) * sizeof(uint2) : 0;
        uint2** bufs[6] = {&np.fs_lo_f, &np.fs_lo_i, &np.fs_hi_f, &np.fs_hi_i, &np.t3_f, &np.t3_i};
        const size_t sizes[6] = {lo_b, lo_b, hi_b, hi_b, t3_b, t3_b};
        for (int k = 0; k < 6; ++k) {
            if (!sizes[k]) continue;
            cudaError_t e = dev_alloc((void**)bufs[k], sizes[k]);
            if (e != cudaSuccess) {                 // nothing of the plan is kept
                for (int j = 0; j < k; ++j)
                    if (*bufs[j]) cudaFree(*bufs[j]);
                return cuda_fail(e, "plan tables");
            }
        }
        if (np.m3 >= 0) {
            for (int q = 0; q < SBG_NP; ++q) {     // cube roots of unity w_N1^M
                const uint32_t p = kPrimes[q];
                const uint32_t w = host_powmod(kGenerators[q], (p - 1) / 3, p);
                const uint32_t wi = host_powmod(w, 2, p);
                np.w3f[q] = w;
                np.w3fs[q] = host_shoup(w, p);
                np.w3i[q] = wi;
                np.w3is[q] = host_shoup(wi, p);
            }
        }
        CK(gen_len_tables(&np, c->stream));
    }
    for (int q = 0; q < SBG_NP; ++q) np.scale[q] = host_scale(np.L, q);
    *lp = np;
    return SBG_OK;
}

}  // namespace sbg

static int ensure_ws(sbg_ctx* c, size_t words, size_t flag_words) {
    if (words > c->ws_cap) {
        CK(cudaStreamSynchronize(c->stream));
        if (c->ws) cudaFree(c->ws);
        c->ws = nullptr;
        c->ws_cap = 0;
        CK(dev_alloc((void**)&c->ws, words * sizeof(uint32_t)));
        c->ws_cap = words;
    }
    if (flag_words > c->flags_cap) {
        CK(cudaStreamSynchronize(c->stream));
        if (c->flags) cudaFree(c->flags);
        c->flags = nullptr;
        c->flags_cap = 0;
        size_t fw = flag_words < 4096 ? 4096 : flag_words;
        CK(dev_alloc((void**)&c->flags, fw * sizeof(uint32_t)));
        c->flags_cap = fw;
    }
    return SBG_OK;
}

// One windowed convolution: the limbs [off, off + nout) of
// sum_{cmin <= j <= cmax} c_j 2^(64 j) where c = a * b (cyclic length 2^lgL).
static int run_conv(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp,
                    int64_t bn, int sq, int lgL, int64_t cmin, int64_t cmax, int64_t off,
                    int64_t nout, cudaEvent_t b_ready = nullptr) {
    if (lgL > SBG_NCODES || code_len(lgL) > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
    int st = ensure_plan(c, lgL);
    if (st) return st;
    st = ensure_ws(c, ws_words(lgL, sq), carry_flag_words(nout));
    if (st) return st;
    const LenPlan* lp = &c->plans[lgL];
    CK(launch_conv(ap, an, bp, bn, sq, lgL, lp, c->tw_f, c->tw_i, c->ws, c->stream, c->timer, b_ready));
    CK(launch_crt_carry(c->ws, lgL, lp, cmin, cmax, off, rp, nout, c->flags, c->err, c->stream,
                        c->timer));
    // the split forward columns (b_ready on the four-step path) are two launches
    c->launches += class_launches(lgL) + ((b_ready && !sq && lgL > SBG_SMALL_MAX_LG && lp->m3 < 0) ? 1 : 0);
    return SBG_OK;
}

// A plain product of at most SBG_SCHOOL_MAX limbs: one schoolbook warp.
static int run_school(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp,
                      int64_t bn) {
    KT_BEGIN(c->timer, KID_SMALL, c->stream);
    CK(launch_school(ap, an, bp, bn, rp, c->stream));
    KT_END(c->timer, KID_SMALL, c->stream);
    c->launches += 1;
    return SBG_OK;
}

// ---- batch engine -----------------------------------------------------------
// Jobs are bucketed by transform length; each size class is one launch per
// stage covering all its jobs (blocks -> job by index arithmetic), and the
// classes run on forked streams.  A batch can be captured into a CUDA graph
// once and replayed.

#define SBG_BATCH_STREAMS 4

struct sbg_batch {
    sbg_ctx* ctx = nullptr;
    struct Cls {
        int lgL;
        int njobs;
        int64_t max_nout;
        JobDesc* djobs;
        uint32_t* flags;
        size_t flag_words;
    };
    std::vector<Cls> classes;
    void* dmem = nullptr;
    cudaStream_t aux[SBG_BATCH_STREAMS] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[SBG_BATCH_STREAMS] = {};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t count = 0;
    // engine: 0 = the persistent kernel over a work-item queue for the
    // classes it runs (the others keep per-class launches), 1 = per-class
    // launches for every class (the default: the fastest on the mixed
    // 4096-product batch on B200), 2 = the same queue with one CTA per item
    int engine = 1;
    std::vector<JobDesc> host_jobs;      // descriptors, in device order
    std::vector<int> job_code;           // length code of each
    JobDesc* djobs_all = nullptr;
    void* pmem = nullptr;                // items, progress state, class table
    PItem* d_items = nullptr;
    int nitems = 0;
    uint32_t* d_state = nullptr;         // queue head + one progress counter per job
    size_t state_words = 0;
    PClass* d_cls = nullptr;
    size_t wave_bytes = (size_t)64 << 20;
    int grid = 0;
};

static bool batch_uses_persist(const sbg_batch* b) { return b->engine != 1 && b->nitems > 0; }

static int job_shape(const sbg_job& j, uint32_t mask3, int* lgL, int64_t* cmin, int64_t* cmax,
                     int64_t* off, int64_t* nout, int* sq) {
    if (!j.rp || !j.ap || j.an <= 0) return SBG_EINVAL;
    switch (j.kind) {
        case SBG_JOB_MUL:
            if (!j.bp || j.bn <= 0) return SBG_EINVAL;
            if (j.an + j.bn - 1 > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
            *lgL = j.an + j.bn <= SBG_SCHOOL_MAX ? SBG_CODE_SCHOOL : conv_lg(j.an + j.bn - 1, mask3);
            *cmin = 0; *cmax = j.an + j.bn - 2; *off = 0; *nout = j.an + j.bn; *sq = 0;
            return SBG_OK;
        case SBG_JOB_SQR:
            if (2 * j.an - 1 > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
            *lgL = 2 * j.an <= SBG_SCHOOL_MAX ? SBG_CODE_SCHOOL : conv_lg(2 * j.an - 1, mask3);
            *cmin = 0; *cmax = 2 * j.an - 2; *off = 0; *nout = 2 * j.an; *sq = 1;
            return SBG_OK;
        case SBG_JOB_CYCLIC: {
            if (!j.bp || j.bn <= 0 || j.reserved < 0 || j.reserved > SBG_NCODES) return SBG_EINVAL;
            const int64_t L = code_len(j.reserved);
            if (L > ((int64_t)1 << SBG_MAX_LG) || j.an > L || j.bn > L) return SBG_EINVAL;
            *lgL = j.reserved;
            *cmin = 0; *cmax = L - 1; *off = 0; *nout = L + 3; *sq = 0;
            return SBG_OK;
        }
        case SBG_JOB_MULMID:
            if (!j.bp || j.bn <= 0 || j.an < j.bn) return SBG_EINVAL;
            if (j.an > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
            *lgL = conv_lg(j.an, mask3);
            *cmin = j.bn - 1; *cmax = j.an - 1; *off = j.bn - 1; *nout = j.an - j.bn + 3; *sq = 0;
            return SBG_OK;
        default: return SBG_EINVAL;
    }
}

static int batch_launch(sbg_batch* b, KTimer* kt) {
    sbg_ctx* c = b->ctx;
    const bool pers = batch_uses_persist(b);
    CK(cudaEventRecord(b->fork, c->stream));
    for (int k = 0; k < SBG_BATCH_STREAMS; ++k) CK(cudaStreamWaitEvent(b->aux[k], b->fork, 0));
    int k = 0;
    for (size_t i = 0; i < b->classes.size(); ++i) {
        const auto& cl = b->classes[i];
        if (pers && persist_code(cl.lgL)) continue;
        cudaStream_t st = b->aux[k++ % SBG_BATCH_STREAMS];
        CK(launch_batch_class(cl.djobs, cl.njobs, cl.lgL, &c->plans[cl.lgL], c->tw_f, c->tw_i,
                              cl.max_nout, cl.flags, cl.flag_words, c->err, st, kt));
    }
    if (pers) {
        CK(cudaMemsetAsync(b->d_state, 0, b->state_words * sizeof(uint32_t), c->stream));
        for (const auto& cl : b->classes)
            if (persist_code(cl.lgL) && cl.flag_words)
                CK(cudaMemsetAsync(cl.flags, 0, cl.flag_words * sizeof(uint32_t), c->stream));
        KT_BEGIN(kt, KID_BATCH, c->stream);
        CK(launch_persist(b->d_items, b->nitems, b->djobs_all, b->d_cls, b->d_state, c->tw_f, c->tw_i,
                          c->err, b->engine == 2 ? 0 : b->grid, c->stream));
        KT_END(kt, KID_BATCH, c->stream);
    }
    for (int j = 0; j < SBG_BATCH_STREAMS; ++j) {
        CK(cudaEventRecord(b->join[j], b->aux[j]));
        CK(cudaStreamWaitEvent(c->stream, b->join[j], 0));
    }
    return SBG_OK;
}

// kernel launches of one run of the batch
static int64_t batch_run_launches(const sbg_batch* b) {
    int64_t n = 0;
    const bool pers = batch_uses_persist(b);
    for (const auto& cl : b->classes)
        if (!(pers && persist_code(cl.lgL))) n += class_launches(cl.lgL);
    return n + (pers ? 1 : 0);
}

// The persistent engine's work-item queue: jobs of the classes the
// persistent kernel runs, cut into waves of about wave_bytes of transform
// workspace; step t of the queue holds the carry blocks of wave t - 3, the
// inverse columns of wave t - 2, the rows of wave t - 1 and the forward
// columns (or single-CTA transforms) of wave t, so that every item comes
// after the items it waits for and a stage's input is recent in L2.
static int persist_build(sbg_batch* b) {
    sbg_ctx* c = b->ctx;
    struct Wave {
        std::vector<PItem> s[4];
    };
    std::vector<Wave> waves(1);
    size_t acc = 0;
    std::vector<int> order;                       // job indices, longest transforms first
    for (size_t j = 0; j < b->host_jobs.size(); ++j)
        if (persist_code(b->job_code[j])) order.push_back((int)j);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return code_order_key(b->job_code[x]) > code_order_key(b->job_code[y]);
    });
    // items that wait for nothing -- whole single-CTA products and groups of
    // up to 8 consecutive schoolbook products -- go to the end of the queue
    std::vector<PItem> tail;
    int sch_first = -1, sch_n = 0;
    auto flush_school = [&]() {
        if (sch_n) tail.push_back(PItem{(uint32_t)sch_first, PK_SCHOOL, SBG_CODE_SCHOOL, (uint32_t)sch_n, 0});
        sch_first = -1;
        sch_n = 0;
    };
    for (int j : order) {
        const int l = b->job_code[j];
        const JobDesc& d = b->host_jobs[j];
        if (l == SBG_CODE_SCHOOL) {
            if (sch_n == PERSIST_THREADS / 32 || (sch_n && sch_first + sch_n != j)) flush_school();
            if (!sch_n) sch_first = j;
            ++sch_n;
            continue;
        }
        const uint32_t nb = (uint32_t)crt_blocks(d.nout);
        const uint16_t lg = (uint16_t)l;
        if (l <= SBG_SMALL_MAX_LG) {
            tail.push_back(PItem{(uint32_t)j, PK_SMALLJOB, lg, nb, 0});
            continue;
        }
        const size_t wsb = ws_words(l, d.sq) * 4;
        if (acc && acc + wsb > b->wave_bytes) {
            waves.emplace_back();
            acc = 0;
        }
        acc += wsb;
        Wave& w = waves.back();
        const int lgN1 = l - 12;
        const uint32_t nt = (uint32_t)col_tiles(lgN1);
        const uint32_t nops = d.sq ? 1 : 2;
        const uint32_t n_colf = nops * nt * SBG_NP, n_row = ((uint32_t)SBG_NP << lgN1) / PERSIST_ROWS,
                       n_coli = nt * SBG_NP, n_crt = (nb + PERSIST_CRT - 1) / PERSIST_CRT;
        for (uint32_t i = 0; i < n_colf; ++i) w.s[0].push_back(PItem{(uint32_t)j, PK_COLF, lg, i, 0});
        for (uint32_t i = 0; i < n_row; ++i) w.s[1].push_back(PItem{(uint32_t)j, PK_ROW, lg, i, n_colf});
        for (uint32_t i = 0; i < n_coli; ++i) w.s[2].push_back(PItem{(uint32_t)j, PK_COLI, lg, i, n_colf + n_row});
        for (uint32_t k = 0; k < n_crt; ++k)
            w.s[3].push_back(PItem{(uint32_t)j, PK_CRT, lg, k, n_colf + n_row + n_coli});
    }
    flush_school();
    std::vector<PItem> q;
    const int nw = (int)waves.size();
    for (int t = 0; t < nw + 3; ++t)
        for (int st = 3; st >= 0; --st) {
            const int w = t - st;
            if (w >= 0 && w < nw) q.insert(q.end(), waves[w].s[st].begin(), waves[w].s[st].end());
        }
    q.insert(q.end(), tail.begin(), tail.end());
    // class table, items and progress state in one allocation
    std::vector<PClass> cls(SBG_NCODES + 1);
    for (int l = 0; l <= SBG_NCODES; ++l) {
        const LenPlan& lp = c->plans[l];
        if (lp.lgL != l) continue;
        cls[l].fsf = FsTables{lp.fs_lo_f, lp.fs_hi_f, lp.hi_n};
        cls[l].fsi = FsTables{lp.fs_lo_i, lp.fs_hi_i, lp.hi_n};
        for (int p = 0; p < SBG_NP; ++p) {
            cls[l].sc.w[p] = lp.scale[p].w;
            cls[l].sc.ws[p] = lp.scale[p].ws;
        }
    }
    const size_t cls_b = cls.size() * sizeof(PClass);
    const size_t items_b = q.size() * sizeof(PItem);
    const size_t state_w = 1 + b->host_jobs.size();
    const size_t off_items = (cls_b + 255) & ~(size_t)255;
    const size_t off_state = (off_items + items_b + 255) & ~(size_t)255;
    const size_t total = off_state + state_w * sizeof(uint32_t);
    if (b->pmem) {
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(b->pmem);
        b->pmem = nullptr;
    }
    CK(cudaMalloc(&b->pmem, total));
    uint8_t* base = (uint8_t*)b->pmem;
    b->d_cls = (PClass*)base;
    b->d_items = (PItem*)(base + off_items);
    b->d_state = (uint32_t*)(base + off_state);
    b->state_words = state_w;
    b->nitems = (int)q.size();
    CK(cudaMemcpy(b->d_cls, cls.data(), cls_b, cudaMemcpyHostToDevice));
    if (items_b) CK(cudaMemcpy(b->d_items, q.data(), items_b, cudaMemcpyHostToDevice));
    b->grid = persist_grid(c->device);
    if (b->grid <= 0) return SBG_ECUDA;
    return SBG_OK;
}

namespace sbg {

// Descriptor uploads are pulled by a kernel from the ring's page-locked
// host buffer (device-addressable), not copied by a DMA engine: a caller's
// large host<->device copies queued on the copy engines would otherwise
// delay every batch's small descriptor upload behind them.
__global__ void k_ring_pull(uint4* __restrict__ dst, const uint4* __restrict__ src, size_t n16) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

int UploadRing::push(const void* src, size_t bytes, cudaStream_t st, void** dev) {
    const size_t need = (bytes + 255) & ~(size_t)255;
    if (need > cap || head + need > cap) {
        // the bytes about to be reused may still feed a copy or a kernel
        if (last && last != st && cudaStreamSynchronize(last) != cudaSuccess) return SBG_ECUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return SBG_ECUDA;
        head = 0;
        if (need > cap) {
            release();
            // 32 MB: a 1024-division batch uploads about 4.5 MB of descriptors,
            // so the ring wraps (and drains the stream) once every few calls
            const size_t nc = std::max(need * 4, (size_t)32 << 20);
            if (cudaHostAlloc(&h, nc, cudaHostAllocMapped) != cudaSuccess) return SBG_EALLOC;
            if (cudaHostGetDevicePointer((void**)&hd, h, 0) != cudaSuccess) {
                cudaFreeHost(h);
                h = nullptr;
                return SBG_EALLOC;
            }
            if (cudaMalloc(&d, nc) != cudaSuccess) {
                cudaFreeHost(h);
                h = nullptr;
                return SBG_EALLOC;
            }
            cap = nc;
        }
    }
    std::memcpy(h + head, src, bytes);
    if (bytes) {
        const size_t n16 = need / 16;      // the whole 256-byte-rounded block
        const unsigned blocks = (unsigned)std::min<size_t>((n16 + 255) / 256, 64);
        k_ring_pull<<<blocks, 256, 0, st>>>((uint4*)(d + head), (const uint4*)(hd + head), n16);
        if (cudaGetLastError() != cudaSuccess) return SBG_ECUDA;
        ++pulls;
    }
    *dev = d + head;
    head += need;
    last = st;
    return SBG_OK;
}

void UploadRing::release() {
    if (h) cudaFreeHost(h);
    if (d) cudaFree(d);
    h = nullptr;
    hd = nullptr;
    d = nullptr;
    cap = head = 0;
}

int enqueue_products(sbg_ctx* c, const sbg_job* jobs, int64_t count, uint32_t* err) {
    if (count <= 0) return SBG_OK;
    std::vector<JobDesc> by_lg[SBG_NCODES + 1];
    int64_t max_nout[SBG_NCODES + 1] = {};
    for (int64_t i = 0; i < count; ++i) {
        int lgL, sq;
        int64_t cmin, cmax, off, nout;
        int st = job_shape(jobs[i], c->len3_mask, &lgL, &cmin, &cmax, &off, &nout, &sq);
        if (st) return st;
        JobDesc d{};
        d.a = jobs[i].ap;
        d.b = sq ? jobs[i].ap : jobs[i].bp;
        d.out = jobs[i].rp;
        d.an = jobs[i].an;
        d.bn = sq ? jobs[i].an : jobs[i].bn;
        d.cmin = cmin; d.cmax = cmax; d.off = off; d.nout = nout;
        d.sq = sq;
        by_lg[lgL].push_back(d);
        max_nout[lgL] = std::max(max_nout[lgL], nout);
    }
    size_t ws_total = 0, flag_total = 0;
    for (int l = 0; l <= SBG_NCODES; ++l) {
        if (by_lg[l].empty()) continue;
        int st = ensure_plan(c, l);
        if (st) return st;
        for (auto& d : by_lg[l]) ws_total += ws_words(l, d.sq);
        flag_total += by_lg[l].size() * ((size_t)crt_blocks(max_nout[l]) + 1 + 3) / 4 * 4;
    }
    const size_t bytes = (ws_total + flag_total) * 4;
    if (bytes > c->pw_cap) {
        // earlier lists on this stream may still use the arena
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(c->pw);
        c->pw = nullptr;
        c->pw_cap = 0;
        const size_t nb = bytes + bytes / 4;
        CK(cudaMalloc(&c->pw, nb));
        c->pw_cap = nb;
    }
    if (!c->fork) {
        for (int k = 0; k < SBG_AUX_STREAMS; ++k) {
            CK(cudaStreamCreateWithPriority(&c->aux[k], cudaStreamNonBlocking, c->stream_priority));
            CK(cudaEventCreateWithFlags(&c->join[k], cudaEventDisableTiming));
        }
        CK(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    }
    uint32_t* ws = (uint32_t*)c->pw;
    uint32_t* fl = ws + ws_total;
    struct Cls {
        int lgL, njobs;
        size_t first, flag_words;
        uint32_t* flags;
    };
    std::vector<Cls> cls;
    std::vector<JobDesc> all;
    all.reserve((size_t)count);
    int order[SBG_NCODES + 1];                        // longest transforms first
    for (int l = 0; l <= SBG_NCODES; ++l) order[l] = l;
    std::stable_sort(order, order + SBG_NCODES + 1,
                     [](int x, int y) { return code_order_key(x) > code_order_key(y); });
    for (int oi = 0; oi <= SBG_NCODES; ++oi) {
        const int l = order[oi];
        if (by_lg[l].empty()) continue;
        const size_t fpj = ((size_t)crt_blocks(max_nout[l]) + 1 + 3) / 4 * 4;
        cls.push_back(Cls{l, (int)by_lg[l].size(), all.size(), fpj * by_lg[l].size(), fl});
        for (auto& d : by_lg[l]) {
            d.ws = ws;
            ws += ws_words(l, d.sq);
            d.flags = fl;
            fl += fpj;
            all.push_back(d);
        }
    }
    void* dd = nullptr;
    int st = c->ring.push(all.data(), all.size() * sizeof(JobDesc), c->stream, &dd);
    if (st) return st;
    CK(cudaEventRecord(c->fork, c->stream));
    const int nst = std::min<int>(SBG_AUX_STREAMS, (int)cls.size());
    for (int k = 0; k < nst; ++k) CK(cudaStreamWaitEvent(c->aux[k], c->fork, 0));
    for (size_t i = 0; i < cls.size(); ++i) {
        const Cls& k = cls[i];
        CK(launch_batch_class((const JobDesc*)dd + k.first, k.njobs, k.lgL, &c->plans[k.lgL], c->tw_f,
                              c->tw_i, max_nout[k.lgL], k.flags, k.flag_words, err ? err : c->err,
                              c->aux[i % SBG_AUX_STREAMS], c->timer));
        c->launches += class_launches(k.lgL);
    }
    for (int k = 0; k < nst; ++k) {
        CK(cudaEventRecord(c->join[k], c->aux[k]));
        CK(cudaStreamWaitEvent(c->stream, c->join[k], 0));
    }
    return SBG_OK;
}

}  // namespace sbg

extern "C" {

const char* sbg_strerror(int status) {
    switch (status) {
        case SBG_OK: return "ok";
        case SBG_EINVAL: return "invalid argument";
        case SBG_EBAND: return "operands beyond the transform band";
        case SBG_EALLOC: return "device allocation failed";
        case SBG_ECUDA: return "CUDA runtime error";
        case SBG_ETIMEOUT: return "bounded device wait expired";
        case SBG_ESPILL: return "product spilled past its top limb";
        case SBG_EADMIT: return "request rejected by admission control";
        case SBG_ENODEV: return "no CUDA device";
        case SBG_ECANCELED: return "request cancelled before it was launched";
        default: return "unknown status";
    }
}

int64_t sbg_max_total_limbs(void) { return ((int64_t)1 << SBG_MAX_LG) + 1; }

int sbg_ctx_create(int device, sbg_ctx** out) {
    if (!out) return SBG_EINVAL;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return SBG_ENODEV;
    if (device < 0 || device >= ndev) return SBG_EINVAL;
    CK(cudaSetDevice(device));
    sbg_ctx* c = new sbg_ctx();
    c->device = device;
    int st = SBG_OK;
    do {
        if ((st = cuda_fail(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking),
                            "stream")))
            break;
        c->stream = c->own_stream;
        if ((st = cuda_fail(set_kernel_attributes(), "attributes"))) break;
        if ((st = cuda_fail(upload_constants(c->stream), "constants"))) break;
        size_t tb = master_table_entries() * sizeof(uint2);
        if ((st = cuda_fail(cudaMalloc(&c->tw_f, tb), "tw_f"))) break;
        if ((st = cuda_fail(cudaMalloc(&c->tw_i, tb), "tw_i"))) break;
        if ((st = cuda_fail(gen_master_tables(c->tw_f, c->tw_i, c->stream), "tables"))) break;
        if ((st = cuda_fail(cudaMalloc(&c->err, sizeof(uint32_t)), "err"))) break;
        if ((st = cuda_fail(cudaMemsetAsync(c->err, 0, sizeof(uint32_t), c->stream), "err0")))
            break;
        if ((st = cuda_fail(cudaStreamSynchronize(c->stream), "sync"))) break;
    } while (0);
    if (st) {
        sbg_ctx_destroy(c);
        return st;
    }
    *out = c;
    return SBG_OK;
}

void sbg_ctx_destroy(sbg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int l = 0; l <= SBG_NCODES; ++l) {
        LenPlan* lp = &c->plans[l];
        cudaFree(lp->t3_f);
        cudaFree(lp->t3_i);
        cudaFree(lp->fs_lo_f);
        cudaFree(lp->fs_lo_i);
        cudaFree(lp->fs_hi_f);
        cudaFree(lp->fs_hi_i);
    }
    cudaFree(c->tw_f);
    cudaFree(c->tw_i);
    cudaFree(c->ws);
    cudaFree(c->flags);
    cudaFree(c->err);
    cudaFree(c->d_stage);
    if (c->s_stage) cudaStreamDestroy(c->s_stage);
    if (c->stage_a) cudaEventDestroy(c->stage_a);
    if (c->stage_b) cudaEventDestroy(c->stage_b);
    if (c->stage_go) cudaEventDestroy(c->stage_go);
    host_pipe_release(c);
    cudaFree(c->pw);
    cudaFree(c->dscr);
    cudaFree(c->derr);
    cudaFree(c->u52buf);
    c->ring.release();
    for (int k = 0; k < SBG_AUX_STREAMS; ++k) {
        if (c->aux[k]) cudaStreamDestroy(c->aux[k]);
        if (c->join[k]) cudaEventDestroy(c->join[k]);
    }
    if (c->fork) cudaEventDestroy(c->fork);
    delete c->timer;
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

int sbg_ctx_set_stream(sbg_ctx* c, void* stream) {
    if (!c) return SBG_EINVAL;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return SBG_OK;
}

void* sbg_ctx_get_stream(sbg_ctx* c) { return c ? (void*)c->stream : nullptr; }

int sbg_ctx_sync(sbg_ctx* c) {
    if (!c) return SBG_EINVAL;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (host_pipe_sync(c) != SBG_OK) return SBG_ECUDA;
    uint32_t h = 0;
    CK(cudaMemcpy(&h, c->err, sizeof(h), cudaMemcpyDeviceToHost));
    if (h) {
        CK(cudaMemset(c->err, 0, sizeof(uint32_t)));
        if (h & 1u) return SBG_ETIMEOUT;
        if (h & 2u) return SBG_ESPILL;
        return SBG_ECUDA;
    }
    return SBG_OK;
}

int sbg_ctx_set_timing(sbg_ctx* c, int on) {
    if (!c) return SBG_EINVAL;
    CK(cudaSetDevice(c->device));
    if (on && !c->timer) c->timer = new EventTimer();
    if (!on && c->timer) {
        cudaStreamSynchronize(c->stream);
        delete c->timer;
        c->timer = nullptr;
    }
    return SBG_OK;
}

int sbg_ctx_kernel_times(sbg_ctx* c, double* ms, int64_t* counts, int n) {
    if (!c || !ms || !counts || n < KID_COUNT) return SBG_EINVAL;
    for (int i = 0; i < n; ++i) {
        ms[i] = 0.0;
        counts[i] = 0;
    }
    if (!c->timer) return SBG_OK;
    CK(cudaSetDevice(c->device));
    c->timer->collect(ms, counts);
    return SBG_OK;
}

int sbg_ctx_reserve(sbg_ctx* c, int64_t total) {
    if (!c || total < 2) return SBG_EINVAL;
    if (total - 1 > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
    CK(cudaSetDevice(c->device));
    int lg = conv_lg(total - 1, c->len3_mask);
    for (int l = 4; l <= SBG_NCODES; ++l) {            // every length up to the largest
        if (l > SBG_MAX_LG && l < SBG_CODE3 + SBG_THREE_MIN_LG) continue;
        if (code_len(l) > code_len(lg)) continue;
        int st = ensure_plan(c, l);
        if (st) return st;
    }
    int st = ensure_ws(c, ws_words(lg, 0), carry_flag_words(total));
    if (st) return st;
    CK(cudaStreamSynchronize(c->stream));
    return SBG_OK;
}

int sbg_mul(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp,
            int64_t bn) {
    if (!c || !rp || !ap || !bp || an <= 0 || bn <= 0) return SBG_EINVAL;
    if (an + bn - 1 > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
    CK(cudaSetDevice(c->device));
    if (an + bn <= SBG_SCHOOL_MAX) return run_school(c, rp, ap, an, bp, bn);
    int lgL = conv_lg(an + bn - 1, c->len3_mask);
    return run_conv(c, rp, ap, an, bp, bn, 0, lgL, 0, an + bn - 2, 0, an + bn);
}

int sbg_sqr(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an) {
    if (!c || !rp || !ap || an <= 0) return SBG_EINVAL;
    if (2 * an - 1 > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
    CK(cudaSetDevice(c->device));
    if (2 * an <= SBG_SCHOOL_MAX) return run_school(c, rp, ap, an, ap, an);
    int lgL = conv_lg(2 * an - 1, c->len3_mask);
    return run_conv(c, rp, ap, an, ap, an, 1, lgL, 0, 2 * an - 2, 0, 2 * an);
}

void sbg_batch_destroy(sbg_batch* b) {
    if (!b) return;
    if (b->ctx) {
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
    }
    for (int k = 0; k < SBG_BATCH_STREAMS; ++k) {
        if (b->aux[k]) cudaStreamSynchronize(b->aux[k]);
    }
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (int k = 0; k < SBG_BATCH_STREAMS; ++k) {
        if (b->aux[k]) cudaStreamDestroy(b->aux[k]);
        if (b->join[k]) cudaEventDestroy(b->join[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    cudaFree(b->dmem);
    cudaFree(b->pmem);
    delete b;
}

int sbg_batch_create(sbg_ctx* c, const sbg_job* jobs, int64_t count, sbg_batch** out) {
    if (!c || !out || (count > 0 && !jobs) || count < 0) return SBG_EINVAL;
    *out = nullptr;
    CK(cudaSetDevice(c->device));
    // bucket by transform length
    std::vector<std::vector<JobDesc>> by_lg(SBG_NCODES + 1);
    std::vector<int64_t> max_nout(SBG_NCODES + 1, 0);
    for (int64_t i = 0; i < count; ++i) {
        int lgL, sq;
        int64_t cmin, cmax, off, nout;
        int st = job_shape(jobs[i], c->len3_mask, &lgL, &cmin, &cmax, &off, &nout, &sq);
        if (st) return st;
        JobDesc d{};
        d.a = jobs[i].ap;
        d.b = sq ? jobs[i].ap : jobs[i].bp;
        d.out = jobs[i].rp;
        d.an = jobs[i].an;
        d.bn = sq ? jobs[i].an : jobs[i].bn;
        d.cmin = cmin; d.cmax = cmax; d.off = off; d.nout = nout;
        d.sq = sq;
        by_lg[lgL].push_back(d);
        if (nout > max_nout[lgL]) max_nout[lgL] = nout;
    }
    // sizes: workspace, flags, descriptors -- one allocation
    size_t ws_total = 0, flag_total = 0, desc_total = 0;
    for (int l = 0; l <= SBG_NCODES; ++l) {
        if (by_lg[l].empty()) continue;
        int st = ensure_plan(c, l);
        if (st) return st;
        const size_t bpj = (size_t)crt_blocks(max_nout[l]);
        for (auto& d : by_lg[l]) ws_total += ws_words(l, d.sq);
        flag_total += by_lg[l].size() * (bpj + 1 + 3) / 4 * 4;
        desc_total += by_lg[l].size();
    }
    sbg_batch* b = new sbg_batch();
    b->ctx = c;
    b->count = count;
    size_t bytes = ws_total * 4 + flag_total * 4 + desc_total * sizeof(JobDesc) + 1024;
    int st = cuda_fail(cudaMalloc(&b->dmem, bytes), "batch workspace");
    if (st) {
        sbg_batch_destroy(b);
        return st;
    }
    uint32_t* ws = (uint32_t*)b->dmem;
    uint32_t* fl = ws + ws_total;
    JobDesc* dd = (JobDesc*)(((uintptr_t)(fl + flag_total) + 255) & ~(uintptr_t)255);
    std::vector<JobDesc> host_all;
    host_all.reserve(desc_total);
    for (int l = 0; l <= SBG_NCODES; ++l) {
        if (by_lg[l].empty()) continue;
        const size_t bpj = (size_t)crt_blocks(max_nout[l]);
        const size_t fpj = (bpj + 1 + 3) / 4 * 4;
        sbg_batch::Cls cl;
        cl.lgL = l;
        cl.njobs = (int)by_lg[l].size();
        cl.max_nout = max_nout[l];
        cl.djobs = dd + host_all.size();
        cl.flags = fl;
        cl.flag_words = fpj * by_lg[l].size();
        for (auto& d : by_lg[l]) {
            d.ws = ws;
            ws += ws_words(l, d.sq);
            d.flags = fl;
            fl += fpj;
            host_all.push_back(d);
        }
        b->classes.push_back(cl);
    }
    b->host_jobs = host_all;
    b->djobs_all = dd;
    for (int l = 0; l <= SBG_NCODES; ++l)
        for (size_t k = 0; k < by_lg[l].size(); ++k) b->job_code.push_back(l);
    // largest classes first: they start early on the forked streams
    std::stable_sort(b->classes.begin(), b->classes.end(),
                     [](const sbg_batch::Cls& x, const sbg_batch::Cls& y) {
                         return (int64_t)x.njobs * code_len(x.lgL) > (int64_t)y.njobs * code_len(y.lgL);
                     });
    do {
        if ((st = cuda_fail(cudaMemcpy(dd, host_all.data(), host_all.size() * sizeof(JobDesc),
                                       cudaMemcpyHostToDevice), "batch descriptors")))
            break;
        for (int k = 0; k < SBG_BATCH_STREAMS && !st; ++k) {
            st = cuda_fail(cudaStreamCreateWithFlags(&b->aux[k], cudaStreamNonBlocking), "aux");
            if (!st) st = cuda_fail(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming), "ev");
        }
        if (!st) st = cuda_fail(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "ev");
        if (!st) st = persist_build(b);
        if (!st) st = cuda_fail(cudaStreamSynchronize(c->stream), "sync");
    } while (0);
    if (st) {
        sbg_batch_destroy(b);
        return st;
    }
    *out = b;
    return SBG_OK;
}

int sbg_batch_capture(sbg_batch* b) {
    if (!b) return SBG_EINVAL;
    sbg_ctx* c = b->ctx;
    CK(cudaSetDevice(c->device));
    if (b->exec) return SBG_OK;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int st = batch_launch(b, nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    CK(e);
    b->graph = g;
    CK(cudaGraphInstantiate(&b->exec, g, 0));
    return SBG_OK;
}

int sbg_batch_run(sbg_batch* b) {
    if (!b) return SBG_EINVAL;
    sbg_ctx* c = b->ctx;
    CK(cudaSetDevice(c->device));
    c->launches += batch_run_launches(b);
    if (b->exec) {
        CK(cudaGraphLaunch(b->exec, c->stream));
        return SBG_OK;
    }
    return batch_launch(b, c->timer);
}

int sbg_batch_set_engine(sbg_batch* b, int engine, int64_t wave_bytes) {
    if (!b || engine < 0 || engine > 2 || wave_bytes < 0) return SBG_EINVAL;
    CK(cudaSetDevice(b->ctx->device));
    const bool rebuild = wave_bytes > 0 && (size_t)wave_bytes != b->wave_bytes;
    if (engine == b->engine && !rebuild) return SBG_OK;
    CK(cudaStreamSynchronize(b->ctx->stream));
    if (b->exec) cudaGraphExecDestroy(b->exec);    // the next capture records the new engine
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->engine = engine;
    if (rebuild) {
        b->wave_bytes = (size_t)wave_bytes;
        return persist_build(b);
    }
    return SBG_OK;
}

// Times the engines on the batch -- the queue engines at two wave sizes
// (their best waves differ: 64 MB for the persistent CTAs, 16 MB for one CTA
// per item on B200) -- and keeps the fastest.
int sbg_batch_autotune(sbg_batch* b, double* ms) {
    if (!b) return SBG_EINVAL;
    sbg_ctx* c = b->ctx;
    CK(cudaSetDevice(c->device));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    struct Cfg {
        int engine;
        int64_t wave;
    };
    const Cfg cfgs[5] = {{0, (int64_t)64 << 20}, {0, (int64_t)16 << 20}, {1, 0},
                         {2, (int64_t)16 << 20}, {2, (int64_t)64 << 20}};
    double best = 0.0, eng_ms[3] = {0.0, 0.0, 0.0};
    int best_i = 0, st = SBG_OK;
    for (int i = 0; i < 5 && !st; ++i) {
        if ((st = sbg_batch_set_engine(b, cfgs[i].engine, cfgs[i].wave))) break;
        for (int w = 0; w < 2 && !st; ++w) st = batch_launch(b, nullptr);     // warm-up
        if (st) break;
        if ((st = cuda_fail(cudaEventRecord(e0, c->stream), "event"))) break;
        for (int r = 0; r < 3 && !st; ++r) st = batch_launch(b, nullptr);
        if (st) break;
        float t = 0.f;
        if ((st = cuda_fail(cudaEventRecord(e1, c->stream), "event")) ||
            (st = cuda_fail(cudaEventSynchronize(e1), "event")) ||
            (st = cuda_fail(cudaEventElapsedTime(&t, e0, e1), "event")))
            break;
        const double m = t / 3.0;
        const int e = cfgs[i].engine;
        if (eng_ms[e] == 0.0 || m < eng_ms[e]) eng_ms[e] = m;
        if (i == 0 || m < best) {
            best = m;
            best_i = i;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if (ms)
        for (int e = 0; e < 3; ++e) ms[e] = eng_ms[e];
    return sbg_batch_set_engine(b, cfgs[best_i].engine, cfgs[best_i].wave ? cfgs[best_i].wave : 0);
}

int64_t sbg_ctx_launches(sbg_ctx* c) { return c ? c->launches.load() + c->ring.pulls : 0; }

// For every size class k where a 3 * 2^k transform could replace 2^(k+2),
// time one full product (an = bn = 3 * 2^(k-1), the largest of the class)
// at both lengths on this context's stream and keep the faster.
int sbg_ctx_autotune(sbg_ctx* c, double* times) {
    if (!c) return SBG_EINVAL;
    CK(cudaSetDevice(c->device));
    const int kmax = SBG_MAX_LG - 2;
    const int64_t nmax = (int64_t)3 << (kmax - 1);
    uint64_t* buf = nullptr;
    CK(cudaMalloc(&buf, (size_t)4 * nmax * 8));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = cuda_fail(cudaEventCreate(&e0), "event");
    if (!st) st = cuda_fail(cudaEventCreate(&e1), "event");
    if (!st) st = cuda_fail(cudaMemsetAsync(buf, 0x5a, (size_t)2 * nmax * 8, c->stream), "fill");
    uint32_t mask = 0;
    for (int k = SBG_THREE_MIN_LG; k <= kmax && !st; ++k) {
        const int64_t n = (int64_t)3 << (k - 1);            // 2n - 1 = 3 * 2^k - 1 coefficients
        float best[2] = {0.f, 0.f};
        for (int v = 0; v < 2 && !st; ++v) {
            const int code = v ? SBG_CODE3 + k : k + 2;
            auto one = [&]() {
                return run_conv(c, buf + 2 * nmax, buf, n, buf + nmax, n, 0, code, 0, 2 * n - 2, 0, 2 * n);
            };
            st = one();                                      // builds plan and workspace
            float ms_min = 1e30f;
            for (int rep = 0; rep < 3 && !st; ++rep) {
                if ((st = cuda_fail(cudaEventRecord(e0, c->stream), "rec"))) break;
                if ((st = one())) break;
                if ((st = cuda_fail(cudaEventRecord(e1, c->stream), "rec"))) break;
                if ((st = cuda_fail(cudaEventSynchronize(e1), "sync"))) break;
                float ms = 0.f;
                if ((st = cuda_fail(cudaEventElapsedTime(&ms, e0, e1), "elapsed"))) break;
                ms_min = std::min(ms_min, ms);
            }
            best[v] = ms_min;
        }
        if (st) break;
        if (times) {
            times[2 * (k - SBG_THREE_MIN_LG)] = best[0];
            times[2 * (k - SBG_THREE_MIN_LG) + 1] = best[1];
        }
        if (best[1] < best[0]) mask |= 1u << k;
    }
    if (!st) st = sbg_ctx_sync(c);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    if (!st) c->len3_mask = mask;
    return st;
}

int sbg_ctx_set_len3_mask(sbg_ctx* c, uint32_t mask) {
    if (!c) return SBG_EINVAL;
    c->len3_mask = mask;
    return SBG_OK;
}

uint32_t sbg_ctx_get_len3_mask(sbg_ctx* c) { return c ? c->len3_mask : 0u; }

int sbg_mul_batch(sbg_ctx* c, const sbg_job* jobs, int64_t count) {
    if (!c || (count > 0 && !jobs) || count < 0) return SBG_EINVAL;
    CK(cudaSetDevice(c->device));
    int st = enqueue_products(c, jobs, count);
    if (st) return st;
    return sbg_ctx_sync(c);
}

int sbg_mulmid(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp,
               int64_t bn) {
    if (!c || !rp || !ap || !bp || bn <= 0 || an < bn) return SBG_EINVAL;
    if (an > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
    CK(cudaSetDevice(c->device));
    // the wanted coefficients [bn-1, an-1] are untouched by wrap-around once L >= an
    int lgL = conv_lg(an, c->len3_mask);
    return run_conv(c, rp, ap, an, bp, bn, 0, lgL, bn - 1, an - 1, bn - 1, an - bn + 3);
}

// ---- reference-signature drop-ins -----------------------------------------

static std::mutex g_ctx_mu;
static sbg_ctx* g_ctx[64];

static sbg_ctx* default_ctx() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> g(g_ctx_mu);
    if (!g_ctx[dev]) {
        sbg_ctx* c = nullptr;
        if (sbg_ctx_create(dev, &c) != SBG_OK) return nullptr;
        g_ctx[dev] = c;
    }
    return g_ctx[dev];
}

extern "C" sbg_ctx* sbg_default_ctx_internal(void) { return default_ctx(); }

static bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static int ensure_stage(sbg_ctx* c, size_t limbs) {
    if (limbs > c->stage_cap) {
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(c->d_stage);
        c->d_stage = nullptr;
        c->stage_cap = 0;
        CK(cudaMalloc(&c->d_stage, limbs * sizeof(uint64_t)));
        c->stage_cap = limbs;
    }
    return SBG_OK;
}

#define DROPIN_SPLIT_MIN ((int64_t)1 << 20)   // product limbs from which the uploads overlap

// host-or-device mul/sqr through the default context; synchronous
static int dropin(uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp, int64_t bn,
                  int sq) {
    if (!rp || !ap || an <= 0 || (!sq && (!bp || bn <= 0))) return 0;
    if (an + (sq ? an : bn) - 1 > ((int64_t)1 << SBG_MAX_LG)) return 0;    // beyond the band
    sbg_ctx* c = default_ctx();
    if (!c) return 0;
    std::lock_guard<std::mutex> g(g_ctx_mu);
    bool dev = is_device_ptr(rp) && is_device_ptr(ap) && (sq || is_device_ptr(bp));
    int st;
    if (dev) {
        st = sq ? sbg_sqr(c, rp, ap, an) : sbg_mul(c, rp, ap, an, bp, bn);
    } else {
        int64_t nb = sq ? 0 : bn;
        size_t tot = (size_t)an + (size_t)nb + (size_t)(an + (sq ? an : bn));
        if (ensure_stage(c, tot) != SBG_OK) return 0;
        uint64_t* da = c->d_stage;
        uint64_t* db = da + an;
        uint64_t* dr = db + nb;
        if (!sq && an + bn >= DROPIN_SPLIT_MIN) {
            // the operands upload one after the other on their own stream;
            // the first one's forward transform runs while the second uploads
            // (2^24 x 2^24 limbs: 2,510 -> 2,617 Mlimb/s end to end; below
            // 2^20 limbs the extra stream hand-offs cost more than it saves)
            if (!c->s_stage &&
                (cudaStreamCreateWithFlags(&c->s_stage, cudaStreamNonBlocking) != cudaSuccess ||
                 cudaEventCreateWithFlags(&c->stage_a, cudaEventDisableTiming) != cudaSuccess ||
                 cudaEventCreateWithFlags(&c->stage_b, cudaEventDisableTiming) != cudaSuccess ||
                 cudaEventCreateWithFlags(&c->stage_go, cudaEventDisableTiming) != cudaSuccess))
                return 0;
            if (cudaEventRecord(c->stage_go, c->stream) != cudaSuccess ||
                cudaStreamWaitEvent(c->s_stage, c->stage_go, 0) != cudaSuccess ||
                cudaMemcpyAsync(da, ap, an * 8, cudaMemcpyDefault, c->s_stage) != cudaSuccess ||
                cudaEventRecord(c->stage_a, c->s_stage) != cudaSuccess ||
                cudaMemcpyAsync(db, bp, bn * 8, cudaMemcpyDefault, c->s_stage) != cudaSuccess ||
                cudaEventRecord(c->stage_b, c->s_stage) != cudaSuccess ||
                cudaStreamWaitEvent(c->stream, c->stage_a, 0) != cudaSuccess)
                return 0;
            const int lgL = conv_lg(an + bn - 1, c->len3_mask);
            st = run_conv(c, dr, da, an, db, bn, 0, lgL, 0, an + bn - 2, 0, an + bn, c->stage_b);
        } else {
            if (cudaMemcpyAsync(da, ap, an * 8, cudaMemcpyDefault, c->stream) != cudaSuccess) return 0;
            if (!sq && cudaMemcpyAsync(db, bp, bn * 8, cudaMemcpyDefault, c->stream) != cudaSuccess)
                return 0;
            st = sq ? sbg_sqr(c, dr, da, an) : sbg_mul(c, dr, da, an, db, bn);
        }
        if (st == SBG_OK) {
            size_t outl = (size_t)an + (size_t)(sq ? an : bn);
            if (cudaMemcpyAsync(rp, dr, outl * 8, cudaMemcpyDefault, c->stream) != cudaSuccess)
                return 0;
        }
    }
    if (st != SBG_OK) return 0;
    return sbg_ctx_sync(c) == SBG_OK ? 1 : 0;
}

int sbg_nt_mul(uint64_t* rp, const uint64_t* ap, ptrdiff_t an, const uint64_t* bp, ptrdiff_t bn) {
    return dropin(rp, ap, (int64_t)an, bp, (int64_t)bn, 0);
}

int sbg_nt_sqr(uint64_t* rp, const uint64_t* ap, ptrdiff_t an) {
    return dropin(rp, ap, (int64_t)an, nullptr, 0, 1);
}

}  // extern "C"

// ---- test hooks ---------------------------------------------------------------
extern "C" int sbg_debug_inject(uint32_t mask) { return cuda_fail(set_inject(mask), "inject"); }

extern "C" void sbg_debug_fail_allocs(int n) { g_fail_allocs.store(n < 0 ? 0 : n); }
