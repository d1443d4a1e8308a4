// sbg_serve.cu -- the serving loop: continuous batching of mul / sqr /
// reciprocal requests with admission by HBM footprint.
//
// Requests arrive through sbg_server_submit / sbg_server_submit_many (any
// host thread) and wait in FIFOs.  A scheduler thread owns S "slots" (CUDA
// streams).  Whenever a slot is free it takes multiply requests from the head
// of a FIFO while their footprint -- transform workspace, carry flags, job
// descriptor and the result buffer -- fits in the server's HBM arena (first-
// fit allocator over one device allocation) and the batch's transform points
// stay under a cap, groups them by transform length and launches the batch
// engine's stages on the slot's stream.  Short requests (transforms up to
// 2^17 points) have their own FIFO, served first by slot 0, whose stream has
// the highest priority, so they do not queue behind long batches.  Requests
// that arrive while other batches run join the next batch of a free slot, so
// batches from different arrivals overlap on the device; finished batches are
// retired as soon as their completion event fires, which frees their
// workspace for the next admissions.  Reciprocal requests are batched the same
// way by worker threads (recip_workers, default 2) running the Newton
// reciprocal (all divisors of a batch in lockstep), each on its own context
// and low-priority stream.  A request is complete when its result is in
// device memory; its latency is measured from submission to the moment the
// server observes the completion.  Results stay in the arena until the client
// releases them.  There is no counterpart in the reference, which has no
// serving layer; each result is the one sbg_mul / sbg_sqr / sbg_recip
// compute for the same request alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/simd_bigint_b200.h"
#include "sbg_internal.h"

namespace sbg {

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// first-fit allocator over [base, base + size) in 256-byte units, coalescing
// on free; offsets are absolute within the server's device allocation
class Arena {
   public:
    void init(size_t base, size_t size) {
        free_.clear();
        size_ = size & ~(size_t)255;
        free_[base] = size_;
        used_ = 0;
    }
    bool alloc(size_t bytes, size_t* off) {
        bytes = (bytes + 255) & ~(size_t)255;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                size_t rest = it->second - bytes;
                size_t noff = it->first + bytes;
                free_.erase(it);
                if (rest) free_[noff] = rest;
                used_ += bytes;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = (bytes + 255) & ~(size_t)255;
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }

   private:
    std::map<size_t, size_t> free_;
    size_t size_ = 0, used_ = 0;
};

struct SReq {
    uint64_t ticket = 0;
    sbg_request r{};
    double t_arrive = 0.0, t_launch = 0.0;
    // shape
    int lgL = 0, sq = 0;
    int64_t cmin = 0, cmax = 0, off = 0, nout = 0;
    // arena blocks
    size_t ws_off = 0, ws_bytes = 0;     // workspace (+ flags) or Newton scratch charge
    size_t out_off = 0, out_bytes = 0;   // result
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<SReq> reqs;
    size_t meta_off = 0, meta_bytes = 0;
    JobDesc* staging = nullptr;          // pinned host copy of the descriptors (max_batch)
    uint32_t* herr = nullptr;            // pinned copy of the batch's device error word
};

// device error bits (bit 0 look-back timeout, bit 1 carry spill) -> status
static int err_status(uint32_t h) {
    if (!h) return SBG_OK;
    if (h & 1u) return SBG_ETIMEOUT;
    if (h & 2u) return SBG_ESPILL;
    return SBG_ECUDA;
}

}  // namespace sbg

using namespace sbg;

struct sbg_server {
    sbg_ctx* ctx = nullptr;              // multiplies
    std::vector<sbg_ctx*> rctx;          // reciprocal workers (own stream and workspace each)
    std::vector<cudaStream_t> rstreams;  // their low-priority streams
    int prio_high = 0, prio_low = 0;
    sbg_server_config cfg{};
    uint8_t* arena_base = nullptr;
    // two pools in one allocation: transient blocks (workspaces, descriptors,
    // reciprocal scratch charges; freed when their batch ends) and results
    // (held until the client releases them), so that results scattered over
    // time never fragment the space the next batches need
    Arena arena;
    Arena res;
    std::mutex mu;                       // guards queues, arena, completions
    std::condition_variable cv_work, cv_done;
    // multiply FIFOs by size: transforms up to 2^SMALL_LG points go to
    // pending_small, served first by slot 0 (and by the others when no large
    // request waits), so short requests do not queue behind long batches
    std::deque<SReq> pending_small, pending_mul, pending_recip;
    std::vector<Slot> slots;
    std::deque<sbg_completion> done;
    std::unordered_map<uint64_t, std::pair<size_t, size_t>> results;   // ticket -> out block
    std::atomic<bool> stop{false};
    std::thread sched;
    std::vector<std::thread> recip;
    uint64_t next_ticket = 1;
    int64_t n_done = 0, n_batches = 0;
    int64_t mul_launches = 0;            // kernels of multiply batches
};

#define SMALL_LG 17

static size_t flag_words_of(const SReq& q) { return (size_t)(crt_blocks(q.nout) + 1 + 3) / 4 * 4; }
static size_t mul_ws_bytes(const SReq& q) { return ws_words(q.lgL, q.sq) * 4; }

static void complete(sbg_server* s, const SReq& q, int status, double t) {
    sbg_completion c{};
    c.ticket = q.ticket;
    c.status = status;
    c.rp = status == SBG_OK ? (uint64_t*)(s->arena_base + q.out_off) : nullptr;
    c.rn = q.nout;
    c.latency_s = t - q.t_arrive;
    c.queue_s = (q.t_launch > 0.0 ? q.t_launch : t) - q.t_arrive;
    if (status == SBG_OK)
        s->results[q.ticket] = {q.out_off, q.out_bytes};
    else
        s->res.release(q.out_off, q.out_bytes);
    s->done.push_back(c);
    s->n_done++;
}

// one batch of multiplies on a free slot: requests and arena blocks are
// taken with s->mu held (lk), the CUDA calls run with it released so that
// submissions and polls do not wait behind them
static int launch_slot(sbg_server* s, Slot& sl, std::deque<SReq>& fifo,
                       std::unique_lock<std::mutex>& lk) {
    sbg_ctx* c = s->ctx;
    std::vector<SReq> take;
    const size_t batch_cap = s->arena.size() / (size_t)std::max(1, s->cfg.slots);
    const int64_t point_cap = (int64_t)1 << s->cfg.batch_lg_points;
    size_t batch_bytes = 0;
    int64_t batch_points = 0;
    while (!fifo.empty() && (int)take.size() < s->cfg.max_batch) {
        SReq& q = fifo.front();
        const size_t need = mul_ws_bytes(q) + q.out_bytes;
        if (!take.empty() && batch_bytes + need > batch_cap) break;   // leave room for other slots
        // bounded work per batch, so that slots turn over and late arrivals start soon
        if (!take.empty() && batch_points + code_len(q.lgL) > point_cap) break;
        size_t wo, oo;
        if (!s->arena.alloc(mul_ws_bytes(q), &wo)) break;             // FIFO: wait for memory
        if (!s->res.alloc(q.out_bytes, &oo)) {
            s->arena.release(wo, mul_ws_bytes(q));
            break;
        }
        q.ws_off = wo;
        q.ws_bytes = mul_ws_bytes(q);
        q.out_off = oo;
        take.push_back(q);
        batch_bytes += need;
        batch_points += code_len(q.lgL);
        fifo.pop_front();
    }
    if (take.empty()) return 0;
    const double t_launch = now_s();
    for (auto& q : take) q.t_launch = t_launch;
    // descriptors grouped by length; the batch's carry flags follow them
    std::stable_sort(take.begin(), take.end(), [](const SReq& a, const SReq& b) { return a.lgL < b.lgL; });
    size_t nflags = 0;
    for (auto& q : take) nflags += flag_words_of(q);
    nflags += 4;                                     // the batch's error word (last)
    const size_t meta = take.size() * sizeof(JobDesc) + 256 + nflags * 4;
    size_t mo;
    if (!s->arena.alloc(meta, &mo)) {
        for (auto& q : take) {                       // give everything back, retry later
            s->arena.release(q.ws_off, q.ws_bytes);
            s->res.release(q.out_off, q.out_bytes);
        }
        for (auto it = take.rbegin(); it != take.rend(); ++it) fifo.push_front(*it);
        return 0;
    }
    // a failed enqueue fails the whole batch: wait for what was enqueued, free its memory
    auto fail_batch = [&]() {
        cudaStreamSynchronize(sl.st);
        lk.lock();
        const double t = now_s();
        for (auto& q : take) {
            s->arena.release(q.ws_off, q.ws_bytes);
            complete(s, q, SBG_ECUDA, t);
        }
        s->arena.release(mo, meta);
        return -1;
    };
    lk.unlock();
    uint32_t* flags = (uint32_t*)(s->arena_base + mo + ((take.size() * sizeof(JobDesc) + 255) & ~(size_t)255));
    uint32_t* derr = flags + nflags - 4;
    uint32_t* fcur = flags;
    for (size_t i = 0; i < take.size(); ++i) {
        const SReq& q = take[i];
        JobDesc d{};
        d.a = q.r.ap;
        d.b = q.sq ? q.r.ap : q.r.bp;
        d.out = (uint64_t*)(s->arena_base + q.out_off);
        d.an = q.r.an;
        d.bn = q.sq ? q.r.an : q.r.bn;
        d.cmin = q.cmin;
        d.cmax = q.cmax;
        d.off = q.off;
        d.nout = q.nout;
        d.ws = (uint32_t*)(s->arena_base + q.ws_off);
        d.flags = fcur;
        fcur += flag_words_of(q);
        d.sq = q.sq;
        sl.staging[i] = d;
    }
    JobDesc* dd = (JobDesc*)(s->arena_base + mo);
    if (cudaMemcpyAsync(dd, sl.staging, take.size() * sizeof(JobDesc), cudaMemcpyHostToDevice,
                        sl.st) != cudaSuccess ||
        cudaMemsetAsync(flags, 0, nflags * 4, sl.st) != cudaSuccess)
        return fail_batch();
    // one launch sequence per length class (flags already zeroed above)
    int64_t nlaunch = 0;
    size_t i = 0;
    while (i < take.size()) {
        size_t j = i;
        int64_t max_nout = 0;
        while (j < take.size() && take[j].lgL == take[i].lgL) {
            max_nout = std::max(max_nout, take[j].nout);
            ++j;
        }
        if (launch_batch_class(dd + i, (int)(j - i), take[i].lgL, &c->plans[take[i].lgL], c->tw_f,
                               c->tw_i, max_nout, sl.staging[i].flags, 0, derr, sl.st) !=
            cudaSuccess)
            return fail_batch();
        nlaunch += class_launches(take[i].lgL);
        i = j;
    }
    if (cudaMemcpyAsync(sl.herr, derr, 4, cudaMemcpyDeviceToHost, sl.st) != cudaSuccess ||
        cudaEventRecord(sl.done, sl.st) != cudaSuccess)
        return fail_batch();
    lk.lock();
    s->mul_launches += nlaunch;
    sl.reqs = std::move(take);
    sl.meta_off = mo;
    sl.meta_bytes = meta;
    sl.busy = true;
    s->n_batches++;
    return 1;
}

static void sched_loop(sbg_server* s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        bool progress = false;
        for (auto& sl : s->slots) {
            if (!sl.busy) continue;
            cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) continue;
            const double t = now_s();
            const int status = q == cudaSuccess ? err_status(*sl.herr) : SBG_ECUDA;
            for (auto& r : sl.reqs) {
                s->arena.release(r.ws_off, r.ws_bytes);
                complete(s, r, status, t);
            }
            s->arena.release(sl.meta_off, sl.meta_bytes);
            sl.reqs.clear();
            sl.busy = false;
            progress = true;
        }
        if (progress) s->cv_done.notify_all();
        for (size_t k = 0; k < s->slots.size(); ++k) {
            Slot& sl = s->slots[k];
            if (sl.busy) continue;
            const bool small_only = k == 0 && s->slots.size() > 1;
            std::deque<SReq>& fifo =
                (small_only || s->pending_mul.empty()) ? s->pending_small : s->pending_mul;
            if (fifo.empty()) continue;
            if (launch_slot(s, sl, fifo, lk) != 0) progress = true;
        }
        bool any_busy = false;
        for (auto& sl : s->slots) any_busy |= sl.busy;
        if (!progress) {
            if (any_busy)
                s->cv_work.wait_for(lk, std::chrono::microseconds(20));
            else
                s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
        }
    }
}

static void recip_loop(sbg_server* s, sbg_ctx* rc) {
    cudaSetDevice(rc->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        if (s->pending_recip.empty()) {
            s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            continue;
        }
        std::vector<SReq> take;
        const int64_t point_cap = (int64_t)1 << s->cfg.batch_lg_points;
        int64_t points = 0;
        while (!s->pending_recip.empty() && (int)take.size() < s->cfg.max_batch) {
            SReq& q = s->pending_recip.front();
            // a Newton reciprocal of n limbs costs about a product of 4n points
            if (!take.empty() && points + 4 * q.r.an > point_cap) break;
            size_t wo, oo;
            if (!s->arena.alloc(q.ws_bytes, &wo)) break;
            if (!s->res.alloc(q.out_bytes, &oo)) {
                s->arena.release(wo, q.ws_bytes);
                break;
            }
            q.ws_off = wo;
            q.out_off = oo;
            take.push_back(q);
            points += 4 * q.r.an;
            s->pending_recip.pop_front();
        }
        if (take.empty()) {
            s->cv_work.wait_for(lk, std::chrono::milliseconds(1));
            continue;
        }
        const double t_launch = now_s();
        for (auto& q : take) q.t_launch = t_launch;
        std::vector<const uint64_t*> D;
        std::vector<uint64_t*> V;
        std::vector<int64_t> n;
        for (auto& q : take) {
            D.push_back(q.r.ap);
            V.push_back((uint64_t*)(s->arena_base + q.out_off));
            n.push_back(q.r.an);
        }
        lk.unlock();
        int st = recip_batch(rc, D.data(), V.data(), n.data(), (int)take.size());
        lk.lock();
        const double t = now_s();
        for (auto& q : take) {
            s->arena.release(q.ws_off, q.ws_bytes);
            complete(s, q, st, t);
        }
        s->n_batches++;
        s->cv_done.notify_all();
    }
}

extern "C" int sbg_server_create(sbg_ctx* ctx, const sbg_server_config* cfg, sbg_server** out) {
    if (!ctx || !out) return SBG_EINVAL;
    *out = nullptr;
    sbg_server* s = new sbg_server();
    s->ctx = ctx;
    s->cfg.arena_bytes = cfg && cfg->arena_bytes ? cfg->arena_bytes : ((size_t)8 << 30);
    s->cfg.slots = cfg && cfg->slots > 0 ? cfg->slots : 4;
    s->cfg.max_batch = cfg && cfg->max_batch > 0 ? cfg->max_batch : 512;
    s->cfg.recip_workers = cfg && cfg->recip_workers > 0 ? cfg->recip_workers : 2;
    s->cfg.batch_lg_points =
        cfg && cfg->batch_lg_points > 0 ? std::min(cfg->batch_lg_points, 40) : 26;
    int st = SBG_OK;
    do {
        if ((st = cuda_fail(cudaSetDevice(ctx->device), "device"))) break;
        for (int l = 4; l <= 22 && !st; ++l) st = ensure_plan(ctx, l);   // tables to 2^22 points
        for (int k = SBG_THREE_MIN_LG; k <= 20 && !st; ++k) st = ensure_plan(ctx, SBG_CODE3 + k);
        if (st) break;
        // stream priorities: multiply slots highest, reciprocal workers lowest,
        // so short multiplies are not queued behind long Newton batches
        int prio_low = 0, prio_high = 0;
        if ((st = cuda_fail(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high), "priorities"))) break;
        s->prio_high = prio_high;
        s->prio_low = prio_low;
        for (int w = 0; w < s->cfg.recip_workers && !st; ++w) {
            sbg_ctx* rc = nullptr;
            if ((st = sbg_ctx_create(ctx->device, &rc))) break;
            s->rctx.push_back(rc);
            rc->stream_priority = prio_low;
            rc->len3_mask = ctx->len3_mask;
            cudaStream_t rs = nullptr;
            if ((st = cuda_fail(cudaStreamCreateWithPriority(&rs, cudaStreamNonBlocking, prio_low), "rstream")))
                break;
            s->rstreams.push_back(rs);
            sbg_ctx_set_stream(rc, rs);
        }
        if (st) break;
        if ((st = cuda_fail(cudaMalloc(&s->arena_base, s->cfg.arena_bytes), "arena"))) break;
        const size_t transient = (s->cfg.arena_bytes / 8 * 5) & ~(size_t)255;
        s->arena.init(0, transient);
        s->res.init(transient, s->cfg.arena_bytes - transient);
        s->slots.resize((size_t)s->cfg.slots);
        for (auto& sl : s->slots) {
            // slot 0 (short requests) above the other slots, which are above
            // the reciprocal workers
            const int pr = &sl == &s->slots[0] ? s->prio_high : std::min(s->prio_high + 1, s->prio_low);
            if ((st = cuda_fail(cudaStreamCreateWithPriority(&sl.st, cudaStreamNonBlocking, pr), "slot")))
                break;
            if ((st = cuda_fail(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "ev")))
                break;
            if ((st = cuda_fail(cudaHostAlloc(&sl.herr, 4, 0), "herr"))) break;
            if ((st = cuda_fail(cudaHostAlloc(&sl.staging, (size_t)s->cfg.max_batch * sizeof(JobDesc), 0),
                                "staging")))
                break;
            *sl.herr = 0;
        }
    } while (0);
    if (st) {
        sbg_server_destroy(s);
        return st;
    }
    s->sched = std::thread(sched_loop, s);
    for (sbg_ctx* rc : s->rctx) s->recip.emplace_back(recip_loop, s, rc);
    *out = s;
    return SBG_OK;
}

extern "C" void sbg_server_destroy(sbg_server* s) {
    if (!s) return;
    s->stop = true;
    s->cv_work.notify_all();
    if (s->sched.joinable()) s->sched.join();
    for (auto& t : s->recip)
        if (t.joinable()) t.join();
    if (s->ctx) cudaSetDevice(s->ctx->device);
    for (auto& sl : s->slots) {
        if (sl.st) cudaStreamSynchronize(sl.st);
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.done) cudaEventDestroy(sl.done);
        cudaFreeHost(sl.staging);
        cudaFreeHost(sl.herr);
    }
    cudaFree(s->arena_base);
    for (sbg_ctx* rc : s->rctx) sbg_ctx_destroy(rc);
    for (cudaStream_t rs : s->rstreams) cudaStreamDestroy(rs);
    delete s;
}

// validation and footprint of one request (no lock needed)
static int prepare(sbg_server* s, const sbg_request* req, SReq& q) {
    if (!req || !req->ap || req->an <= 0) return SBG_EINVAL;
    q = SReq{};
    q.r = *req;
    if (req->kind == SBG_REQ_RECIP) {
        q.nout = req->an;
        q.ws_bytes = div_scratch_limbs(req->an) * 8;
        q.out_bytes = (size_t)req->an * 8;
        if (2 * req->an + 2 > ((int64_t)1 << 25)) return SBG_EBAND;
    } else {
        if (req->kind != SBG_REQ_MUL && req->kind != SBG_REQ_SQR) return SBG_EINVAL;
        if (req->kind == SBG_REQ_MUL && (!req->bp || req->bn <= 0)) return SBG_EINVAL;
        int64_t need = req->kind == SBG_REQ_SQR ? 2 * req->an - 1 : req->an + req->bn - 1;
        if (need > ((int64_t)1 << SBG_MAX_LG)) return SBG_EBAND;
        q.lgL = need + 1 <= SBG_SCHOOL_MAX ? SBG_CODE_SCHOOL : conv_lg(need, s->ctx->len3_mask);
        q.sq = req->kind == SBG_REQ_SQR;
        q.cmin = 0;
        q.cmax = need - 1;
        q.off = 0;
        q.nout = need + 1;
        q.out_bytes = (size_t)q.nout * 8;
        q.ws_bytes = mul_ws_bytes(q);
    }
    if (q.ws_bytes + 4096 > s->arena.size() || q.out_bytes > s->res.size())
        return SBG_EADMIT;                           // can never fit
    return SBG_OK;
}

// queue prepared requests (s->mu held); stops at the first failure
static int enqueue(sbg_server* s, SReq* q, int64_t n, uint64_t* tickets, int64_t* accepted) {
    const double t = now_s();
    for (int64_t i = 0; i < n; ++i) {
        if (q[i].lgL > 0 && s->ctx->plans[q[i].lgL].lgL != q[i].lgL) {
            int st = ensure_plan(s->ctx, q[i].lgL);
            if (st) return st;
        }
        q[i].t_arrive = t;
        q[i].ticket = s->next_ticket++;
        if (q[i].r.kind == SBG_REQ_RECIP)
            s->pending_recip.push_back(q[i]);
        else
            (code_len(q[i].lgL) <= ((int64_t)1 << SMALL_LG) ? s->pending_small : s->pending_mul)
                .push_back(q[i]);
        if (tickets) tickets[i] = q[i].ticket;
        if (accepted) *accepted = i + 1;
    }
    return SBG_OK;
}

extern "C" int sbg_server_submit(sbg_server* s, const sbg_request* req, uint64_t* ticket) {
    if (!s) return SBG_EINVAL;
    SReq q;
    int st = prepare(s, req, q);
    if (st) return st;
    {
        std::lock_guard<std::mutex> g(s->mu);
        st = enqueue(s, &q, 1, ticket, nullptr);
    }
    s->cv_work.notify_all();
    return st;
}

extern "C" int sbg_server_submit_many(sbg_server* s, const sbg_request* reqs, int64_t count,
                                      uint64_t* tickets, int64_t* accepted) {
    if (!s || (count > 0 && !reqs) || count < 0) return SBG_EINVAL;
    if (accepted) *accepted = 0;
    std::vector<SReq> q((size_t)count);
    int st = SBG_OK;
    int64_t ok = 0;
    for (; ok < count; ++ok)
        if ((st = prepare(s, &reqs[ok], q[ok]))) break;
    if (ok > 0) {
        std::lock_guard<std::mutex> g(s->mu);
        int st2 = enqueue(s, q.data(), ok, tickets, accepted);
        if (st2) st = st2;
    }
    s->cv_work.notify_all();
    return st;
}

extern "C" int sbg_server_poll(sbg_server* s, sbg_completion* out, int max, int* n, int wait_ms) {
    if (!s || !out || !n || max <= 0) return SBG_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    int k = 0;
    while (k < max && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *n = k;
    return SBG_OK;
}

extern "C" int sbg_server_release(sbg_server* s, uint64_t ticket) {
    if (!s) return SBG_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->results.find(ticket);
    if (it == s->results.end()) return SBG_EINVAL;
    s->res.release(it->second.first, it->second.second);
    s->results.erase(it);
    s->cv_work.notify_all();
    return SBG_OK;
}

extern "C" int sbg_server_cancel(sbg_server* s, uint64_t ticket) {
    if (!s) return SBG_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    for (std::deque<SReq>* fifo : {&s->pending_small, &s->pending_mul, &s->pending_recip}) {
        for (auto it = fifo->begin(); it != fifo->end(); ++it) {
            if (it->ticket != ticket) continue;
            // still queued: it holds no arena block yet, so it completes
            // without touching the allocators
            sbg_completion c{};
            c.ticket = ticket;
            c.status = SBG_ECANCELED;
            c.rp = nullptr;
            c.rn = 0;
            const double t = now_s();
            c.latency_s = t - it->t_arrive;
            c.queue_s = c.latency_s;
            fifo->erase(it);
            s->done.push_back(c);
            s->n_done++;
            s->cv_done.notify_all();
            return SBG_OK;
        }
    }
    return SBG_EINVAL;          // unknown, already launched, or already complete
}

extern "C" int64_t sbg_server_launches(sbg_server* s) {
    if (!s) return 0;
    std::lock_guard<std::mutex> g(s->mu);
    int64_t n = s->mul_launches;
    for (sbg_ctx* rc : s->rctx) n += rc->launches.load();
    return n;
}

extern "C" int sbg_server_stats(sbg_server* s, int64_t* pending, int64_t* completed,
                                int64_t* batches, size_t* arena_used) {
    if (!s) return SBG_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    if (pending)
        *pending = (int64_t)(s->pending_small.size() + s->pending_mul.size() + s->pending_recip.size());
    if (completed) *completed = s->n_done;
    if (batches) *batches = s->n_batches;
    if (arena_used) *arena_used = s->arena.used() + s->res.used();
    return SBG_OK;
}
