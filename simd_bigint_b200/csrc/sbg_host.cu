// sbg_host.cu -- products of HOST operands, stream-ordered and pipelined.
//
// sbg_mul_host / sbg_sqr_host queue: upload of the operands (copy stream),
// the product on the context stream, download of the result (second copy
// stream), and return at once.  Two staging slots alternate between calls,
// so with page-locked host buffers the download of one product, the upload
// of the next and the transforms of a third overlap (PCIe is full duplex).
// The reference multiplies host arrays synchronously (include/ntmul.h:71);
// sbg_nt_mul keeps that contract, these entries are its asynchronous form
// for callers with a stream of products.
#include <cuda_runtime.h>

#include "../../include/simd_bigint_b200.h"
#include "sbg_internal.h"

namespace sbg {

static int host_pipe_init(sbg_ctx* c) {
    if (c->s_in) return SBG_OK;
    if (cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking) != cudaSuccess)
        return SBG_ECUDA;
    for (auto& h : c->hslot) {
        if (cudaEventCreateWithFlags(&h.in_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h.comp_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h.out_done, cudaEventDisableTiming) != cudaSuccess)
            return SBG_ECUDA;
    }
    return SBG_OK;
}

// grow a slot's staging; everything that may still use it is finished first
static int host_slot_reserve(sbg_ctx* c, sbg_ctx::HostSlot& h, size_t limbs) {
    if (limbs <= h.cap) return SBG_OK;
    if (cudaStreamSynchronize(c->s_in) != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->s_out) != cudaSuccess)
        return SBG_ECUDA;
    cudaFree(h.d);
    h.d = nullptr;
    h.cap = 0;
    if (cudaMalloc(&h.d, limbs * 8) != cudaSuccess) return SBG_EALLOC;
    h.cap = limbs;
    return SBG_OK;
}

// Copies in 8 MB pieces: with an upload and a download running at once, the
// two copy engines interleave pieces of this size more evenly on PCIe than
// whole 100 MB transfers (measured on B200, 268 MB each way: 5.54 ms in
// 8 MB pieces against 5.83 ms whole; 4.84 ms for one direction alone).
#define HOST_COPY_PIECE ((size_t)8 << 20)
static cudaError_t copy_pieces(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind,
                               cudaStream_t st) {
    for (size_t o = 0; o < bytes; o += HOST_COPY_PIECE) {
        const size_t len = bytes - o < HOST_COPY_PIECE ? bytes - o : HOST_COPY_PIECE;
        cudaError_t e = cudaMemcpyAsync((char*)dst + o, (const char*)src + o, len, kind, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static int host_product(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp,
                        int64_t bn, int sq) {
    if (!c || !rp || !ap || an <= 0 || (!sq && (!bp || bn <= 0))) return SBG_EINVAL;
    if (cudaSetDevice(c->device) != cudaSuccess) return SBG_ECUDA;
    int st = host_pipe_init(c);
    if (st) return st;
    const int64_t nb = sq ? 0 : bn;
    const int64_t nout = an + (sq ? an : bn);
    auto& h = c->hslot[c->hnext];
    c->hnext ^= 1;
    if ((st = host_slot_reserve(c, h, (size_t)(an + nb + nout)))) return st;
    uint64_t* da = h.d;
    uint64_t* db = da + an;
    uint64_t* dr = db + nb;
    // the slot's operands are free once its previous product has run, its
    // result buffer once that result has been downloaded
    if (cudaStreamWaitEvent(c->s_in, h.comp_done, 0) != cudaSuccess ||
        copy_pieces(da, ap, (size_t)an * 8, cudaMemcpyHostToDevice, c->s_in) != cudaSuccess ||
        (!sq && copy_pieces(db, bp, (size_t)bn * 8, cudaMemcpyHostToDevice, c->s_in) != cudaSuccess) ||
        cudaEventRecord(h.in_done, c->s_in) != cudaSuccess ||
        cudaStreamWaitEvent(c->stream, h.in_done, 0) != cudaSuccess ||
        cudaStreamWaitEvent(c->stream, h.out_done, 0) != cudaSuccess)
        return SBG_ECUDA;
    st = sq ? sbg_sqr(c, dr, da, an) : sbg_mul(c, dr, da, an, db, bn);
    if (st) return st;
    if (cudaEventRecord(h.comp_done, c->stream) != cudaSuccess ||
        cudaStreamWaitEvent(c->s_out, h.comp_done, 0) != cudaSuccess ||
        copy_pieces(rp, dr, (size_t)nout * 8, cudaMemcpyDeviceToHost, c->s_out) != cudaSuccess ||
        cudaEventRecord(h.out_done, c->s_out) != cudaSuccess)
        return SBG_ECUDA;
    return SBG_OK;
}

void host_pipe_release(sbg_ctx* c) {
    if (c->s_in) cudaStreamSynchronize(c->s_in);
    if (c->s_out) cudaStreamSynchronize(c->s_out);
    for (auto& h : c->hslot) {
        cudaFree(h.d);
        if (h.in_done) cudaEventDestroy(h.in_done);
        if (h.comp_done) cudaEventDestroy(h.comp_done);
        if (h.out_done) cudaEventDestroy(h.out_done);
        h = sbg_ctx::HostSlot{};
    }
    if (c->s_in) cudaStreamDestroy(c->s_in);
    if (c->s_out) cudaStreamDestroy(c->s_out);
    c->s_in = c->s_out = nullptr;
}

int host_pipe_sync(sbg_ctx* c) {
    if (c->s_in && cudaStreamSynchronize(c->s_in) != cudaSuccess) return SBG_ECUDA;
    if (c->s_out && cudaStreamSynchronize(c->s_out) != cudaSuccess) return SBG_ECUDA;
    return SBG_OK;
}

}  // namespace sbg

extern "C" int sbg_mul_host(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp,
                            int64_t bn) {
    return sbg::host_product(c, rp, ap, an, bp, bn, 0);
}

extern "C" int sbg_sqr_host(sbg_ctx* c, uint64_t* rp, const uint64_t* ap, int64_t an) {
    return sbg::host_product(c, rp, ap, an, nullptr, 0, 1);
}
