// sbg_noalloc.cu -- a multiply entry point that allocates no device memory.
//
// Some callers cannot allocate GPU memory when they multiply: applications
// that reserve all device memory up front and hand the rest of the program a
// fixed budget, plug-ins living inside a host that owns the device allocator,
// and latency-critical loops that cannot afford cudaMalloc's implicit device
// synchronisation.  sbg_mul_noalloc serves them for products of at most
// SBG_NOALLOC_MAX_LIMBS limbs (an + bn), the single-CTA transform band.
//
// Its scratch -- the five residue arrays of one product plus the carry-scan
// flags and an error word -- is the file-scope array g_scratch below, and its
// twiddle tables are the file-scope arrays g_tw_f / g_tw_i.  Every GPU that
// loads this library holds them (about 740 KB) until the process exits.  In
// host code those names are host-side stand-ins, not device addresses, so the
// first call on each device looks up their device addresses with
// cudaGetSymbolAddress (that device current), uploads the prime constants and
// fills the tables; that first call therefore synchronises its stream and
// should come before any stream capture.  Later calls only queue kernels.
//
// All calls share the one scratch array, which keeps the previous call's
// contents: the carry flags are cleared on every call (the residue arrays are
// fully rewritten before they are read).  Calls that overlap on the GPU --
// on different streams, or from several host threads -- race on the scratch;
// callers must order them (one stream, or events).
//
// Errors found on the device (the carry look-back's bounded wait expiring,
// the spill check) set bits in an error word inside the scratch.  They
// accumulate over calls until sbg_noalloc_status reads them: it waits for the
// caller's stream, returns the status the bits map to and zeroes the word, so
// a later call's clean run cannot hide an earlier queued call's error.
//
// The set-up state (symbol addresses, tables, constants) is kept per device
// for the life of the process; a cudaDeviceReset after the first call on a
// device is not supported (the addresses and tables would be stale).  The
// first calls on different devices run their set-up concurrently (one lock
// per device).
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/simd_bigint_b200.h"
#include "sbg_internal.h"
#include "sbg_ntt.cuh"

namespace sbg {

#define SBG_NOALLOC_LG 12                               // transform length 2^12
#define SBG_NOALLOC_RES_WORDS (SBG_NP << SBG_NOALLOC_LG)
#define SBG_NOALLOC_FLAG_WORDS 64
#define SBG_NOALLOC_SCRATCH_WORDS (SBG_NOALLOC_RES_WORDS + SBG_NOALLOC_FLAG_WORDS + 64)

static __device__ __align__(256) uint32_t g_scratch[SBG_NOALLOC_SCRATCH_WORDS];
static __device__ __align__(256) uint2 g_tw_f[SBG_NP * SBG_TW_N];
static __device__ __align__(256) uint2 g_tw_i[SBG_NP * SBG_TW_N];

struct RootSet {
    uint32_t r[SBG_NP];
    uint32_t p[SBG_NP];
};

__device__ __forceinline__ uint32_t na_pow(uint32_t b, uint32_t e, uint32_t p) {
    uint64_t r = 1, x = b;
    while (e) {
        if (e & 1) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

// per-resolution twiddle table (same layout as the context tables): entry
// S/2 - 1 + j holds (w_S^j, shoup) for S = 2 .. 2^13
__global__ void k_noalloc_tables(uint2* out, RootSet roots) {
    const int q = blockIdx.y;
    const uint32_t p = roots.p[q];
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < SBG_TW_N - 1;
         idx += gridDim.x * blockDim.x) {
        int lgS = 32 - __clz(idx + 1);
        int j = idx - ((1 << (lgS - 1)) - 1);
        uint32_t e = (uint32_t)j << (SBG_TW_LG - lgS);
        uint32_t w = na_pow(roots.r[q], e, p);
        out[(size_t)q * SBG_TW_N + idx] = make_uint2(w, shoup_of(w, p));
    }
}

struct NoallocDev {
    bool ready = false;
    uint32_t* scratch = nullptr;
    uint2* tw_f = nullptr;
    uint2* tw_i = nullptr;
};

#define SBG_NOALLOC_MAX_DEV 64
static std::mutex g_na_mu[SBG_NOALLOC_MAX_DEV];
static NoallocDev g_na[SBG_NOALLOC_MAX_DEV];

static cudaError_t noalloc_setup(int dev, cudaStream_t st, NoallocDev** out) {
    std::lock_guard<std::mutex> g(g_na_mu[dev]);
    NoallocDev* d = &g_na[dev];
    if (!d->ready) {
        cudaError_t e = cudaGetSymbolAddress((void**)&d->scratch, g_scratch);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress((void**)&d->tw_f, g_tw_f);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress((void**)&d->tw_i, g_tw_i);
        if (e != cudaSuccess) return e;
        e = upload_constants(st);
        if (e != cudaSuccess) return e;
        RootSet rf, ri;
        for (int q = 0; q < SBG_NP; ++q) {
            uint32_t p = kPrimes[q];
            rf.r[q] = host_powmod(kGenerators[q], (p - 1) >> SBG_TW_LG, p);
            ri.r[q] = host_powmod(rf.r[q], p - 2, p);
            rf.p[q] = p;
            ri.p[q] = p;
        }
        dim3 grid(32, SBG_NP);
        k_noalloc_tables<<<grid, 256, 0, st>>>(d->tw_f, rf);
        k_noalloc_tables<<<grid, 256, 0, st>>>(d->tw_i, ri);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        d->ready = true;
    }
    *out = d;
    return cudaSuccess;
}

}  // namespace sbg

using namespace sbg;

extern "C" int64_t sbg_noalloc_max_limbs(void) { return SBG_NOALLOC_MAX_LIMBS; }

extern "C" int sbg_mul_noalloc(uint64_t* rp, const uint64_t* ap, int64_t an, const uint64_t* bp,
                               int64_t bn, void* stream) {
    if (!rp || !ap || !bp || an <= 0 || bn <= 0) return SBG_EINVAL;
    if (an + bn > SBG_NOALLOC_MAX_LIMBS) return SBG_EBAND;   // beyond the static scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SBG_NOALLOC_MAX_DEV) return SBG_ENODEV;
    cudaStream_t st = (cudaStream_t)stream;
    NoallocDev* d = nullptr;
    if (noalloc_setup(dev, st, &d) != cudaSuccess) return SBG_ECUDA;
    int lgL = 4;
    while (((int64_t)1 << lgL) < an + bn - 1) ++lgL;
    LenPlan lp;                                 // single-CTA band: only the scale is used
    lp.lgL = lgL;
    lp.lgN1 = 0;
    lp.lgN2 = lgL;
    lp.L = (int64_t)1 << lgL;
    for (int q = 0; q < SBG_NP; ++q) lp.scale[q] = host_scale(lp.L, q);
    uint32_t* res = d->scratch;
    uint32_t* flags = d->scratch + SBG_NOALLOC_RES_WORDS;
    uint32_t* err = flags + SBG_NOALLOC_FLAG_WORDS;
    if (launch_conv(ap, an, bp, bn, 0, lgL, &lp, d->tw_f, d->tw_i, res, st) != cudaSuccess)
        return SBG_ECUDA;
    if (launch_crt_carry(res, lgL, &lp, 0, an + bn - 2, 0, rp, an + bn, flags, err, st) !=
        cudaSuccess)
        return SBG_ECUDA;
    return SBG_OK;
}

extern "C" int sbg_noalloc_status(void* stream) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SBG_NOALLOC_MAX_DEV) return SBG_ENODEV;
    NoallocDev* d = &g_na[dev];
    {
        std::lock_guard<std::mutex> g(g_na_mu[dev]);
        if (!d->ready) return SBG_OK;           // no call has run on this device
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* err = d->scratch + SBG_NOALLOC_RES_WORDS + SBG_NOALLOC_FLAG_WORDS;
    uint32_t h = 0;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SBG_ECUDA;
    if (cudaMemcpy(&h, err, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return SBG_ECUDA;
    if (!h) return SBG_OK;
    if (cudaMemsetAsync(err, 0, sizeof(uint32_t), st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return SBG_ECUDA;
    if (h & 1u) return SBG_ETIMEOUT;
    if (h & 2u) return SBG_ESPILL;
    return SBG_ECUDA;
}
