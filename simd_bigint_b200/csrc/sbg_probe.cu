// sbg_probe.cu -- integer-pipe ceiling for the transform kernels.
//
// The NTT kernels are bounded by integer issue, not by HBM: every radix-2
// level costs one Gentleman-Sande butterfly per point pair (bfly_gs in
// sbg_arith.cuh: on the sum an add and a conditional subtract of p; on the
// difference an add of p, a Shoup product -- a high multiply by the
// companion, a low multiply by the twiddle, a multiply-subtract of the
// quotient estimate times p -- and a conditional subtract).  This probe runs that exact
// butterfly on registers only (16 independent chains per thread, no memory
// traffic, 4 CTAs of 256 threads per SM) and reports butterflies per second:
// the compute roofline the benchmark divides the kernels' butterfly rate by.
#include <cuda_runtime.h>
#include <cstdint>

#include "sbg_arith.cuh"

namespace sbg {

__global__ void __launch_bounds__(256) k_probe_bfly(uint32_t* sink, int iters, uint32_t p,
                                                    uint32_t w, uint32_t ws) {
    uint32_t x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = (threadIdx.x * 2654435761u + i * 40503u) % p;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) bfly_gs(x[i], x[i + 8], w, ws, p);
#pragma unroll
        for (int i = 0; i < 16; i += 2) bfly_gs(x[i], x[i + 1], w, ws, p);
    }
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) acc ^= x[i];
    if (acc == 0x12345678u) sink[threadIdx.x] = acc;   // keeps the chains live
}

}  // namespace sbg

extern "C" int sbg_probe_bfly_peak(int device, double* bfly_per_s) {
    using namespace sbg;
    if (!bfly_per_s) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 4;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    uint32_t* sink = nullptr;
    if (cudaMalloc(&sink, 256 * sizeof(uint32_t)) != cudaSuccess) return 3;
    const uint32_t p = kPrimes[4];
    const uint32_t w = 123456789u % p;
    const uint32_t ws = (uint32_t)(((uint64_t)w << 32) / p);
    const int blocks = sms * 4, iters = 4096;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_probe_bfly<<<blocks, 256>>>(sink, 64, p, w, ws);   // warm-up
    cudaEventRecord(a);
    k_probe_bfly<<<blocks, 256>>>(sink, iters, p, w, ws);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess || ms <= 0.f) return 4;
    double bflies = (double)blocks * 256.0 * iters * 16.0;
    *bfly_per_s = bflies / (ms * 1e-3);
    return 0;
}
