// sbg_persist.cuh -- the persistent batch kernel (included by sbg_kernels.cu,
// whose transform bodies it runs).
//
// One launch runs a whole batch of uneven products.  Its CTAs (as many as
// fit on the device at once) take work items from a queue in device memory,
// one at a time, by an atomic increment of the queue head.  An item is one
// stage of one job on one tile -- a column-forward tile, a row, a
// column-inverse tile, a carry-scan block -- or a whole short product: a
// single-CTA product (five transforms of at most 2^12 points and its carry
// blocks) or a group of up to eight schoolbook products, one warp each.  Every job has a progress counter that each finished item of the job
// increments; an item carries the counter value its job's earlier stages
// reach, and the CTA that takes it waits (bounded) until the counter gets
// there.
//
// The host orders the queue so that every item comes after all the items it
// waits for (stages in order, and a job's carry blocks in block order, which
// the carry scan's look-back needs).  A CTA takes an item only while it is
// resident, so every item an item waits for is already held by a running
// CTA: the waits always end.  Each wait is bounded nevertheless; on expiry
// the kernel sets the error word's timeout bit and goes on.
//
// Jobs are grouped into waves of a bounded workspace footprint (L2 blocking)
// and the queue is software-pipelined over the waves: step t holds the
// carry blocks of wave t - 3, the inverse columns of wave t - 2, the rows of
// wave t - 1 and the forward columns of wave t.  A stage's input was written
// one step earlier, so it is mostly still in L2, and the items of a step do
// not wait on each other.  The whole short products, which wait for
// nothing, come last: they fill the CTAs that the last waves' stages leave
// idle.
#pragma once

namespace sbg {

#define PERSIST_WAIT_LIMIT (1 << 25)

// Waits until the job's progress counter reaches `need`.  Bounded, and once
// any wait of the launch has expired (the error word's timeout bit is set)
// the others give up at once, so a fault in the queue's order costs one
// expiry, not one per item.
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void persist_wait(const uint32_t* cnt, uint32_t need, uint32_t* err) {
    const volatile uint32_t* e = err;
    int spins = 0;
    while (ld_acquire(cnt) < need) {
        if (++spins > PERSIST_WAIT_LIMIT || ((spins & 63) == 0 && (*e & 1u))) {
            atomicOr(err, 1u);
            break;
        }
        __nanosleep(64);
    }
}

// A finished item: the CTA's writes (ordered before this by the barrier the
// caller passed) are released to the device with the counter increment; no
// return value is waited for.
__device__ __forceinline__ void persist_signal(uint32_t* cnt) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(cnt) : "memory");
}

// A persistent CTA takes one item per queue-head increment (taking 4 at a
// time made the mixed batch 1.7x slower on B200: a CTA sits on items that
// idle CTAs could run) and, with PERSIST_PREFETCH, takes its next item while
// it runs the current one.
#ifndef PERSIST_PREFETCH
#define PERSIST_PREFETCH 1
#endif

template <int LGN1>
__device__ __forceinline__ void persist_col(const PItem& I, const JobDesc& J, const uint2* __restrict__ twf,
                                            const uint2* __restrict__ twi) {
    constexpr int NTILES = col_ntiles(LGN1);
    if (I.kind == PK_COLF) {
        const int q = (int)(I.idx % SBG_NP);
        const int r = (int)(I.idx / SBG_NP);
        uint32_t* YB = J.ws + ((size_t)SBG_NP << (LGN1 + SBG_ROW_LG));
        col_fwd_body<LGN1>(q, r % NTILES, 0, r / NTILES, J.a, J.an, J.b, J.bn, twf, J.ws, YB);
    } else {
        col_inv_body<LGN1>((int)(I.idx % SBG_NP), (int)(I.idx / SBG_NP), 0, J.ws, twi);
    }
}

// One work item (the CTA's whole block takes part); the item's fields come
// in as warp-uniform values.
__device__ __forceinline__ void persist_item(uint32_t kind, uint32_t job, uint32_t lg, uint32_t idx,
                                             const JobDesc* __restrict__ jobs, const PClass* __restrict__ cls,
                                             const uint2* __restrict__ twf, const uint2* __restrict__ twi,
                                             uint32_t* err, uint32_t* sm) {
    switch (kind) {
        case PK_SCHOOL: {
            const int w = threadIdx.x >> 5;
            if (w < (int)idx) {
                const JobDesc& J = jobs[job + w];
                uint64_t* sa = reinterpret_cast<uint64_t*>(sm) + w * (2 * SBG_SCHOOL_MAX);
                school_warp(J.a, (int)J.an, J.b, (int)J.bn, J.out, sa, sa + SBG_SCHOOL_MAX);
            }
            break;
        }
        case PK_SMALL: {
            const JobDesc& J = jobs[job];
            small_body((int)idx, J.a, J.an, J.b, J.bn, J.sq, (int)lg, twf, twi, cls[lg].sc, J.ws);
            break;
        }
        case PK_SMALLJOB: {
            // a whole single-CTA product: the five primes' transforms, then
            // its carry blocks in order (each block's look-back finds its
            // predecessor's flag already published)
            const JobDesc& J = jobs[job];
            for (int q = 0; q < SBG_NP; ++q) {
                small_body(q, J.a, J.an, J.b, J.bn, J.sq, (int)lg, twf, twi, cls[lg].sc, J.ws);
                __syncthreads();
            }
            __threadfence_block();
            for (uint32_t k = 0; k < idx; ++k) {
                crt_body(k, J.ws, (int64_t)1 << lg, J.cmin, J.cmax, J.off, J.out, J.nout, J.flags, err,
                         *reinterpret_cast<CrtSmem*>(sm));
                __syncthreads();
            }
            break;
        }
        case PK_COLF:
        case PK_COLI: {
            const PItem I{job, (uint16_t)kind, (uint16_t)lg, idx, 0};
            const JobDesc& J = jobs[job];
            switch ((int)lg - SBG_ROW_LG) {
                case 1: persist_col<1>(I, J, twf, twi); break;
                case 2: persist_col<2>(I, J, twf, twi); break;
                case 3: persist_col<3>(I, J, twf, twi); break;
                case 4: persist_col<4>(I, J, twf, twi); break;
                case 5: persist_col<5>(I, J, twf, twi); break;
                case 6: persist_col<6>(I, J, twf, twi); break;
                case 7: persist_col<7>(I, J, twf, twi); break;
                case 8: persist_col<8>(I, J, twf, twi); break;
                default: break;
            }
            break;
        }
        case PK_ROW: {
            // PERSIST_ROWS consecutive rows of one prime (2^lgN1 >= 2 rows)
            const JobDesc& J = jobs[job];
            const int lgN1 = (int)lg - SBG_ROW_LG;
            const PClass& C = cls[lg];
            uint32_t* YB = J.ws + ((size_t)SBG_NP << lg);
            for (int k = 0; k < PERSIST_ROWS; ++k) {
                const int r = (int)idx * PERSIST_ROWS + k;
                const int q = r >> lgN1;
                row_body(q, r & ((1 << lgN1) - 1), J.ws, YB, J.sq, lgN1, -1, C.fsf, C.fsi, C.sc.w[q],
                         C.sc.ws[q], twf, twi, *reinterpret_cast<RowSmem*>(sm));
                __syncthreads();
            }
            break;
        }
        case PK_CRT: {
            // up to PERSIST_CRT consecutive carry blocks, in block order
            const JobDesc& J = jobs[job];
            const uint32_t nb = (uint32_t)((J.nout + 1 + CRT_BLK - 1) / CRT_BLK);
            for (uint32_t k = idx * PERSIST_CRT; k < nb && k < (idx + 1) * PERSIST_CRT; ++k) {
                crt_body(k, J.ws, (int64_t)1 << lg, J.cmin, J.cmax, J.off, J.out, J.nout, J.flags, err,
                         *reinterpret_cast<CrtSmem*>(sm));
                __syncthreads();
            }
            break;
        }
        default: break;
    }
}

// LOOP: persistent CTAs (grid = what fits on the device) take items until
// the queue is empty; otherwise one item per CTA (grid = the item count),
// in the same queue order.
#ifndef PERSIST_MINB
#define PERSIST_MINB 4             // resident CTAs per SM the register budget is set for
#endif
template <bool LOOP>
__global__ void __launch_bounds__(PERSIST_THREADS, PERSIST_MINB)
    k_persist(const PItem* __restrict__ items, int nitems, const JobDesc* __restrict__ jobs,
              const PClass* __restrict__ cls, uint32_t* state, const uint2* __restrict__ twf,
              const uint2* __restrict__ twi, uint32_t* err) {
    extern __shared__ uint32_t sm[];
    // the current item and the next one, in shared memory so that nothing of
    // them stays live in registers across the stage bodies.  A persistent
    // CTA takes its next item (queue-head increment and item load) at the
    // start of the current one, so those round trips overlap the body; it
    // runs the two in queue order, so the waits' progress argument holds.
    __shared__ PItem s_it, s_nx;
    __shared__ int s_more, s_hasnx;
    if (threadIdx.x == 0) {
        const int it = (int)atomicAdd(&state[0], 1u);
        s_hasnx = it < nitems;
        if (it < nitems) s_nx = items[it];
    }
    do {
        if (threadIdx.x == 0) {
            s_more = s_hasnx;
            if (s_more) {
                const PItem I = s_nx;
                s_it = I;
                if (I.need) persist_wait(&state[1 + I.job], I.need, err);
            }
        }
        __syncthreads();
        if (!s_more) return;
        if (LOOP && PERSIST_PREFETCH && threadIdx.x == 0) {
            const int it = (int)atomicAdd(&state[0], 1u);
            s_hasnx = it < nitems;
            if (it < nitems) s_nx = items[it];
        }
        // warp-uniform copies (a warp reduction's result), so that the
        // bodies' index arithmetic stays on the uniform datapath
        const uint32_t kind = __reduce_max_sync(0xffffffffu, (uint32_t)s_it.kind);
        const uint32_t job = __reduce_max_sync(0xffffffffu, s_it.job);
        persist_item(kind, job, __reduce_max_sync(0xffffffffu, (uint32_t)s_it.lg),
                     __reduce_max_sync(0xffffffffu, s_it.idx), jobs, cls, twf, twi, err, sm);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (kind != PK_SCHOOL && kind != PK_SMALLJOB) persist_signal(&state[1 + job]);
            if (LOOP && !PERSIST_PREFETCH) {
                const int it = (int)atomicAdd(&state[0], 1u);
                s_hasnx = it < nitems;
                if (it < nitems) s_nx = items[it];
            }
        }
    } while (LOOP);
}

size_t persist_smem_bytes() {
    size_t b = sizeof(RowSmem);
    b = std::max(b, sizeof(CrtSmem));
    b = std::max(b, (size_t)2 * padded_len(1 << SBG_SMALL_MAX_LG) * 4);
    b = std::max(b, (size_t)(PERSIST_THREADS / 32) * 2 * SBG_SCHOOL_MAX * 8);
    b = std::max(b, (size_t)col_smem_bytes(5));
    b = std::max(b, (size_t)col_smem_bytes(6));
    b = std::max(b, (size_t)col_smem_bytes(7));
    b = std::max(b, (size_t)col_smem_bytes(8));
    return (b + 255) & ~(size_t)255;
}

int persist_grid(int device) {
    static int cached[64] = {};
    if (device < 0 || device >= 64) return 0;
    if (cached[device]) return cached[device];
    const size_t smem = persist_smem_bytes();
    if (cudaFuncSetAttribute(k_persist<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_persist<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return 0;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist<true>, PERSIST_THREADS, smem) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return 0;
    cached[device] = std::max(1, per_sm) * sms;
    return cached[device];
}

cudaError_t launch_persist(const PItem* items, int nitems, const JobDesc* jobs, const PClass* cls,
                           uint32_t* state, const uint2* tw_f, const uint2* tw_i, uint32_t* err, int grid,
                           cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    const size_t smem = persist_smem_bytes();
    if (grid > 0)
        k_persist<true><<<std::min(grid, nitems), PERSIST_THREADS, smem, st>>>(items, nitems, jobs, cls, state,
                                                                                tw_f, tw_i, err);
    else
        k_persist<false><<<nitems, PERSIST_THREADS, smem, st>>>(items, nitems, jobs, cls, state, tw_f, tw_i,
                                                                 err);
    return cudaGetLastError();
}

}  // namespace sbg
