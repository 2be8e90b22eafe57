// Grid-barrier and reduction helpers shared by the persistent CG kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tcb200.h"

namespace tcb {
namespace cgk {

constexpr int kCgThreads = 512;
constexpr int kCgWarps = kCgThreads / 32;
constexpr int kMinSlicesPerBlock = 2 * kCgWarps;
constexpr int kMaxBlocks = 2048;
constexpr uint64_t kBarrierTimeoutNs = 2000000000ull;  // 2 s: a wait that long means a lost block

// Limits of the bounded device waits (grid barriers, bulk-copy mbarriers).
// In normal runs: the 2 s timeout and nothing else.  The failure-detection
// tests set TCB_TEST_WAIT_STALL (wait_limit() in api.cu): then the timeout is
// 10 ms and either every grid barrier waits for one arrival more than the grid
// has ("grid") or the first bulk copies of the batched kernels' first warp or
// block are not made while their mbarrier still expects the bytes ("copy"), so
// that a wait runs out, the error word is set and every block returns.
struct WaitLimit {
    uint64_t timeout_ns;
    uint32_t extra_arrivals;
    uint32_t drop_first_copy;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Grid-wide barrier with a bounded wait: returns false (and the kernel must
// return) if any block recorded an error or the wait ran past the timeout.
// One 64-bit word (bar[0..1], 8-byte aligned): arrivals in the low half, the
// generation in the high half.  A block's arrival (one atomic add) returns the
// generation it waits to see change; the last arrival adds 2^32 - gridDim.x,
// which clears the count and advances the generation in one operation, so no
// block can arrive at the next barrier before the count is clear.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, int32_t* err, const WaitLimit& w) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        unsigned long long* word = reinterpret_cast<unsigned long long*>(bar);
        __threadfence();   // this block's writes before its arrival
        const unsigned long long old = atomicAdd(word, 1ull);
        const unsigned gen = (unsigned)(old >> 32);
        if ((unsigned)old == gridDim.x - 1 + w.extra_arrivals) {
            atomicAdd(word, (1ull << 32) - (unsigned long long)gridDim.x);
        } else {
            const uint64_t t0 = globaltimer();
            while ((unsigned)(ld_acquire64(word) >> 32) == gen) {
                if (*(volatile int32_t*)err != 0) {
                    good = 0;
                    break;
                }
                if (globaltimer() - t0 > w.timeout_ns) {
                    atomicCAS(err, 0, TCB_ETIMEOUT);
                    good = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (*(volatile int32_t*)err != 0) good = 0;
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Block partial of NV float64 values -> parts[blockIdx.x * NV + i] (fixed order).
template <int NV>
__device__ __forceinline__ void block_partial(double (&v)[NV], double* parts, double* sh) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double t = warp_sum(v[i]);
        if (lane == 0) sh[warp * NV + i] = t;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double t = lane < kCgWarps ? sh[lane * NV + i] : 0.0;
            t = warp_sum(t);
            if (lane == 0) parts[blockIdx.x * NV + i] = t;
        }
    }
}

// Sum of all blocks' partials; every block computes the same value.  Each lane
// adds the partials of blocks lane, lane + 32, ... in that order; the loads of
// eight strides are issued before their adds, so a lane waits for one L2 round
// trip per eight strides instead of one per stride (same sums, bit for bit).
template <int NV>
__device__ __forceinline__ void grid_total(const double* parts, double (&out)[NV], double* sh) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        constexpr int kBatch = 8;
        double acc[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) acc[i] = 0.0;
        const unsigned nb = gridDim.x;
        unsigned b = lane;
        for (; b + 32 * (kBatch - 1) < nb; b += 32 * kBatch) {
            double t[kBatch][NV];
#pragma unroll
            for (int k = 0; k < kBatch; ++k)
#pragma unroll
                for (int i = 0; i < NV; ++i) t[k][i] = __ldcg(parts + (b + 32 * k) * NV + i);
#pragma unroll
            for (int k = 0; k < kBatch; ++k)
#pragma unroll
                for (int i = 0; i < NV; ++i) acc[i] += t[k][i];
        }
        for (; b < nb; b += 32)
#pragma unroll
            for (int i = 0; i < NV; ++i) acc[i] += __ldcg(parts + b * NV + i);
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            acc[i] = warp_sum(acc[i]);
            if (lane == 0) sh[i] = acc[i];
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; ++i) out[i] = sh[i];
}

}  // namespace cgk
}  // namespace tcb
