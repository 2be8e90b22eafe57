// L2 eviction priorities for the per-step streams (createpolicy + L2::cache_hint).
//
// A monodomain step moves more bytes than the 126 MB L2 holds: the ionic state
// (read and written once a step), M and K (read once a step by the right-hand
// side) and the column offsets and A values (read by every CG pass; 91 MB for a
// million-node cube).  The resident CG kernel loads the column offsets (30 MB) as
// last-to-go and M, K and A as first-to-go, so the offsets the right-hand side
// read stay in L2 through the A p passes; with A last-to-go too the set no longer
// fitted and a launch took 10 % longer.  Hints only: no result depends on them.
#pragma once

#include <stdint.h>

namespace tcb {

// policy for data read again by later passes and steps
__device__ __forceinline__ uint64_t l2_keep() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// policy for data touched once a step
__device__ __forceinline__ uint64_t l2_once() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Read-only (non-coherent path) loads of data no thread writes during the kernel,
// in two forms, because the two CG kernels need opposite ones (measured on B200):
//  * ld_hint: volatile asm, issued in program order where written.  The resident
//    CG kernel relies on that: with the plain form the compiler rescheduled its
//    loads and a launch on a million-node cube went from 0.099 to 0.128 ms;
//  * ld_hint_sched (with l2_once_sched): plain asm without a memory clobber, which
//    the compiler schedules like __ldg.  The batched CG kernel needs that for its
//    column prefetch: with the volatile form a 64-cube batch step took 1.21 ms
//    instead of 0.70.
__device__ __forceinline__ float ld_hint(const float* a, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_hint(const int32_t* a, uint64_t pol) {
    int v;
    asm volatile("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_hint(const int16_t* a, uint64_t pol) {
    short v;
    asm volatile("ld.global.nc.L2::cache_hint.s16 %0, [%1], %2;" : "=h"(v) : "l"(a), "l"(pol));
    return (int)v;
}


// the schedulable form (see above)
__device__ __forceinline__ uint64_t l2_once_sched() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ float ld_hint_sched(const float* a, uint64_t pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_hint_sched(const int32_t* a, uint64_t pol) {
    int v;
    asm("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_hint_sched(const int16_t* a, uint64_t pol) {
    short v;
    asm("ld.global.nc.L2::cache_hint.s16 %0, [%1], %2;" : "=h"(v) : "l"(a), "l"(pol));
    return (int)v;
}

}  // namespace tcb
