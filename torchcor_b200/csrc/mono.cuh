// Device view of one monodomain simulation (built from tcb_mono on the host).
#pragma once
#include <stdint.h>

#include "cg_common.cuh"
#include "tcb200.h"

namespace tcb {

// limits of the bounded device waits for this process (TCB_TEST_WAIT_STALL, see cg_common.cuh)
cgk::WaitLimit wait_limit();

struct MonoDev {
    int64_t n, n_pad, n_slices, nt;
    const int64_t* slice_ptr;
    const int32_t* col;
    const int16_t* dcol;   // int16 column offsets from the row, or null
    const float *mv, *kv, *av, *dinv;
    float* state;
    const float* tables;
    float *x, *bp, *r, *p, *ap, *z, *p2, *at, *rt, *snap;
    const float* node_params;   // per-node model parameters (n_params, n_pad), or null
    const uint32_t* stim_bits;
    const float* step_t;
    const uint32_t* step_stim;
    int32_t* step_iters;
    int32_t* counter;
    double* scratch;
    uint32_t* bar;
    double a_tol, r_tol;
    int32_t max_iter, linear_guess, at_rt, per_frame;
    int32_t a_split;   // A == fp32(fp32(M*Cm) + K') verified at assembly
    float cm, dt;
    int32_t snap_ring;        // snapshot rows: 0 = one per frame, > 0 = ring of that many
    int32_t cg_per_sm;        // resident CG blocks per SM: 0 = most that fit, 1 or 2 pinned
    cgk::WaitLimit wait;      // bounded-wait limits of the grid barriers
    float amp[TCB_MAX_STIMULI];
};

MonoDev make_dev(const tcb_mono* m);

// snapshot row of frame f (frame f = solution of step f * per_frame)
__host__ __device__ inline int64_t snap_row(const MonoDev& d, int64_t f) { return d.snap_ring > 0 ? f % d.snap_ring : f; }

// membrane-potential ring: step n reads slot (n-1)%3, guesses from (n+1)%3, writes n%3
__host__ __device__ inline int64_t ring_cur(int64_t n) { return (n + 2) % 3; }
__host__ __device__ inline int64_t ring_prev(int64_t n) { return (n + 1) % 3; }
__host__ __device__ inline int64_t ring_next(int64_t n) { return n % 3; }

// launchers implemented in ionic.cu / cg.cu
int launch_mono_ionic(const tcb_mono* m, const MonoDev& d, cudaStream_t s);
int launch_mono_finish(const MonoDev& d, cudaStream_t s);
int launch_cg(const MonoDev& d, cudaStream_t s);
int launch_cg_resident(const MonoDev& d, cudaStream_t s);
int resident_blocks(const MonoDev& d);
int launch_mono_step(const tcb_mono* m, const MonoDev& d, cudaStream_t s);   // 1 launched, 0 not applicable
int mono_step_fusable(const tcb_mono* m, const MonoDev& d);
bool cg_forced_fallback();
// 1 if tcb_mono_run runs this simulation's steps as the fused kernel
inline int uses_fused_step(const tcb_mono* m, const MonoDev& d) {
    return m->fused_step && !cg_forced_fallback() && mono_step_fusable(m, d);
}
int cg_uses_resident(const MonoDev& d);

}  // namespace tcb
