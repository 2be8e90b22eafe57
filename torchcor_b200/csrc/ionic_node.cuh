// Per-node work of the fused monodomain ionic step, shared by the
// single-simulation and batched kernels (both compiled with -fmad=false).
#pragma once
#include "ionic_common.cuh"
#include "mono.cuh"

namespace tcb {

// activation / repolarisation update of monodomain.py:174-176 for time t
__device__ __forceinline__ void at_rt_update(float u, float t, float* at, float* rt, int64_t i) {
    float a = at[i];
    if (u > 0.0f && a == -1.0f) {
        a = t;
        at[i] = a;
    }
    if (a > 0.0f && u < -70.0f && rt[i] == -1.0f) rt[i] = t;
}

// What one step of a simulation needs besides its arrays.
struct StepView {
    const float* u;       // solution of the previous step
    float t_prev;         // time of the previous step (for AT/RT)
    bool do_atrt;
    float* snap;          // snapshot row of the previous step, or null
    uint32_t smask;       // stimuli active at this step
};

__device__ __forceinline__ StepView step_view(const MonoDev& d, int64_t n) {
    StepView v;
    v.u = d.x + ring_cur(n) * d.n_pad;
    const int64_t prev = n - 1;
    v.do_atrt = d.at_rt && prev >= 1;
    v.t_prev = d.step_t[prev];
    // step numbers and frame intervals are below 2^31 (validated on the host)
    const uint32_t pv = (uint32_t)prev, pf = (uint32_t)d.per_frame;
    v.snap = (d.snap && d.per_frame > 0 && prev >= 1 && pv % pf == 0u) ? d.snap + snap_row(d, pv / pf) * d.n
                                                                      : nullptr;
    v.smask = d.step_stim[n];
    return v;
}

// AT/RT and snapshot of the previous step, ionic update, stimulus and
// b' = u*Cm + dt*du/100 + dt*Istim/100 (monodomain.py:117-128) for node i.
template <class M>
__device__ __forceinline__ void ionic_node(const MonoDev& d, const typename M::C& c, const typename M::Tables& T,
                                           const StepView& sv, int64_t i) {
    const float v = sv.u[i];
    if (sv.do_atrt) at_rt_update(v, sv.t_prev, d.at, d.rt, i);
    if (sv.snap) sv.snap[i] = v;
    float s[M::kStates];
#pragma unroll
    for (int k = 0; k < M::kStates; ++k) s[k] = d.state[k * d.n_pad + i];
    const float dV = M::step(v, s, c, T);
#pragma unroll
    for (int k = 0; k < M::kStates; ++k) d.state[k * d.n_pad + i] = s[k];
    // b = u*Cm + dt*du, du = dV/100  (monodomain.py:117-118)
    float b = v * d.cm + d.dt * (dV / 100.0f);
    if (sv.smask) {
        // Istim = sum of the active stimuli in list order (stimulation.py:59-61), /100 (:127)
        const uint32_t bits = d.stim_bits[i] & sv.smask;
        if (bits) {
            float I = 0.0f;
            bool first = true;
            for (int k = 0; k < TCB_MAX_STIMULI; ++k) {
                if ((sv.smask >> k) & 1u) {
                    const float a = ((bits >> k) & 1u) ? d.amp[k] : 0.0f;
                    I = first ? a : I + a;
                    first = false;
                }
            }
            b = b + d.dt * (I / 100.0f);
        }
    }
    d.bp[i] = b;
}

}  // namespace tcb
