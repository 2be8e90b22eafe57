// Per-node work of the fused monodomain ionic step, shared by the
// single-simulation and batched kernels.
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

// Istim = sum of the active stimuli of a node in list order (stimulation.py:59-61)
__device__ __forceinline__ float stim_sum(const MonoDev& d, uint32_t smask, uint32_t bits) {
    float I = 0.0f;
    bool first = true;
    for (int k = 0; k < TCB_MAX_STIMULI; ++k) {
        if ((smask >> k) & 1u) {
            const float a = ((bits >> k) & 1u) ? d.amp[k] : 0.0f;
            I = first ? a : I + a;
            first = false;
        }
    }
    return I;
}

// AT/RT and snapshot of the previous step, ionic update, stimulus and
// b' = u*Cm + dt*du/100 + dt*Istim/100 (monodomain.py:117-128) for node i.
template <class M, class Q>
__device__ __forceinline__ void ionic_node(const MonoDev& d, const typename M::C& c, const typename M::Tables& T,
                                           const StepView& sv, int64_t i) {
    const float v = sv.u[i];
    if (sv.do_atrt) at_rt_update(v, sv.t_prev, d.at, d.rt, i);
    if (sv.snap) sv.snap[i] = v;
    float s[M::kStates];
#pragma unroll
    for (int k = 0; k < M::kStates; ++k) s[k] = d.state[k * d.n_pad + i];
    const float dV = M::template step<Q>(v, s, c, T, M::node_g(c, d.node_params, d.n_pad, i));
#pragma unroll
    for (int k = 0; k < M::kStates; ++k) d.state[k * d.n_pad + i] = s[k];
    // b = u*Cm + dt*du, du = dV/100  (monodomain.py:117-118)
    float b = v * d.cm + d.dt * Q::div(dV, 100.0f);
    if (sv.smask) {
        // Istim/100 (monodomain.py:127), b += dt*Istim (:128)
        const uint32_t bits = d.stim_bits[i] & sv.smask;
        if (bits) b = b + d.dt * Q::div(stim_sum(d, sv.smask, bits), 100.0f);
    }
    d.bp[i] = b;
}

// V consecutive per-node values as one 8- or 16-byte access (the arrays are
// n_pad long, n_pad a multiple of 128, and aligned to the vector).
template <int V, typename T>
__device__ __forceinline__ void ld_nodes(const T* __restrict__ p, T (&o)[V]) {
    static_assert(sizeof(T) == 4 && (V == 2 || V == 4), "2 or 4 four-byte values");
    if constexpr (V == 4) {
        const uint4 t = *reinterpret_cast<const uint4*>(p);
        const uint32_t w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) o[j] = __builtin_bit_cast(T, w[j]);
    } else {
        const uint2 t = *reinterpret_cast<const uint2*>(p);
        o[0] = __builtin_bit_cast(T, t.x);
        o[1] = __builtin_bit_cast(T, t.y);
    }
}

template <int V>
__device__ __forceinline__ void st_nodes(float* __restrict__ p, const float (&v)[V]) {
    static_assert(V == 1 || V == 2 || V == 4, "1, 2 or 4 floats");
    if constexpr (V == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else if constexpr (V == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else *p = v[0];
}

// ionic_node for the V consecutive nodes i0 .. i0+V-1 (V = 1, 2 or 4; Q the
// division policy), with the
// per-node arrays moved as vectors for V > 1.  Nodes between n and n_pad are
// padding: their ionic arithmetic runs on memory that exists but nothing reads
// its results; their u stays 0, so AT/RT are never set for them, and snapshots
// are written for real nodes only.
template <class M, int V, class Q>
__device__ __forceinline__ void ionic_group(const MonoDev& d, const typename M::C& c, const typename M::Tables& T,
                                            const StepView& sv, int64_t i0) {
    if constexpr (V == 1) {
        ionic_node<M, Q>(d, c, T, sv, i0);
    } else {
        float v[V];
        ld_nodes<V>(sv.u + i0, v);
        if (sv.do_atrt) {
            float a[V], r[V];
            ld_nodes<V>(d.at + i0, a);
            ld_nodes<V>(d.rt + i0, r);
#pragma unroll
            for (int j = 0; j < V; ++j) {
                if (v[j] > 0.0f && a[j] == -1.0f) {
                    a[j] = sv.t_prev;
                    d.at[i0 + j] = a[j];
                }
                if (a[j] > 0.0f && v[j] < -70.0f && r[j] == -1.0f) d.rt[i0 + j] = sv.t_prev;
            }
        }
        if (sv.snap) {
#pragma unroll
            for (int j = 0; j < V; ++j)
                if (i0 + j < d.n) sv.snap[i0 + j] = v[j];
        }
        float s[V][M::kStates];
#pragma unroll
        for (int k = 0; k < M::kStates; ++k) {
            float t[V];
            ld_nodes<V>(d.state + k * d.n_pad + i0, t);
#pragma unroll
            for (int j = 0; j < V; ++j) s[j][k] = t[j];
        }
        float b[V];
#pragma unroll
        for (int j = 0; j < V; ++j)
            b[j] = v[j] * d.cm +
                   d.dt * Q::div(M::template step<Q>(v[j], s[j], c, T, M::node_g(c, d.node_params, d.n_pad, i0 + j)),
                                 100.0f);
#pragma unroll
        for (int k = 0; k < M::kStates; ++k) {
            float t[V];
#pragma unroll
            for (int j = 0; j < V; ++j) t[j] = s[j][k];
            st_nodes<V>(d.state + k * d.n_pad + i0, t);
        }
        if (sv.smask) {
            uint32_t bits[V];
            ld_nodes<V>(d.stim_bits + i0, bits);
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const uint32_t on = bits[j] & sv.smask;
                if (on) b[j] = b[j] + d.dt * Q::div(stim_sum(d, sv.smask, on), 100.0f);
            }
        }
        st_nodes<V>(d.bp + i0, b);
    }
}

}  // namespace tcb
