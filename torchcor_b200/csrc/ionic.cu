// Per-step ionic kernels: the stand-alone differentiate() and the fused
// per-step kernel of the monodomain loop (activation/repolarisation update of
// the previous step, snapshot, ionic update, stimulus injection and the
// right-hand side b' = u*Cm + dt*du/100 + dt*Istim/100 of monodomain.py:117-128).
//
// The fused kernel is instantiated for several launch shapes: 1, 2 or 4
// consecutive nodes per thread (structure-of-arrays state read and written as
// 4-, 8- or 16-byte vectors), a register budget set by the blocks per SM it is
// compiled for, and a division/logarithm policy (QFast or QExact,
// ionic_common.cuh).  tcb_mono.ionic_variant picks one (the autotuner measures
// them); every instance runs the reference's per-node order of operations.
//
// Compiled with multiply-add contraction.  Lookup tables are built in tables.cu
// with separate roundings.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "ionic_crn.cuh"
#include "ionic_ms.cuh"
#include "ionic_node.cuh"
#include "ionic_ttp.cuh"
#include "mono.cuh"
#include "tcb_internal.h"

namespace tcb {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) {
    int64_t b = ceil_div(n, kThreads);
    return (unsigned)(b > 148 * 64 ? 148 * 64 : b);
}

template <class M>
__global__ void differentiate_kernel(typename M::C c, typename M::Tables T, float* state, int64_t n_pad, int64_t n,
                                     const float* __restrict__ v, float* __restrict__ dv) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float s[M::kStates];
#pragma unroll
        for (int k = 0; k < M::kStates; ++k) s[k] = state[k * n_pad + i];
        float d = M::template step<QFast>(v[i], s, c, T);
#pragma unroll
        for (int k = 0; k < M::kStates; ++k) state[k * n_pad + i] = s[k];
        dv[i] = d;
    }
}

template <class M, int V, int MINB, class Q>
__global__ void __launch_bounds__(kThreads, MINB) mono_ionic_kernel(MonoDev d, typename M::C c, typename M::Tables T) {
    const StepView sv = step_view(d, d.counter[0]);
    const int64_t groups = (d.n + V - 1) / V;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += (int64_t)gridDim.x * blockDim.x)
        ionic_group<M, V, Q>(d, c, T, sv, g * V);
}

__global__ void mono_finish_kernel(MonoDev d) {
    const int64_t n = d.counter[0];  // nt + 1 after the last step
    const int64_t last = n - 1;
    if (last < 1) return;
    const float* u = d.x + ring_cur(n) * d.n_pad;
    const float t = d.step_t[last];
    float* snap = (d.snap && d.per_frame > 0 && last % d.per_frame == 0) ? d.snap + snap_row(d, last / d.per_frame) * d.n
                                                                          : nullptr;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += (int64_t)gridDim.x * blockDim.x) {
        float v = u[i];
        if (d.at_rt) at_rt_update(v, t, d.at, d.rt, i);
        if (snap) snap[i] = v;
    }
}

template <class M>
using LaunchFn = int (*)(const MonoDev&, const typename M::C&, const typename M::Tables&, cudaStream_t);

template <class M, int V, int MINB, class Q>
int launch_shape(const MonoDev& d, const typename M::C& c, const typename M::Tables& T, cudaStream_t s) {
    mono_ionic_kernel<M, V, MINB, Q><<<grid_for(ceil_div(d.n, V)), kThreads, 0, s>>>(d, c, T);
    TCB_CHECK_LAUNCH("mono ionic kernel");
    return TCB_OK;
}

// The instances of each model: nodes per thread, 256-thread blocks per SM the
// register budget is set for, division/log policy (1 = QFast, 0 = QExact);
// entry 0 is the default (the fastest measured on the million-node cubes).
struct Shape {
    int32_t nodes_per_thread, blocks_per_sm, fast;
};
template <class M>
struct Shapes;
template <>
struct Shapes<MS> {
    static constexpr int kCount = 5;
    static constexpr Shape shape[kCount] = {{4, 8, 0}, {1, 1, 0}, {2, 1, 0}, {4, 4, 0}, {4, 1, 0}};
    static constexpr LaunchFn<MS> fn[kCount] = {launch_shape<MS, 4, 8, QExact>, launch_shape<MS, 1, 1, QExact>,
                                                launch_shape<MS, 2, 1, QExact>, launch_shape<MS, 4, 4, QExact>,
                                                launch_shape<MS, 4, 1, QExact>};
};
template <>
struct Shapes<TTP> {
    static constexpr int kCount = 8;
    static constexpr Shape shape[kCount] = {{1, 4, 0}, {1, 6, 0}, {2, 3, 0}, {4, 2, 0},
                                            {1, 2, 1}, {1, 3, 1}, {2, 2, 1}, {4, 1, 1}};
    static constexpr LaunchFn<TTP> fn[kCount] = {
        launch_shape<TTP, 1, 4, QExact>, launch_shape<TTP, 1, 6, QExact>, launch_shape<TTP, 2, 3, QExact>,
        launch_shape<TTP, 4, 2, QExact>, launch_shape<TTP, 1, 2, QFast>,  launch_shape<TTP, 1, 3, QFast>,
        launch_shape<TTP, 2, 2, QFast>,  launch_shape<TTP, 4, 1, QFast>};
};
template <>
struct Shapes<CRN> {
    static constexpr int kCount = 6;
    static constexpr Shape shape[kCount] = {{2, 2, 1}, {1, 3, 1}, {1, 2, 1}, {4, 1, 1}, {1, 3, 0}, {2, 2, 0}};
    static constexpr LaunchFn<CRN> fn[kCount] = {
        launch_shape<CRN, 2, 2, QFast>, launch_shape<CRN, 1, 3, QFast>,  launch_shape<CRN, 1, 2, QFast>,
        launch_shape<CRN, 4, 1, QFast>, launch_shape<CRN, 1, 3, QExact>, launch_shape<CRN, 2, 2, QExact>};
};

inline bool aligned(const void* p, unsigned bytes) { return ((uintptr_t)p & (bytes - 1)) == 0; }

// Vector accesses need every per-node array aligned to the vector: otherwise the
// first one-node-per-thread instance runs.
template <class M>
int launch_mono(const tcb_mono* m, const MonoDev& d, cudaStream_t s) {
    typename M::C c = M::derive(m->params);
    typename M::Tables T = M::tables(m->tables, m->params);
    int k = m->ionic_variant > 0 ? m->ionic_variant - 1 : 0;
    if (k >= Shapes<M>::kCount) return fail(TCB_ERANGE, "tcb_mono: no such ionic kernel variant");
    const unsigned vb = 4u * (unsigned)Shapes<M>::shape[k].nodes_per_thread;
    if (vb > 4 && !(aligned(d.x, vb) && aligned(d.state, vb) && aligned(d.bp, vb) && aligned(d.at, vb) &&
                    aligned(d.rt, vb) && aligned(d.stim_bits, vb))) {
        k = 0;
        while (Shapes<M>::shape[k].nodes_per_thread != 1) ++k;
    }
    return Shapes<M>::fn[k](d, c, T, s);
}

template <class M>
int run_differentiate(const double* params, const float* tables, float* state, int64_t n_pad, int64_t n,
                      const float* v, float* dv, cudaStream_t s) {
    differentiate_kernel<M><<<grid_for(n), kThreads, 0, s>>>(M::derive(params), M::tables(tables, params), state,
                                                             n_pad, n, v, dv);
    TCB_CHECK_LAUNCH("differentiate kernel");
    return TCB_OK;
}

}  // namespace

int launch_mono_ionic(const tcb_mono* m, const MonoDev& d, cudaStream_t s) {
    switch (m->model) {
        case TCB_MODEL_MS: return launch_mono<MS>(m, d, s);
        case TCB_MODEL_TTP: return launch_mono<TTP>(m, d, s);
        case TCB_MODEL_CRN: return launch_mono<CRN>(m, d, s);
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

template <class M>
int variant_info(int32_t variant, int32_t* count, int32_t* nodes_per_thread, int32_t* blocks_per_sm,
                 int32_t* fast) {
    *count = Shapes<M>::kCount;
    if (variant < 0 || variant > Shapes<M>::kCount) return fail(TCB_ERANGE, "no such ionic kernel variant");
    const Shape& sh = Shapes<M>::shape[variant > 0 ? variant - 1 : 0];
    *nodes_per_thread = sh.nodes_per_thread;
    *blocks_per_sm = sh.blocks_per_sm;
    *fast = sh.fast;
    return TCB_OK;
}

int launch_mono_finish(const MonoDev& d, cudaStream_t s) {
    mono_finish_kernel<<<grid_for(d.n), kThreads, 0, s>>>(d);
    TCB_CHECK_LAUNCH("mono finish kernel");
    return TCB_OK;
}

}  // namespace tcb

using namespace tcb;

extern "C" int tcb_model_differentiate(int32_t model, const double* params, const float* tables, float* state,
                                       int64_t n_pad, int64_t n, const float* v, float* dv, void* stream) {
    if (!params || !state || !v || !dv || n <= 0 || n_pad < n) return fail(TCB_EINVAL, "tcb_model_differentiate: bad arguments");
    if (model != TCB_MODEL_MS && !tables) return fail(TCB_EINVAL, "tcb_model_differentiate: null tables");
    if (model != TCB_MODEL_MS && ((uintptr_t)tables & 15u))
        return fail(TCB_EINVAL, "tcb_model_differentiate: tables not 16-byte aligned");
    cudaStream_t s = as_stream(stream);
    switch (model) {
        case TCB_MODEL_MS: return run_differentiate<MS>(params, tables, state, n_pad, n, v, dv, s);
        case TCB_MODEL_TTP: return run_differentiate<TTP>(params, tables, state, n_pad, n, v, dv, s);
        case TCB_MODEL_CRN: return run_differentiate<CRN>(params, tables, state, n_pad, n, v, dv, s);
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

extern "C" int tcb_ionic_variant(int32_t model, int32_t variant, int32_t* count, int32_t* nodes_per_thread,
                                 int32_t* blocks_per_sm, int32_t* fast_math) {
    if (!count || !nodes_per_thread || !blocks_per_sm || !fast_math)
        return fail(TCB_EINVAL, "tcb_ionic_variant: null output");
    switch (model) {
        case TCB_MODEL_MS: return variant_info<MS>(variant, count, nodes_per_thread, blocks_per_sm, fast_math);
        case TCB_MODEL_TTP: return variant_info<TTP>(variant, count, nodes_per_thread, blocks_per_sm, fast_math);
        case TCB_MODEL_CRN: return variant_info<CRN>(variant, count, nodes_per_thread, blocks_per_sm, fast_math);
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}
