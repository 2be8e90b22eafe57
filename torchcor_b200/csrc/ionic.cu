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

#include <algorithm>
#include <math.h>
#include <string.h>

#include "bulk.cuh"
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
__global__ void differentiate_kernel(typename M::C c, typename M::Tables T, const float* node_params, float* state,
                                     int64_t n_pad, int64_t n, const float* __restrict__ v, float* __restrict__ dv) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float s[M::kStates];
#pragma unroll
        for (int k = 0; k < M::kStates; ++k) s[k] = state[k * n_pad + i];
        float d = M::template step<QFast>(v[i], s, c, T, M::node_g(c, node_params, n_pad, i));
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

// Persistent, double-buffered instance: a block walks 256*V-node tiles; one
// thread copies the next tile's state rows, u, AT/RT and stimulus bits into
// shared memory by bulk asynchronous copies (mbarrier completion) while the
// block computes the current tile from shared memory, so the loads of one tile
// overlap the arithmetic of the other.  Results go straight to global memory.
// Blocks never wait for each other; every mbarrier wait is bounded (the error
// word gets TCB_ETIMEOUT, the block lets its other copies land, then returns).
// tiles in flight per block: two (three measured slower on B200: TTP 37.5 -> 39.5
// us a launch at (1,3,fast), the four-blocks-per-SM instances no longer resident)
#ifndef TCB_IONIC_STAGES
#define TCB_IONIC_STAGES 2
#endif
template <class M, int V>
struct StagedTile {
    static constexpr int kStages = TCB_IONIC_STAGES;     // tiles in flight per block
    static constexpr int kTile = kThreads * V;           // nodes per tile
    static constexpr int kRows = M::kStates + 4;         // state rows, u, AT, RT, stimulus bits
    static constexpr size_t kBytes = (size_t)kStages * kRows * kTile * sizeof(float);   // all stages
};

template <class M, int V, int MINB, class Q>
__global__ void __launch_bounds__(kThreads, MINB) mono_ionic_staged_kernel(MonoDev d, typename M::C c,
                                                                            typename M::Tables T, int64_t n_tiles) {
    using ST = StagedTile<M, V>;
    constexpr int S = M::kStates, kTile = ST::kTile, kRows = ST::kRows, NS = ST::kStages;
    extern __shared__ __align__(128) float stage[];      // [NS][kRows][kTile]
    __shared__ __align__(8) uint64_t bar[NS];
    const StepView sv = step_view(d, d.counter[0]);
    int32_t* err = d.counter + 1;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int st = 0; st < NS; ++st) mbar_init(&bar[st]);
        mbar_init_fence();
    }
    __syncthreads();
    // thread 0: copy tile `tile` into stage `st`
    auto issue = [&](int st, int64_t tile) {
        const int64_t i0 = tile * kTile;
        const uint32_t bytes = (uint32_t)(min((int64_t)kTile, d.n_pad - i0) * 4);
        float* buf = stage + (size_t)st * kRows * kTile;
        const uint32_t total = bytes * (S + 1) + (sv.do_atrt ? 2 * bytes : 0) + (sv.smask ? bytes : 0);
        fence_proxy_async_smem();
        mbar_arrive_tx(&bar[st], total);
        for (int k = 0; k < S; ++k) bulk_load(buf + k * kTile, d.state + k * d.n_pad + i0, bytes, &bar[st]);
        bulk_load(buf + S * kTile, sv.u + i0, bytes, &bar[st]);
        if (sv.do_atrt) {
            bulk_load(buf + (S + 1) * kTile, d.at + i0, bytes, &bar[st]);
            bulk_load(buf + (S + 2) * kTile, d.rt + i0, bytes, &bar[st]);
        }
        if (sv.smask) bulk_load(buf + (S + 3) * kTile, d.stim_bits + i0, bytes, &bar[st]);
    };
    const int64_t first = blockIdx.x, stride = gridDim.x;
    if (tid == 0)
        for (int st = 0; st < NS; ++st)
            if (first + st * stride < n_tiles) issue(st, first + st * stride);
    uint32_t phase = 0;
    int k = 0;
    for (int64_t tile = first; tile < n_tiles; tile += stride, ++k) {
        const int st = k % NS;
        const bool ok = __syncthreads_and(mbar_wait_thread(&bar[st], (phase >> st) & 1u, d.wait.timeout_ns));
        if (!ok) {
            // a copy did not complete in time: record it, give the other stage's
            // copies (issued for the next tile) a bounded wait, and return
            if (tid == 0) atomicCAS(err, 0, TCB_ETIMEOUT);
            for (int j = 1; j < NS; ++j) {   // the other stages hold tiles tile + j*stride
                const int o = (st + j) % NS;
                if (tile + j * stride < n_tiles) mbar_wait_thread(&bar[o], (phase >> o) & 1u, d.wait.timeout_ns);
            }
            return;
        }
        phase ^= 1u << st;
        const float* buf = stage + (size_t)st * kRows * kTile;
        const int j0 = tid * V;
        const int64_t i0 = tile * kTile + j0;
        if (i0 < d.n_pad) {
            float v[V];
#pragma unroll
            for (int j = 0; j < V; ++j) v[j] = buf[S * kTile + j0 + j];
            if (sv.do_atrt) {
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    float a = buf[(S + 1) * kTile + j0 + j];
                    if (v[j] > 0.0f && a == -1.0f) {   // padding nodes keep u = 0 and never pass
                        a = sv.t_prev;
                        d.at[i0 + j] = a;
                    }
                    if (a > 0.0f && v[j] < -70.0f && buf[(S + 2) * kTile + j0 + j] == -1.0f) d.rt[i0 + j] = sv.t_prev;
                }
            }
            if (sv.snap) {
#pragma unroll
                for (int j = 0; j < V; ++j)
                    if (i0 + j < d.n) sv.snap[i0 + j] = v[j];
            }
            float s[V][S];
#pragma unroll
            for (int q = 0; q < S; ++q)
#pragma unroll
                for (int j = 0; j < V; ++j) s[j][q] = buf[q * kTile + j0 + j];
            float b[V];
#pragma unroll
            for (int j = 0; j < V; ++j)
                b[j] = v[j] * d.cm +
                       d.dt * Q::div(M::template step<Q>(v[j], s[j], c, T, M::node_g(c, d.node_params, d.n_pad, i0 + j)),
                                     100.0f);
#pragma unroll
            for (int q = 0; q < S; ++q) {
                float t[V];
#pragma unroll
                for (int j = 0; j < V; ++j) t[j] = s[j][q];
                st_nodes<V>(d.state + q * d.n_pad + i0, t);
            }
            if (sv.smask) {
                const uint32_t* bits = reinterpret_cast<const uint32_t*>(buf + (S + 3) * kTile + j0);
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const uint32_t on = bits[j] & sv.smask;
                    if (on) b[j] = b[j] + d.dt * Q::div(stim_sum(d, sv.smask, on), 100.0f);
                }
            }
            st_nodes<V>(d.bp + i0, b);
        }
        __syncthreads();   // every thread is done with this stage
        if (tid == 0 && tile + NS * stride < n_tiles) issue(st, tile + NS * stride);
    }
}

template <class M, int V, int MINB, class Q>
int launch_staged(const MonoDev& d, const typename M::C& c, const typename M::Tables& T, cudaStream_t s) {
    using ST = StagedTile<M, V>;
    static bool configured[64] = {};
    int dev = 0;
    TCB_CHECK_CUDA(cudaGetDevice(&dev));
    if (!configured[dev & 63]) {
        TCB_CHECK_CUDA(cudaFuncSetAttribute(mono_ionic_staged_kernel<M, V, MINB, Q>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ST::kBytes));
        configured[dev & 63] = true;
    }
    const int64_t n_tiles = ceil_div(d.n_pad, ST::kTile);
    const int64_t grid = std::min<int64_t>(n_tiles, (int64_t)num_sms() * MINB);
    mono_ionic_staged_kernel<M, V, MINB, Q><<<(unsigned)grid, kThreads, ST::kBytes, s>>>(d, c, T, n_tiles);
    TCB_CHECK_LAUNCH("mono ionic staged kernel");
    return TCB_OK;
}

template <class M, int V, int MINB, class Q>
int launch_shape(const MonoDev& d, const typename M::C& c, const typename M::Tables& T, cudaStream_t s) {
    mono_ionic_kernel<M, V, MINB, Q><<<grid_for(ceil_div(d.n, V)), kThreads, 0, s>>>(d, c, T);
    TCB_CHECK_LAUNCH("mono ionic kernel");
    return TCB_OK;
}

// The instances of each model: nodes per thread, 256-thread blocks per SM the
// register budget is set for, division/log policy (1 = QFast, 0 = QExact), and
// 1 for the persistent double-buffered form; entry 0 is the default (the fastest
// measured on B200 for million-node cubes: TTP 37.4 us, CRN 22.6 us at 531 k
// nodes, MS 15.4 us).
struct Shape {
    int32_t nodes_per_thread, blocks_per_sm, fast, staged;
};
template <class M>
struct Shapes;
template <>
struct Shapes<MS> {
    static constexpr int kCount = 6;
    static constexpr Shape shape[kCount] = {{4, 8, 0, 0}, {1, 1, 0, 0}, {2, 1, 0, 0},
                                            {4, 4, 0, 0}, {4, 1, 0, 0}, {4, 4, 0, 1}};
    static constexpr LaunchFn<MS> fn[kCount] = {launch_shape<MS, 4, 8, QExact>, launch_shape<MS, 1, 1, QExact>,
                                                launch_shape<MS, 2, 1, QExact>, launch_shape<MS, 4, 4, QExact>,
                                                launch_shape<MS, 4, 1, QExact>, launch_staged<MS, 4, 4, QExact>};
};
template <>
struct Shapes<TTP> {
    static constexpr int kCount = 11;
    static constexpr Shape shape[kCount] = {{1, 3, 1, 1}, {1, 4, 0, 0}, {1, 6, 0, 0}, {2, 3, 0, 0},
                                            {4, 2, 0, 0}, {1, 2, 1, 0}, {1, 3, 1, 0}, {2, 2, 1, 0},
                                            {4, 1, 1, 0}, {2, 2, 1, 1}, {1, 4, 1, 1}};
    static constexpr LaunchFn<TTP> fn[kCount] = {
        launch_staged<TTP, 1, 3, QFast>, launch_shape<TTP, 1, 4, QExact>, launch_shape<TTP, 1, 6, QExact>,
        launch_shape<TTP, 2, 3, QExact>, launch_shape<TTP, 4, 2, QExact>, launch_shape<TTP, 1, 2, QFast>,
        launch_shape<TTP, 1, 3, QFast>,  launch_shape<TTP, 2, 2, QFast>,  launch_shape<TTP, 4, 1, QFast>,
        launch_staged<TTP, 2, 2, QFast>, launch_staged<TTP, 1, 4, QFast>};
};
template <>
struct Shapes<CRN> {
    static constexpr int kCount = 9;
    static constexpr Shape shape[kCount] = {{1, 4, 1, 1}, {2, 2, 1, 0}, {1, 3, 1, 0}, {1, 2, 1, 0}, {4, 1, 1, 0},
                                            {1, 3, 0, 0}, {2, 2, 0, 0}, {2, 2, 1, 1}, {1, 3, 1, 1}};
    static constexpr LaunchFn<CRN> fn[kCount] = {
        launch_staged<CRN, 1, 4, QFast>, launch_shape<CRN, 2, 2, QFast>,  launch_shape<CRN, 1, 3, QFast>,
        launch_shape<CRN, 1, 2, QFast>,  launch_shape<CRN, 4, 1, QFast>,  launch_shape<CRN, 1, 3, QExact>,
        launch_shape<CRN, 2, 2, QExact>, launch_staged<CRN, 2, 2, QFast>, launch_staged<CRN, 1, 3, QFast>};
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
    // vector accesses need the vector's alignment, bulk copies 16 bytes
    const unsigned vb = Shapes<M>::shape[k].staged ? 16u : 4u * (unsigned)Shapes<M>::shape[k].nodes_per_thread;
    if (vb > 4 && !(aligned(d.x, vb) && aligned(d.state, vb) && aligned(d.bp, vb) && aligned(d.at, vb) &&
                    aligned(d.rt, vb) && aligned(d.stim_bits, vb))) {
        k = 0;
        while (Shapes<M>::shape[k].nodes_per_thread != 1 || Shapes<M>::shape[k].staged) ++k;
    }
    return Shapes<M>::fn[k](d, c, T, s);
}

template <class M>
int run_differentiate(const double* params, const float* tables, const float* node_params, float* state,
                      int64_t n_pad, int64_t n, const float* v, float* dv, cudaStream_t s) {
    differentiate_kernel<M><<<grid_for(n), kThreads, 0, s>>>(M::derive(params), M::tables(tables, params),
                                                             node_params, state, n_pad, n, v, dv);
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
                 int32_t* fast, int32_t* staged) {
    *count = Shapes<M>::kCount;
    if (variant < 0 || variant > Shapes<M>::kCount) return fail(TCB_ERANGE, "no such ionic kernel variant");
    const Shape& sh = Shapes<M>::shape[variant > 0 ? variant - 1 : 0];
    *nodes_per_thread = sh.nodes_per_thread;
    *blocks_per_sm = sh.blocks_per_sm;
    *fast = sh.fast;
    *staged = sh.staged;
    return TCB_OK;
}

int launch_mono_finish(const MonoDev& d, cudaStream_t s) {
    mono_finish_kernel<<<grid_for(d.n), kThreads, 0, s>>>(d);
    TCB_CHECK_LAUNCH("mono finish kernel");
    return TCB_OK;
}

}  // namespace tcb

using namespace tcb;

extern "C" int tcb_model_differentiate(int32_t model, const double* params, const float* tables,
                                       const float* node_params, float* state, int64_t n_pad, int64_t n,
                                       const float* v, float* dv, void* stream) {
    if (!params || !state || !v || !dv || n <= 0 || n_pad < n) return fail(TCB_EINVAL, "tcb_model_differentiate: bad arguments");
    if (model != TCB_MODEL_MS && !tables) return fail(TCB_EINVAL, "tcb_model_differentiate: null tables");
    if (model != TCB_MODEL_MS && ((uintptr_t)tables & 15u))
        return fail(TCB_EINVAL, "tcb_model_differentiate: tables not 16-byte aligned");
    cudaStream_t s = as_stream(stream);
    switch (model) {
        case TCB_MODEL_MS: return run_differentiate<MS>(params, tables, node_params, state, n_pad, n, v, dv, s);
        case TCB_MODEL_TTP: return run_differentiate<TTP>(params, tables, node_params, state, n_pad, n, v, dv, s);
        case TCB_MODEL_CRN: return run_differentiate<CRN>(params, tables, node_params, state, n_pad, n, v, dv, s);
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

extern "C" const char* tcb_model_node_params(int32_t model) {
    switch (model) {
        case TCB_MODEL_MS: return "";
        case TCB_MODEL_TTP: return "GCaL,GKr,GKs,Gto";
        case TCB_MODEL_CRN: return "";
    }
    return nullptr;
}

extern "C" int tcb_ionic_variant(int32_t model, int32_t variant, int32_t* count, int32_t* nodes_per_thread,
                                 int32_t* blocks_per_sm, int32_t* fast_math, int32_t* staged) {
    if (!count || !nodes_per_thread || !blocks_per_sm || !fast_math || !staged)
        return fail(TCB_EINVAL, "tcb_ionic_variant: null output");
    switch (model) {
        case TCB_MODEL_MS: return variant_info<MS>(variant, count, nodes_per_thread, blocks_per_sm, fast_math, staged);
        case TCB_MODEL_TTP: return variant_info<TTP>(variant, count, nodes_per_thread, blocks_per_sm, fast_math, staged);
        case TCB_MODEL_CRN: return variant_info<CRN>(variant, count, nodes_per_thread, blocks_per_sm, fast_math, staged);
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}
