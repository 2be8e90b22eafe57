// Batched persistent cooperative CG: every simulation of a batch takes its
// right-hand side, guess and Jacobi-PCG solve (torchcor/core/solver.py:40-76)
// in one launch, with its own alpha, beta, norms, stopping test and iteration
// count (per-simulation convergence masks).
//
// Work split.  Simulations converge after different numbers of iterations, so
// a static split of all slices over the blocks would leave most blocks idle in
// the late passes while a few carry the simulations that still iterate.
// Instead, at the start of every pass each block forms the prefix sum of the
// slice counts of the simulations still active (identical in every block,
// since every block holds the same scalars) and takes its even share of that
// virtual slice space.  A pass therefore costs in proportion to the rows still
// iterating.  Each block's share is contiguous, so neighbouring rows of its
// simulations stay close in L1/L2.
//
// Arithmetic is that of the single-simulation kernels: fused p-update with a
// double-buffered p, float64 row sums and inner products, int16 column offsets
// and A rebuilt from M and K' where the simulation allows.
//
// Reductions are per simulation and deterministic: each lane accumulates its
// rows of one simulation in slice order, a warp reduces its lanes with a fixed
// shuffle tree when its simulation changes, the block adds its warps' values
// in warp order into its partial slot parts[v][sim][block], and after the grid
// barrier every block sums each active simulation's partials over the blocks
// that hold its slices, in block order.  All blocks thus hold identical
// scalars and take identical control-flow decisions.
#include <cuda_runtime.h>
#include <math.h>

#include <type_traits>

#include "l2_hint.cuh"
#include "batch.cuh"
#include "bulk.cuh"
#include "cg_common.cuh"
#include "tcb_internal.h"

namespace tcb {
namespace {

using namespace cgk;
static_assert(sizeof(CgView) % 8 == 0, "CgView is copied as words");
static_assert(kBatchMaxSims <= 2 * kCgThreads, "prefix scan covers two simulations per thread");

// p_new = z + beta p_old in float32 (one rounding, a fused multiply-add with
// beta rounded to float32); every row that forms a given p_new gets the same value
__device__ __forceinline__ float p_update(float z, float p_old, float beta, bool first) {
    return first ? z : __fmaf_rn(beta, p_old, z);
}

// column of ELL entry e of `row`: int16 offset from the row or int32 index.  The
// matrix streams (columns, M, K, A) of a batch are far larger than L2 and read
// once a pass: they are loaded as first to leave L2, ahead of the row vectors the
// neighbour gathers reuse.
template <bool DC>
__device__ __forceinline__ int col_at(const CgView& d, int64_t e, int row) {
    if constexpr (DC) return row + ld_hint_sched(d.dcol + e, l2_once_sched());
    else return ld_hint_sched(d.col + e, l2_once_sched());
}

// Call f with std::integral_constant<int, flags> for the simulation's combination
// of int16 columns (4), A rebuilt from M and K' (2) and linear guess (1): fixed at
// compile time when the whole batch shares one (FLAGS >= 0), else per slice.
template <int FLAGS, class F>
__device__ __forceinline__ void with_flags(const CgView& d, F&& f) {
    if constexpr (FLAGS >= 0) {
        f(std::integral_constant<int, FLAGS>{});
    } else {
        switch ((d.dcol ? 4 : 0) | (d.a_split ? 2 : 0) | (d.linear_guess ? 1 : 0)) {
            case 0: f(std::integral_constant<int, 0>{}); break;
            case 1: f(std::integral_constant<int, 1>{}); break;
            case 2: f(std::integral_constant<int, 2>{}); break;
            case 3: f(std::integral_constant<int, 3>{}); break;
            case 4: f(std::integral_constant<int, 4>{}); break;
            case 5: f(std::integral_constant<int, 5>{}); break;
            case 6: f(std::integral_constant<int, 6>{}); break;
            default: f(std::integral_constant<int, 7>{}); break;
        }
    }
}

// the same for the column format alone (what A p depends on)
template <int FLAGS, class F>
__device__ __forceinline__ void with_dcol(const CgView& d, F&& f) {
    if constexpr (FLAGS >= 0) {
        f(std::integral_constant<bool, (FLAGS & 4) != 0>{});
    } else {
        if (d.dcol) f(std::integral_constant<bool, true>{});
        else f(std::integral_constant<bool, false>{});
    }
}

// Right-hand side, guess, r0 = b - A x0, z0 = D r0 for the 32 rows of slice ls
// (solver.py:46-55, monodomain.py:130-131); adds ||D b||^2 and r0.z0 into acc.
// DC: int16 column offsets; AS: A rebuilt as fp32(fp32(M*Cm) + K'); LG: linear
// extrapolation guess.  Vectors other than x's next slot are read-only here.
template <bool DC, bool AS, bool LG>
__device__ __forceinline__ void rhs_slice(const CgView& d, int step, int64_t ls, int lane, double (&acc)[2]) {
    const int64_t row = ls * TCB_SLICE + lane;
    if (row >= d.n) return;
    const float* __restrict__ u = d.x + ring_cur(step) * d.n_pad;
    const float* __restrict__ xp = d.x + ring_prev(step) * d.n_pad;
    const float* __restrict__ bp = d.bp;
    const int64_t s0 = __ldg(d.slice_ptr + ls);
    const int w = (int)((__ldg(d.slice_ptr + ls + 1) - s0) / TCB_SLICE);
    const int64_t base = s0 + lane;
    const int r = (int)row;
    // M b' and K u accumulate in float32 (the reference's float32 products),
    // A x0 in float64 (the reference's CG is float64; b - A x0 cancels)
    float mb = 0.0f, ku = 0.0f;
    double ax = 0.0;
    // the columns of the next 4-entry chunk are loaded while this chunk's
    // gathers and coefficients are in flight (a column load heads each chain)
    int c[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) c[j] = j < w ? col_at<DC>(d, base + (int64_t)j * TCB_SLICE, r) : r;
    for (int k0 = 0; k0 < w; k0 += 4) {
        float mv[4], kv[4], av[4], bc[4], uc[4], xc[4];
        int cn[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool ok = k0 + j < w;
            const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
            mv[j] = ok ? ld_hint_sched(d.mv + e, l2_once_sched()) : 0.0f;
            kv[j] = ok ? ld_hint_sched(d.kv + e, l2_once_sched()) : 0.0f;
            if constexpr (!AS) av[j] = ok ? ld_hint_sched(d.av + e, l2_once_sched()) : 0.0f;
            bc[j] = __ldg(bp + c[j]);
            uc[j] = __ldg(u + c[j]);
            if constexpr (LG) xc[j] = __ldg(xp + c[j]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool ok = k0 + 4 + j < w;
            cn[j] = ok ? col_at<DC>(d, base + (int64_t)(k0 + 4 + j) * TCB_SLICE, r) : r;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if constexpr (AS) av[j] = __fadd_rn(__fmul_rn(mv[j], d.cm), kv[j]);
            float xg;
            if constexpr (LG) xg = 2.0f * uc[j] - xc[j];
            else xg = uc[j];
            mb = __fmaf_rn(mv[j], bc[j], mb);
            ku = __fmaf_rn(kv[j], uc[j], ku);
            ax += (double)av[j] * (double)xg;
            c[j] = cn[j];
        }
    }
    const float rhs = mb - ku;
    const float ui = __ldg(u + row);
    float xg0;
    if constexpr (LG) xg0 = 2.0f * ui - __ldg(xp + row);
    else xg0 = ui;
    __stwb(d.x + ring_next(step) * d.n_pad + row, xg0);
    const float r32 = (float)((double)rhs - ax);
    const float di = __ldg(d.dinv + row);
    const float z32 = (float)((double)di * (double)r32);
    __stwb(d.r + row, r32);
    __stwb(d.z + row, z32);
    const double db = (double)di * (double)rhs;
    acc[0] += db * db;
    acc[1] += (double)r32 * (double)z32;
}

// p_new = z + beta p_old formed on the fly for every column, Ap for the rows of
// slice ls; writes p_new and Ap of its rows and adds p.Ap into acc.  z and p
// change during the launch, so they are read with plain (L1-allocating)
// global loads, ordered after their writers by the grid barrier.
template <bool DC, bool FIRST>
__device__ __forceinline__ void ap_slice(const CgView& d, const float* pin, float* pout, float beta, int64_t ls,
                                         int lane, double (&acc)[1]) {
    const int64_t row = ls * TCB_SLICE + lane;
    if (row >= d.n) return;
    const int64_t s0 = __ldg(d.slice_ptr + ls);
    const int w = (int)((__ldg(d.slice_ptr + ls + 1) - s0) / TCB_SLICE);
    const int64_t base = s0 + lane;
    const int r = (int)row;
    const float* z = d.z;
    double a = 0.0;
    for (int k0 = 0; k0 < w; k0 += 8) {
        int c[8];
        float av[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const bool ok = k0 + j < w;
            const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
            c[j] = ok ? col_at<DC>(d, e, r) : r;
            av[j] = ok ? ld_hint_sched(d.av + e, l2_once_sched()) : 0.0f;
        }
        float zc[8], pc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            zc[j] = __ldca(z + c[j]);
            pc[j] = FIRST ? 0.0f : __ldca(pin + c[j]);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) a += (double)av[j] * (double)p_update(zc[j], pc[j], beta, FIRST);
    }
    const float pn = p_update(__ldca(z + row), FIRST ? 0.0f : __ldca(pin + row), beta, FIRST);
    __stwb(pout + row, pn);
    const float a32 = (float)a;
    __stwb(d.ap + row, a32);
    acc[0] += (double)pn * (double)a32;
}

// ---------------------------------------------------------------------------
// Staged variant: the sliced-ELL streams (columns and coefficients) of the next
// units are copied into shared memory by bulk asynchronous copies
// (cp.async.bulk, completion counted on an mbarrier) while the warp works on
// the current unit, so only the gathers of neighbour values are exposed to
// memory latency.  A unit is up to 16 entries of one 32-row slice: in every
// ELL array its entries are one contiguous block (column-major slices).
constexpr int kStages = 2;             // units in flight per warp
constexpr int kMaxUnitEntries = 16;

// warp-uniform wait for a stage's copies; gives up after the timeout (error
// word set) so a lost copy can never hang the kernel
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t* err, const WaitLimit& w) {
    if (__all_sync(0xffffffffu, mbar_test(bar, parity))) return true;
    const uint64_t t0 = globaltimer();
    while (!__all_sync(0xffffffffu, mbar_test(bar, parity))) {
        if (globaltimer() - t0 > w.timeout_ns) {
            if ((threadIdx.x & 31) == 0) atomicCAS(err, 0, TCB_ETIMEOUT);
            return false;
        }
    }
    return true;
}

struct Pipe {
    unsigned char* buf;   // this warp's kStages buffers of stage_bytes
    uint64_t* bar;        // their mbarriers
    uint32_t phase;       // bit s: parity of stage s's next completion
    uint32_t inflight;    // bit s: stage s has copies issued and not yet waited for
    uint32_t drop;        // test hook: skip the copy of the next issue (its bytes never arrive)
    int stage_bytes;
};

// After a timed-out wait: give every stage with issued copies a bounded wait of
// its own, so that no bulk copy still writes this warp's buffers when the block
// returns.
__device__ __forceinline__ void drain(Pipe& P, int32_t* err, const WaitLimit& w) {
    for (int s = 0; s < kStages; ++s)
        if ((P.inflight >> s) & 1u) {
            mbar_wait(P.bar + s, (P.phase >> s) & 1u, err, w);
            P.inflight &= ~(1u << s);
        }
}

struct Row {
    double v[3];   // per-row partial sums carried across a slice's units
};

// what a phase streams: columns, then its coefficient arrays
struct RhsStreams {
    __device__ static int entry_bytes(const CgView& d) { return (d.dcol ? 2 : 4) + 8 + (d.a_split ? 0 : 4); }
    __device__ static void copy(const CgView& d, int64_t e0, int nk, unsigned char* dst, uint64_t* bar) {
        const uint32_t m = (uint32_t)nk * TCB_SLICE;
        if (d.dcol) {
            bulk_load(dst, d.dcol + e0, m * 2, bar);
            dst += m * 2;
        } else {
            bulk_load(dst, d.col + e0, m * 4, bar);
            dst += m * 4;
        }
        bulk_load(dst, d.mv + e0, m * 4, bar);
        bulk_load(dst + m * 4, d.kv + e0, m * 4, bar);
        if (!d.a_split) bulk_load(dst + m * 8, d.av + e0, m * 4, bar);
    }
};

struct ApStreams {
    __device__ static int entry_bytes(const CgView& d) { return (d.dcol ? 2 : 4) + 4; }
    __device__ static void copy(const CgView& d, int64_t e0, int nk, unsigned char* dst, uint64_t* bar) {
        const uint32_t m = (uint32_t)nk * TCB_SLICE;
        if (d.dcol) {
            bulk_load(dst, d.dcol + e0, m * 2, bar);
            dst += m * 2;
        } else {
            bulk_load(dst, d.col + e0, m * 4, bar);
            dst += m * 4;
        }
        bulk_load(dst, d.av + e0, m * 4, bar);
    }
};

struct BatchShared {
    double *rz, *bn, *al, *be;   // [n] per simulation
    double* wp;                  // [warps][kBatchMaxPerBlock][2] warp partials of the staged simulations
    int64_t* pre;                // [n+1] prefix of the active simulations' slice counts
    int64_t* bb;                 // [nb+1] first virtual slice of each block
    CgView* cg;                  // [kBatchMaxPerBlock] staged views
    int *it, *act, *step, *ns;   // [n]
    int *w0, *w1;                // [n] first and last block holding each active simulation's slices
};

__device__ __forceinline__ BatchShared carve(double* smd, int n, int nb) {
    BatchShared s;
    s.rz = smd;
    s.bn = s.rz + n;
    s.al = s.bn + n;
    s.be = s.al + n;
    s.wp = s.be + n;
    s.pre = reinterpret_cast<int64_t*>(s.wp + kCgWarps * kBatchMaxPerBlock * 2);
    s.bb = s.pre + n + 1;
    s.cg = reinterpret_cast<CgView*>(s.bb + nb + 1);
    s.it = reinterpret_cast<int*>(s.cg + kBatchMaxPerBlock);
    s.act = s.it + n;
    s.step = s.act + n;
    s.ns = s.step + n;
    s.w0 = s.ns + n;
    s.w1 = s.w0 + n;
    return s;
}

// the block whose range [b*A/nb, (b+1)*A/nb) holds virtual slice x
__device__ __forceinline__ int block_of(int64_t x, int64_t A, int nb) {
    const int64_t b = ((x + 1) * nb - 1) / A;
    return b < nb - 1 ? (int)b : nb - 1;
}

// Exclusive prefix of the slice counts of the simulations with flag[i] != 0
// into S.pre[0..n], the block boundaries of its even split into S.bb and each
// simulation's block window into S.w0/S.w1; returns the total.  Every block
// computes the same.
__device__ int64_t active_prefix(BatchShared& S, int n, const int* flag) {
    __shared__ int64_t wt[kCgWarps];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int e0 = 2 * t, e1 = 2 * t + 1;
    const int64_t v0 = (e0 < n && flag[e0]) ? (int64_t)S.ns[e0] : 0;
    const int64_t v1 = (e1 < n && flag[e1]) ? (int64_t)S.ns[e1] : 0;
    int64_t s = v0 + v1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
    }
    __syncthreads();   // earlier readers of pre and wt are done
    if (lane == 31) wt[warp] = s;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < kCgWarps ? wt[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kCgWarps) wt[lane] = w;
    }
    __syncthreads();
    const int64_t base = (warp ? wt[warp - 1] : 0) + s - v0 - v1;
    if (e0 < n) S.pre[e0] = base;
    if (e1 < n) S.pre[e1] = base + v0;
    const int64_t total = wt[kCgWarps - 1];
    if (t == 0) S.pre[n] = total;
    // the even split of the total over the blocks, and each simulation's blocks
    const int nb = gridDim.x;
    for (int b = t; b <= nb; b += blockDim.x) S.bb[b] = (int64_t)b * total / nb;
    __syncthreads();
    for (int i = t; i < n; i += blockDim.x) {
        const int64_t P = S.pre[i], cnt = S.pre[i + 1] - P;
        S.w0[i] = cnt ? block_of(P, total, nb) : 0;
        S.w1[i] = cnt ? block_of(P + cnt - 1, total, nb) : -1;
    }
    __syncthreads();
    return total;
}

// largest i in [0, n) with pre[i] <= x (the active simulation holding virtual slice x)
__device__ __forceinline__ int sim_of(const int64_t* pre, int n, int64_t x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= x) lo = mid; else hi = mid - 1;
    }
    return lo;
}


// reduce the lanes' NV values and add them to this warp's slot of staged simulation j
template <int NV>
__device__ __forceinline__ void flush(BatchShared& S, int warp, int lane, int j, double (&acc)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double t = warp_sum(acc[v]);
        if (lane == 0) S.wp[(warp * kBatchMaxPerBlock + j) * 2 + v] += t;
        acc[v] = 0.0;
    }
}

// One sweep over this block's share of the active slices: body(i, view, local
// slice, acc) adds each lane's row into acc; the block's per-simulation sums go
// to parts[v][i][block].
template <int NV, class Body>
__device__ __forceinline__ void sweep(const BatchWS* W, BatchShared& S, double* parts, Body&& body) {
    const int nb = gridDim.x, b = blockIdx.x, n = W->n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t vb = S.bb[b], ve = S.bb[b + 1];
    if (vb >= ve) return;
    const int first = sim_of(S.pre, n, vb), last = sim_of(S.pre, n, ve - 1);
    for (int j0 = first; j0 <= last; j0 += kBatchMaxPerBlock) {
        const int j1 = min(last + 1, j0 + kBatchMaxPerBlock);
        __syncthreads();   // earlier users of the staged views and slots are done
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(W->cg + j0);
            uint32_t* dst = reinterpret_cast<uint32_t*>(S.cg);
            const int words = (j1 - j0) * (int)(sizeof(CgView) / 4);
            for (int t = threadIdx.x; t < words; t += blockDim.x) dst[t] = src[t];
            for (int t = threadIdx.x; t < kCgWarps * kBatchMaxPerBlock * 2; t += blockDim.x) S.wp[t] = 0.0;
        }
        __syncthreads();
        const int64_t sb = max(vb, S.pre[j0]), se = min(ve, S.pre[j1]);
        double acc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = 0.0;
        int i = j0, ci = -1;
        for (int64_t vs = sb + warp; vs < se; vs += kCgWarps) {
            while (S.pre[i + 1] <= vs) ++i;
            if (i != ci) {
                if (ci >= 0) flush<NV>(S, warp, lane, ci - j0, acc);
                ci = i;
            }
            body(i, S.cg[i - j0], vs - S.pre[i], acc);
        }
        if (ci >= 0) flush<NV>(S, warp, lane, ci - j0, acc);
        __syncthreads();
        for (int j = threadIdx.x; j < j1 - j0; j += blockDim.x) {
            const int i2 = j0 + j;
            if (S.pre[i2 + 1] == S.pre[i2]) continue;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double t = 0.0;
                for (int w = 0; w < kCgWarps; ++w) t += S.wp[(w * kBatchMaxPerBlock + j) * 2 + v];
                parts[((size_t)v * n + i2) * nb + b] = t;
            }
        }
    }
}

// A warp's walk over the units of its slices vs = start, start+16, ... < se
// (all values warp-uniform).
template <class Streams>
struct Walk {
    int64_t vs, se, ls, s0;
    int i, w, k0, nk;
    bool ok;
    __device__ void load(const BatchShared& S, int j0, int stage_bytes) {
        ok = vs < se;
        if (!ok) return;
        while (S.pre[i + 1] <= vs) ++i;
        const CgView& d = S.cg[i - j0];
        ls = vs - S.pre[i];
        s0 = __ldg(d.slice_ptr + ls);
        w = (int)((__ldg(d.slice_ptr + ls + 1) - s0) / TCB_SLICE);
        const int fit = stage_bytes / (TCB_SLICE * Streams::entry_bytes(d));
        nk = fit < kMaxUnitEntries ? fit : kMaxUnitEntries;
        k0 = 0;
    }
    __device__ void next(const BatchShared& S, int j0, int stage_bytes) {
        k0 += nk;
        if (k0 >= w) {
            vs += kCgWarps;
            load(S, j0, stage_bytes);
        }
    }
    __device__ int count() const { return nk < w - k0 ? nk : w - k0; }
};

template <class Streams>
__device__ __forceinline__ void issue(Pipe& P, int s, const CgView& d, const Walk<Streams>& u, int lane) {
    if (lane == 0) {
        const int nk = u.count();
        // order this warp's earlier shared-memory reads of the stage before the async writes
        fence_proxy_async_smem();
        mbar_arrive_tx(P.bar + s, (uint32_t)(nk * TCB_SLICE * Streams::entry_bytes(d)));
        if (!P.drop)
            Streams::copy(d, u.s0 + (int64_t)u.k0 * TCB_SLICE, nk, P.buf + (size_t)s * P.stage_bytes, P.bar + s);
    }
    P.drop = 0;
    P.inflight |= 1u << s;
}

// sweep() with the ELL streams staged: unit(i, view, ls, nk, stage buffer, row)
// accumulates one unit into the row's partial sums, end(i, view, ls, row, acc)
// finishes a row after its slice's last unit.  Returns false after a timed-out
// wait (the error word is set; the caller's next grid barrier ends the kernel).
template <int NV, class Streams, class Unit, class End>
__device__ __forceinline__ bool sweep_staged(const BatchWS* W, BatchShared& S, double* parts, Pipe& P,
                                             int32_t* err, Unit&& unit, End&& end) {
    const int nb = gridDim.x, b = blockIdx.x, n = W->n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t vb = S.bb[b], ve = S.bb[b + 1];
    if (vb >= ve) return true;
    bool good = true;
    const int first = sim_of(S.pre, n, vb), last = sim_of(S.pre, n, ve - 1);
    for (int j0 = first; j0 <= last; j0 += kBatchMaxPerBlock) {
        const int j1 = min(last + 1, j0 + kBatchMaxPerBlock);
        __syncthreads();   // earlier users of the staged views and slots are done
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(W->cg + j0);
            uint32_t* dst = reinterpret_cast<uint32_t*>(S.cg);
            const int words = (j1 - j0) * (int)(sizeof(CgView) / 4);
            for (int t = threadIdx.x; t < words; t += blockDim.x) dst[t] = src[t];
            for (int t = threadIdx.x; t < kCgWarps * kBatchMaxPerBlock * 2; t += blockDim.x) S.wp[t] = 0.0;
        }
        __syncthreads();
        Walk<Streams> cons;
        cons.vs = max(vb, S.pre[j0]) + warp;
        cons.se = min(ve, S.pre[j1]);
        cons.i = j0;
        cons.load(S, j0, P.stage_bytes);
        Walk<Streams> prod = cons;
        for (int st = 0; st < kStages && prod.ok; ++st) {
            issue(P, st, S.cg[prod.i - j0], prod, lane);
            prod.next(S, j0, P.stage_bytes);
        }
        double acc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = 0.0;
        Row rw = {};
        int ci = -1;
        for (int u = 0; cons.ok && good; ++u) {
            const int st = u % kStages;
            if (!mbar_wait(P.bar + st, (P.phase >> st) & 1u, err, W->wait)) {
                drain(P, err, W->wait);
                good = false;
                break;
            }
            P.inflight &= ~(1u << st);
            P.phase ^= 1u << st;
            const CgView& d = S.cg[cons.i - j0];
            if (cons.i != ci) {
                if (ci >= 0) flush<NV>(S, warp, lane, ci - j0, acc);
                ci = cons.i;
            }
            if (cons.k0 == 0) rw = Row{};
            const int cnt = cons.count();
            unit(cons.i, d, cons.ls, cnt, P.buf + (size_t)st * P.stage_bytes, rw);
            if (cons.k0 + cnt >= cons.w) end(cons.i, d, cons.ls, rw, acc);
            __syncwarp();   // every lane is done with this stage's buffer
            if (prod.ok) {
                issue(P, st, S.cg[prod.i - j0], prod, lane);
                prod.next(S, j0, P.stage_bytes);
            }
            cons.next(S, j0, P.stage_bytes);
        }
        if (ci >= 0) flush<NV>(S, warp, lane, ci - j0, acc);
        __syncthreads();
        for (int j = threadIdx.x; j < j1 - j0; j += blockDim.x) {
            const int i2 = j0 + j;
            if (S.pre[i2 + 1] == S.pre[i2]) continue;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double t = 0.0;
                for (int w = 0; w < kCgWarps; ++w) t += S.wp[(w * kBatchMaxPerBlock + j) * 2 + v];
                parts[((size_t)v * n + i2) * nb + b] = t;
            }
        }
    }
    return good;
}

// one staged unit of the right-hand side (entries in slice order, the same
// float64 accumulation sequence as rhs_slice)
template <bool DC, bool AS, bool LG>
__device__ __forceinline__ void rhs_unit(const CgView& d, int step, int64_t ls, int nk, const unsigned char* buf,
                                         Row& rw, int lane) {
    const int64_t row = ls * TCB_SLICE + lane;
    if (row >= d.n) return;
    const int r = (int)row;
    const float* __restrict__ u = d.x + ring_cur(step) * d.n_pad;
    const float* __restrict__ xp = d.x + ring_prev(step) * d.n_pad;
    const float* __restrict__ bp = d.bp;
    const int m = nk * TCB_SLICE;
    const int16_t* c16 = reinterpret_cast<const int16_t*>(buf);
    const int32_t* c32 = reinterpret_cast<const int32_t*>(buf);
    const float* mvs = reinterpret_cast<const float*>(buf + m * (DC ? 2 : 4));
    const float* kvs = mvs + m;
    const float* avs = kvs + m;
    float mb = (float)rw.v[0], ku = (float)rw.v[1];
    double ax = rw.v[2];
    for (int k = 0; k < nk; k += 8) {
        int c[8];
        float mv[8], kv[8], av[8], bc[8], uc[8], xc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const bool ok = k + j < nk;
            const int e = (k + j) * TCB_SLICE + lane;
            if constexpr (DC) c[j] = ok ? r + (int)c16[e] : r;
            else c[j] = ok ? c32[e] : r;
            mv[j] = ok ? mvs[e] : 0.0f;
            kv[j] = ok ? kvs[e] : 0.0f;
            if constexpr (AS) av[j] = __fadd_rn(__fmul_rn(mv[j], d.cm), kv[j]);
            else av[j] = ok ? avs[e] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            bc[j] = __ldg(bp + c[j]);
            uc[j] = __ldg(u + c[j]);
            if constexpr (LG) xc[j] = __ldg(xp + c[j]);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (k + j < nk) {
                float xg;
                if constexpr (LG) xg = 2.0f * uc[j] - xc[j];
                else xg = uc[j];
                mb = __fmaf_rn(mv[j], bc[j], mb);
                ku = __fmaf_rn(kv[j], uc[j], ku);
                ax += (double)av[j] * (double)xg;
            }
        }
    }
    rw.v[0] = mb;
    rw.v[1] = ku;
    rw.v[2] = ax;
}

// the end of a right-hand-side row (as the tail of rhs_slice)
__device__ __forceinline__ void rhs_end(const CgView& d, int step, int64_t ls, const Row& rw, double (&acc)[2],
                                        int lane) {
    const int64_t row = ls * TCB_SLICE + lane;
    if (row >= d.n) return;
    const float* __restrict__ u = d.x + ring_cur(step) * d.n_pad;
    const float rhs = (float)rw.v[0] - (float)rw.v[1];   // float32 sums carried in the row state
    const float ui = __ldg(u + row);
    const float xg0 = d.linear_guess ? 2.0f * ui - __ldg(d.x + ring_prev(step) * d.n_pad + row) : ui;
    __stwb(d.x + ring_next(step) * d.n_pad + row, xg0);
    const float r32 = (float)((double)rhs - rw.v[2]);
    const float di = __ldg(d.dinv + row);
    const float z32 = (float)((double)di * (double)r32);
    __stwb(d.r + row, r32);
    __stwb(d.z + row, z32);
    const double db = (double)di * (double)rhs;
    acc[0] += db * db;
    acc[1] += (double)r32 * (double)z32;
}

// one staged unit of A p (p formed on the fly from the gathered z and old p)
template <bool DC, bool FIRST>
__device__ __forceinline__ void ap_unit(const CgView& d, const float* pin, float beta, int64_t ls, int nk,
                                        const unsigned char* buf, Row& rw, int lane) {
    const int64_t row = ls * TCB_SLICE + lane;
    if (row >= d.n) return;
    const int r = (int)row;
    const int m = nk * TCB_SLICE;
    const int16_t* c16 = reinterpret_cast<const int16_t*>(buf);
    const int32_t* c32 = reinterpret_cast<const int32_t*>(buf);
    const float* avs = reinterpret_cast<const float*>(buf + m * (DC ? 2 : 4));
    const float* z = d.z;
    double a = rw.v[0];
    for (int k = 0; k < nk; k += 8) {
        int c[8];
        float av[8], zc[8], pc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const bool ok = k + j < nk;
            const int e = (k + j) * TCB_SLICE + lane;
            if constexpr (DC) c[j] = ok ? r + (int)c16[e] : r;
            else c[j] = ok ? c32[e] : r;
            av[j] = ok ? avs[e] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            zc[j] = __ldca(z + c[j]);
            pc[j] = FIRST ? 0.0f : __ldca(pin + c[j]);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (k + j < nk) a += (double)av[j] * (double)p_update(zc[j], pc[j], beta, FIRST);
    }
    rw.v[0] = a;
}

__device__ __forceinline__ void ap_end(const CgView& d, const float* pin, float* pout, float beta, bool first,
                                       int64_t ls, const Row& rw, double (&acc)[1], int lane) {
    const int64_t row = ls * TCB_SLICE + lane;
    if (row >= d.n) return;
    const float pn = p_update(__ldca(d.z + row), first ? 0.0f : __ldca(pin + row), beta, first);
    __stwb(pout + row, pn);
    const float a32 = (float)rw.v[0];
    __stwb(d.ap + row, a32);
    acc[0] += (double)pn * (double)a32;
}

// every block: totals of every active simulation (warp per simulation, lanes over its blocks)
template <int NV, class F>
__device__ __forceinline__ void totals(const BatchWS* W, BatchShared& S, const double* parts, F&& consume) {
    const int nb = gridDim.x, n = W->n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < n; i += kCgWarps) {
        const int b0 = S.w0[i], b1 = S.w1[i];
        if (b1 < b0) continue;   // not active
        double acc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = 0.0;
        for (int bb = b0 + lane; bb <= b1; bb += 32) {
            if (S.bb[bb] == S.bb[bb + 1]) continue;   // empty block
#pragma unroll
            for (int v = 0; v < NV; ++v) acc[v] += __ldcg(parts + ((size_t)v * n + i) * nb + bb);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = warp_sum(acc[v]);
        if (lane == 0) consume(i, acc);
    }
    __syncthreads();
}

// bytes of the shared carve-out before the staging area (128-byte aligned)
__host__ __device__ inline size_t carve_bytes(int n) {
    const size_t b = (size_t)n * (4 * sizeof(double) + 6 * sizeof(int)) +
                     sizeof(double) * kCgWarps * kBatchMaxPerBlock * 2 + sizeof(int64_t) * (n + 1) +
                     sizeof(int64_t) * (kBatchMaxBlocks + 1) + sizeof(CgView) * kBatchMaxPerBlock;
    return (b + 127) / 128 * 128;
}
constexpr size_t kStageBarBytes = 128 * ((kCgWarps * kStages * 8 + 127) / 128);

// PER_SM: blocks per SM the register budget is sized for (1: 128 registers a
// thread, no spills; 2: 64 registers, twice the warps to hide latency).
// STAGED: the right-hand side and A p stream their ELL blocks through shared
// memory by bulk copies (stage_bytes per warp and stage; 1 block per SM).
// FLAGS: the (int16 columns, A rebuilt, linear guess) combination every
// simulation of the batch shares (0..7: specialised code, fewer registers), or -1
// (chosen per slice).
template <int PER_SM, bool STAGED, int FLAGS>
__global__ void __launch_bounds__(kCgThreads, PER_SM) batch_cg_kernel(const BatchWS* __restrict__ W,
                                                                       int stage_bytes) {
    extern __shared__ __align__(128) double smd[];
    const int n = W->n;
    BatchShared S = carve(smd, n, gridDim.x);
    const int lane = threadIdx.x & 31;
    double* parts0 = W->parts;
    double* parts1 = W->parts + 2 * (size_t)n * gridDim.x;
    int32_t* err = W->err;
    Pipe P = {};
    if constexpr (STAGED) {
        unsigned char* base = reinterpret_cast<unsigned char*>(smd) + carve_bytes(n);
        const int warp = threadIdx.x >> 5;
        P.bar = reinterpret_cast<uint64_t*>(base) + warp * kStages;
        P.buf = base + kStageBarBytes + (size_t)warp * kStages * stage_bytes;
        P.stage_bytes = stage_bytes;
        P.phase = 0;
        P.inflight = 0;
        P.drop = (W->wait.drop_first_copy && blockIdx.x == 0 && warp == 0) ? 1u : 0u;
        if (lane == 0) {
            for (int st = 0; st < kStages; ++st) mbar_init(P.bar + st);
            mbar_init_fence();
        }
        __syncwarp();
    }

    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int64_t st = W->dev[i].counter[0];
        S.step[i] = (st >= 1 && st <= W->dev[i].nt) ? (int)st : 0;   // 0 = not stepping
        S.ns[i] = W->slices[i];
        S.act[i] = 0;
        S.it[i] = 0;
    }
    __syncthreads();

    // ---- right-hand side, guess, r0, z0 (solver.py:46-55; monodomain.py:130-131)
    int64_t A = active_prefix(S, n, S.step);
    if constexpr (STAGED) {
        sweep_staged<2, RhsStreams>(
            W, S, parts0, P, err,
            [&](int i, const CgView& d, int64_t ls, int nk, const unsigned char* buf, Row& rw) {
                const int step = S.step[i];
                with_flags<FLAGS>(d, [&](auto fl) {
                    constexpr int F = decltype(fl)::value;
                    rhs_unit<(F & 4) != 0, (F & 2) != 0, (F & 1) != 0>(d, step, ls, nk, buf, rw, lane);
                });
            },
            [&](int i, const CgView& d, int64_t ls, const Row& rw, double (&acc)[2]) {
                rhs_end(d, S.step[i], ls, rw, acc, lane);
            });
    } else
    sweep<2>(W, S, parts0, [&](int i, const CgView& d, int64_t ls, double (&acc)[2]) {
        const int step = S.step[i];
        with_flags<FLAGS>(d, [&](auto fl) {
            constexpr int F = decltype(fl)::value;
            rhs_slice<(F & 4) != 0, (F & 2) != 0, (F & 1) != 0>(d, step, ls, lane, acc);
        });
    });
    if (!grid_barrier(W->bar, err, W->wait)) return;
    totals<2>(W, S, parts0, [&](int i, double* t) {
        S.bn[i] = sqrt(t[0]);
        S.rz[i] = t[1];
        S.be[i] = 0.0;
        S.act[i] = W->dev[i].max_iter > 0;
    });

    for (int pass = 0;; ++pass) {
        A = active_prefix(S, n, S.act);
        if (A == 0) break;
        const bool first_pass = pass == 0;
        // ---- p = z + beta p (on the fly), Ap, p.Ap
        if constexpr (STAGED) {
            sweep_staged<1, ApStreams>(
                W, S, parts1, P, err,
                [&](int i, const CgView& d, int64_t ls, int nk, const unsigned char* buf, Row& rw) {
                    const float* pin = (pass & 1) ? d.p2 : d.p;
                    const float beta = (float)S.be[i];
                    with_dcol<FLAGS>(d, [&](auto dc) {
                        constexpr bool DC = decltype(dc)::value;
                        if (first_pass) ap_unit<DC, true>(d, pin, beta, ls, nk, buf, rw, lane);
                        else ap_unit<DC, false>(d, pin, beta, ls, nk, buf, rw, lane);
                    });
                },
                [&](int i, const CgView& d, int64_t ls, const Row& rw, double (&acc)[1]) {
                    ap_end(d, (pass & 1) ? d.p2 : d.p, (pass & 1) ? d.p : d.p2, (float)S.be[i], first_pass, ls, rw, acc,
                           lane);
                });
        } else
        sweep<1>(W, S, parts1, [&](int i, const CgView& d, int64_t ls, double (&acc)[1]) {
            const float* pin = (pass & 1) ? d.p2 : d.p;
            float* pout = (pass & 1) ? d.p : d.p2;
            const float beta = (float)S.be[i];
            with_dcol<FLAGS>(d, [&](auto dc) {
                constexpr bool DC = decltype(dc)::value;
                if (first_pass) ap_slice<DC, true>(d, pin, pout, beta, ls, lane, acc);
                else ap_slice<DC, false>(d, pin, pout, beta, ls, lane, acc);
            });
        });
        if (!grid_barrier(W->bar, err, W->wait)) return;
        totals<1>(W, S, parts1, [&](int i, double* t) { S.al[i] = S.rz[i] / t[0]; });

        // ---- x += alpha p, r -= alpha Ap, z = D r; ||z||^2, r.z
        sweep<2>(W, S, parts0, [&](int i, const CgView& d, int64_t ls, double (&acc)[2]) {
            const int64_t row = ls * TCB_SLICE + lane;
            if (row >= d.n) return;
            const float* pnew = (pass & 1) ? d.p : d.p2;
            const double alpha = S.al[i];
            float* x = d.x + ring_next(S.step[i]) * d.n_pad;
            __stwb(x + row, (float)((double)__ldca(x + row) + alpha * (double)__ldca(pnew + row)));
            const float r32 = (float)((double)__ldca(d.r + row) - alpha * (double)__ldca(d.ap + row));
            __stwb(d.r + row, r32);
            const float z32 = (float)((double)__ldg(d.dinv + row) * (double)r32);
            __stwb(d.z + row, z32);
            acc[0] += (double)z32 * (double)z32;
            acc[1] += (double)r32 * (double)z32;
        });
        if (!grid_barrier(W->bar, err, W->wait)) return;
        totals<2>(W, S, parts0, [&](int i, double* t) {
            const MonoDev& d = W->dev[i];
            const double zn = sqrt(t[0]);
            if (zn < d.a_tol || (zn / S.bn[i]) < d.r_tol) {   // solver.py:66-69
                S.act[i] = 0;
                return;
            }
            S.be[i] = t[1] / S.rz[i];
            S.rz[i] = t[1];
            S.it[i] += 1;
            if (S.it[i] >= d.max_iter) S.act[i] = 0;
        });
    }
    // block 0 records the iterations and advances the step counters (every
    // block read the counters before the first grid barrier)
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            if (S.step[i]) {
                W->dev[i].step_iters[S.step[i]] = S.it[i];
                W->dev[i].counter[0] = S.step[i] + 1;
            }
}

}  // namespace

size_t batch_cg_smem(int n) { return carve_bytes(n); }

namespace {

using KernelFn = void (*)(const BatchWS*, int);

// the kernel of a variant (1, 2: streaming; 3: staged) and flag combination
// (-1 or 0..7); the streaming variants have a specialisation per combination
template <int PER_SM, bool STAGED>
KernelFn pick(int flags) {
    if constexpr (STAGED) {
        return batch_cg_kernel<PER_SM, STAGED, -1>;
    } else {
        switch (flags) {
            case 0: return batch_cg_kernel<PER_SM, false, 0>;
            case 1: return batch_cg_kernel<PER_SM, false, 1>;
            case 2: return batch_cg_kernel<PER_SM, false, 2>;
            case 3: return batch_cg_kernel<PER_SM, false, 3>;
            case 4: return batch_cg_kernel<PER_SM, false, 4>;
            case 5: return batch_cg_kernel<PER_SM, false, 5>;
            case 6: return batch_cg_kernel<PER_SM, false, 6>;
            case 7: return batch_cg_kernel<PER_SM, false, 7>;
        }
        return batch_cg_kernel<PER_SM, false, -1>;
    }
}

KernelFn kernel_of(int variant, int flags) {
    switch (variant) {
        case 1: return pick<1, false>(flags);
        case 2: return pick<2, false>(flags);
        case 3: return pick<1, true>(flags);
    }
    return nullptr;
}

}  // namespace

// Staging bytes per warp and stage for n simulations (0 if the staged variant
// does not fit): as much as shared memory allows, at most 8 KB, in whole KB.
int batch_cg_stage_bytes(int n) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const long avail = (long)optin - (long)carve_bytes(n) - (long)kStageBarBytes - 1024;
    long per = avail / (kCgWarps * kStages) / 1024 * 1024;
    if (per > 8192) per = 8192;
    return per >= 2048 ? (int)per : 0;
}

size_t batch_cg_smem_variant(int n, int variant) {
    if (variant != 3) return carve_bytes(n);
    return carve_bytes(n) + kStageBarBytes + (size_t)kCgWarps * kStages * batch_cg_stage_bytes(n);
}

// Blocks of `variant` that fit with `smem` bytes of shared memory (0 if none);
// also sets the shared-memory attribute of the kernel the plan will launch.
int batch_cg_max_blocks(size_t smem, int variant, int flags) {
    const KernelFn k = kernel_of(variant, flags);
    if (!k) return 0;
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kCgThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const int per_sm = variant == 2 ? 2 : 1;
    if (occ > per_sm) occ = per_sm;
    const int cap = sms * occ;
    return cap > kBatchMaxBlocks ? kBatchMaxBlocks : cap;
}

int launch_batch_cg(const BatchWS* ws_dev, int nb, size_t smem, int variant, int stage_bytes, int flags,
                    cudaStream_t s) {
    const KernelFn k = kernel_of(variant, flags);
    if (!k) return fail(TCB_EINVAL, "unknown batched CG variant");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nb);
    cfg.blockDim = dim3(kCgThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TCB_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k, ws_dev, variant == 3 ? stage_bytes : 0));
    return TCB_OK;
}

}  // namespace tcb
