// Persistent cooperative CG with the block's own rows resident in shared
// memory for the whole solve (the variant used whenever they fit).
//
// Same mathematics as cg_kernel in cg.cu (right-hand side, linear
// extrapolation guess, Jacobi-PCG of torchcor/core/solver.py:40-76 with the
// stopping test on the device), organised for the B200 memory system:
//  * x, r, z, p, Ap and 1/diag of a block's rows live in shared memory
//    (24 B per row); only z and p, which neighbouring rows read, go to global
//    memory (L2-resident), and x once at the end;
//  * the search-direction update p = z + beta*p (float32 fused multiply-add) is formed on the fly inside
//    the matrix-vector product from the gathered z and previous p (the global
//    p is double-buffered), so a CG iteration has two grid barriers (after
//    p.Ap and after the ||z||, r.z reductions) instead of three;
//  * sliced-ELL rows are walked in predicated chunks of 4 (right-hand side) and
//    8 (A p) entries so every lane keeps a batch of independent loads in flight;
//  * column indices are read either as int32 or as int16 offsets from the row
//    (2 bytes per non-zero) when every |col - row| < 32768.
//  * the right-hand side phase does not stream A when the assembly verified that
//    every A value equals fp32(fp32(M*Cm) + K') bit for bit (true for theta =
//    0.5, the reference's value): the coefficient is rebuilt from M and K';
//  * the column offsets are loaded as L2 evict-last, M, K and A as evict-first
//    (l2_hint.cuh), so the offsets stay in L2 from the right-hand side through
//    every A p pass; marking A evict-last as well (61 MB more on a million-node
//    cube) pushed the offsets and row vectors out and cost 10 % a launch;
//  * z and p of neighbouring rows are read through L1 after the grid barrier
//    (whose gpu-scope fences order them after the writers' stores).
// All float32 values that neighbours see (z, p) are rounded once and every row
// derives p from the same float32 inputs, so the vector the matrix multiplies
// is one consistent vector.
//
// The fused step (ION = WithIonic<Model, Policy>): the same kernel first runs
// the ionic update of the block's own rows (ionic_node: AT/RT and snapshot of
// the previous step, state update, stimulus, b') and, in the same pass over the
// rows, the parts of the right-hand side that do not need b' (K u in float32,
// A x0 in float64, kept per row in shared memory); one grid barrier publishes
// b', and the second pass forms M b' and r0, z0.  The issue-bound ionic
// arithmetic of some warps overlaps the neighbour gathers of others, and the
// separate ionic launch disappears; the values are those of the two-kernel step
// bit for bit (same sums in the same order).
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cstdlib>

#include "cg_common.cuh"
#include "ionic_crn.cuh"
#include "ionic_ms.cuh"
#include "ionic_node.cuh"
#include "ionic_ttp.cuh"
#include "l2_hint.cuh"
#include "mono.cuh"
#include "tcb_internal.h"

namespace tcb {
namespace {

using namespace cgk;

template <typename IDX>
__device__ __forceinline__ int col_at(const IDX* __restrict__ col, int64_t e, int64_t row, uint64_t pol);
template <>
__device__ __forceinline__ int col_at<int32_t>(const int32_t* __restrict__ col, int64_t e, int64_t, uint64_t pol) {
    return ld_hint(col + e, pol);
}
template <>
__device__ __forceinline__ int col_at<int16_t>(const int16_t* __restrict__ col, int64_t e, int64_t row,
                                               uint64_t pol) {
    return (int)row + ld_hint(col + e, pol);
}

// p_new = z + beta * p_old in float32 (one fused multiply-add, beta rounded to
// float32): the same result for every row that forms it
__device__ __forceinline__ float p_update(float z, float p_old, float beta, bool first) {
    return first ? z : __fmaf_rn(beta, p_old, z);
}

// What the kernel runs before the right-hand side: nothing (the CG of a step
// whose ionic update ran as its own launch) or the model's ionic update.
struct NoIonic {
    static constexpr bool kFused = false;
};
template <class M, class Q>
struct WithIonic {
    static constexpr bool kFused = true;
    using Model = M;
    using Policy = Q;
    typename M::C c;
    typename M::Tables T;
};

template <typename IDX, int MINB, bool ASPLIT, class ION>
__global__ void __launch_bounds__(kCgThreads, MINB) cg_resident_kernel(MonoDev d, const IDX* __restrict__ col,
                                                                       int cap_rows, ION ion) {
    extern __shared__ float sm[];
    float* sx = sm;
    float* sr = sx + cap_rows;
    float* sz = sr + cap_rows;
    float* sp = sz + cap_rows;
    float* sap = sp + cap_rows;
    float* sd = sap + cap_rows;
    __shared__ double sh_part[kCgWarps * 2];
    __shared__ double sh_tot[2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned nb = gridDim.x;
    const int64_t s_begin = (int64_t)blockIdx.x * d.n_slices / nb;
    const int64_t s_end = (int64_t)(blockIdx.x + 1) * d.n_slices / nb;
    const int64_t n = d.counter[0];
    int32_t* err = d.counter + 1;
    const float* __restrict__ u = d.x + ring_cur(n) * d.n_pad;
    const float* __restrict__ xp = d.x + ring_prev(n) * d.n_pad;
    float* __restrict__ xout = d.x + ring_next(n) * d.n_pad;
    const float* __restrict__ bp = d.bp;
    float* zg = d.r;              // z of every row, for neighbours
    float* pg[2] = {d.p, d.ap};   // search direction, double-buffered
    double* parts0 = d.scratch;
    double* parts1 = d.scratch + 2 * kMaxBlocks;
    const bool lg = d.linear_guess != 0;
    const uint64_t keep = l2_keep(), once = l2_once();

    // ---- right-hand side, guess, r0, z0 (solver.py:46-55; monodomain.py:130-131)
    double acc2[2] = {0.0, 0.0};
    if constexpr (ION::kFused) {
        // pass 1: ionic update of the block's rows (monodomain.py:117-128), then K u
        // (float32) and A x0 (float64) of the same rows; K u waits in sr, A x0 in
        // the p / Ap slots (read as one double per row, unused until the CG loop)
        const StepView sv = step_view(d, n);
        double* axd = reinterpret_cast<double*>(sp);
        for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
            const int64_t row = s * TCB_SLICE + lane;
            if (row >= d.n) continue;
            ionic_node<typename ION::Model, typename ION::Policy>(d, ion.c, ion.T, sv, row);
            const int li = (int)((s - s_begin) * TCB_SLICE + lane);
            const int64_t base = d.slice_ptr[s] + lane;
            const int w = (int)((d.slice_ptr[s + 1] - d.slice_ptr[s]) / TCB_SLICE);
            float ku = 0.0f;
            double ax = 0.0;
            for (int k0 = 0; k0 < w; k0 += 4) {
                int c[4];
                float kv[4], av[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const bool ok = k0 + j < w;
                    const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
                    c[j] = ok ? col_at<IDX>(col, e, row, keep) : (int)row;
                    kv[j] = ok ? ld_hint(d.kv + e, once) : 0.0f;
                    // M is read again by the second pass: keep it in L2 until then
                    av[j] = ok ? (ASPLIT ? __fadd_rn(__fmul_rn(ld_hint(d.mv + e, keep), d.cm), kv[j])
                                         : ld_hint(d.av + e, once))
                               : 0.0f;
                }
                float uc[4], xc[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    uc[j] = u[c[j]];
                    xc[j] = xp[c[j]];
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float xg = lg ? 2.0f * uc[j] - xc[j] : uc[j];
                    ku = __fmaf_rn(kv[j], uc[j], ku);
                    ax += (double)av[j] * (double)xg;
                }
            }
            const float ui = u[row];
            sx[li] = lg ? 2.0f * ui - xp[row] : ui;
            sr[li] = ku;
            axd[li] = ax;
            sd[li] = d.dinv[row];
        }
        // b' of every row is written
        if (!grid_barrier(d.bar, err, d.wait)) return;
        // pass 2: M b' (b' read through L2: this kernel wrote it), r0 = rhs - A x0, z0
        for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
            const int64_t row = s * TCB_SLICE + lane;
            if (row >= d.n) continue;
            const int li = (int)((s - s_begin) * TCB_SLICE + lane);
            const int64_t base = d.slice_ptr[s] + lane;
            const int w = (int)((d.slice_ptr[s + 1] - d.slice_ptr[s]) / TCB_SLICE);
            float mb = 0.0f;
            for (int k0 = 0; k0 < w; k0 += 4) {
                int c[4];
                float mv[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const bool ok = k0 + j < w;
                    const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
                    c[j] = ok ? col_at<IDX>(col, e, row, keep) : (int)row;
                    mv[j] = ok ? ld_hint(d.mv + e, once) : 0.0f;
                }
                float bc[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) bc[j] = __ldcg(d.bp + c[j]);
#pragma unroll
                for (int j = 0; j < 4; ++j) mb = __fmaf_rn(mv[j], bc[j], mb);
            }
            const float rhs = mb - sr[li];
            const float r32 = (float)((double)rhs - axd[li]);
            const float di = sd[li];
            const float z32 = (float)((double)di * (double)r32);
            sr[li] = r32;
            sz[li] = z32;
            zg[row] = z32;
            const double db = (double)di * (double)rhs;
            acc2[0] += db * db;
            acc2[1] += (double)r32 * (double)z32;
        }
        __syncthreads();   // the A x0 slots (p, Ap) are free again
    } else {
        for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
            const int64_t row = s * TCB_SLICE + lane;
            if (row >= d.n) continue;
            const int li = (int)((s - s_begin) * TCB_SLICE + lane);
            const int64_t base = d.slice_ptr[s] + lane;
            const int w = (int)((d.slice_ptr[s + 1] - d.slice_ptr[s]) / TCB_SLICE);
            // M b' and K u accumulate in float32 (the reference's float32 products),
            // A x0 in float64 (the reference's CG is float64; b - A x0 cancels)
            float mb = 0.0f, ku = 0.0f;
            double ax = 0.0;
            for (int k0 = 0; k0 < w; k0 += 4) {
                int c[4];
                float mv[4], kv[4], av[4];
    #pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const bool ok = k0 + j < w;
                    const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
                    c[j] = ok ? col_at<IDX>(col, e, row, keep) : (int)row;
                    mv[j] = ok ? ld_hint(d.mv + e, once) : 0.0f;
                    kv[j] = ok ? ld_hint(d.kv + e, once) : 0.0f;
                    av[j] = ok ? (ASPLIT ? __fadd_rn(__fmul_rn(mv[j], d.cm), kv[j]) : ld_hint(d.av + e, once)) : 0.0f;
                }
                float bc[4], uc[4], xc[4];
    #pragma unroll
                for (int j = 0; j < 4; ++j) {
                    bc[j] = bp[c[j]];
                    uc[j] = u[c[j]];
                    xc[j] = xp[c[j]];
                }
    #pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float xg = lg ? 2.0f * uc[j] - xc[j] : uc[j];
                    mb = __fmaf_rn(mv[j], bc[j], mb);
                    ku = __fmaf_rn(kv[j], uc[j], ku);
                    ax += (double)av[j] * (double)xg;
                }
            }
            const float rhs = mb - ku;
            const float ui = u[row];
            sx[li] = lg ? 2.0f * ui - xp[row] : ui;
            const float r32 = (float)((double)rhs - ax);
            const float di = d.dinv[row];
            const float z32 = (float)((double)di * (double)r32);
            sr[li] = r32;
            sz[li] = z32;
            sd[li] = di;
            zg[row] = z32;
            const double db = (double)di * (double)rhs;
            acc2[0] += db * db;
            acc2[1] += (double)r32 * (double)z32;
        }
    }
    block_partial<2>(acc2, parts0, sh_part);
    if (!grid_barrier(d.bar, err, d.wait)) return;
    double tot[2];
    grid_total<2>(parts0, tot, sh_tot);
    const double b_norm = sqrt(tot[0]);
    double rz = tot[1];
    double beta = 0.0;

    int it = 0;
    while (it < d.max_iter) {
        const bool first = it == 0;
        const float beta32 = (float)beta;
        const float* pin = pg[it & 1];
        float* __restrict__ pout = pg[(it + 1) & 1];
        // ---- p = z + beta p (on the fly), Ap, p.Ap
        double acc1[1] = {0.0};
        for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
            const int64_t row = s * TCB_SLICE + lane;
            if (row >= d.n) continue;
            const int li = (int)((s - s_begin) * TCB_SLICE + lane);
            const int64_t base = d.slice_ptr[s] + lane;
            const int w = (int)((d.slice_ptr[s + 1] - d.slice_ptr[s]) / TCB_SLICE);
            double a = 0.0;
            for (int k0 = 0; k0 < w; k0 += 8) {
                int c[8];
                float av[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const bool ok = k0 + j < w;
                    const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
                    c[j] = ok ? col_at<IDX>(col, e, row, keep) : (int)row;
                    av[j] = ok ? ld_hint(d.av + e, once) : 0.0f;
                }
                float zc[8], pc[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    zc[j] = zg[c[j]];
                    pc[j] = first ? 0.0f : pin[c[j]];
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) a += (double)av[j] * (double)p_update(zc[j], pc[j], beta32, first);
            }
            const float pn = p_update(sz[li], first ? 0.0f : sp[li], beta32, first);
            sp[li] = pn;
            pout[row] = pn;
            const float a32 = (float)a;
            sap[li] = a32;
            acc1[0] += (double)pn * (double)a32;
        }
        __syncthreads();
        block_partial<1>(acc1, parts1, sh_part);
        if (!grid_barrier(d.bar, err, d.wait)) return;
        double pap[1];
        grid_total<1>(parts1, pap, sh_tot);
        const double alpha = rz / pap[0];

        // ---- x += alpha p, r -= alpha Ap, z = D r; ||z||^2, r.z
        acc2[0] = acc2[1] = 0.0;
        for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
            const int64_t row = s * TCB_SLICE + lane;
            if (row >= d.n) continue;
            const int li = (int)((s - s_begin) * TCB_SLICE + lane);
            sx[li] = (float)((double)sx[li] + alpha * (double)sp[li]);
            const float r32 = (float)((double)sr[li] - alpha * (double)sap[li]);
            sr[li] = r32;
            const float z32 = (float)((double)sd[li] * (double)r32);
            sz[li] = z32;
            zg[row] = z32;
            acc2[0] += (double)z32 * (double)z32;
            acc2[1] += (double)r32 * (double)z32;
        }
        __syncthreads();
        block_partial<2>(acc2, parts0, sh_part);
        if (!grid_barrier(d.bar, err, d.wait)) return;
        grid_total<2>(parts0, tot, sh_tot);
        const double zn = sqrt(tot[0]);
        if (zn < d.a_tol || (zn / b_norm) < d.r_tol) break;   // solver.py:66-69
        beta = tot[1] / rz;
        rz = tot[1];
        ++it;
    }
    // the solution leaves shared memory once
    for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
        const int64_t row = s * TCB_SLICE + lane;
        if (row < d.n) xout[row] = sx[(s - s_begin) * TCB_SLICE + lane];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d.step_iters[n] = it;
        d.counter[0] = (int32_t)(n + 1);
    }
}

using PickFn = const void* (*)(int per_sm, bool asplit);

template <typename IDX>
const void* pick(int per_sm, bool asplit) {
    if (per_sm == 2)
        return asplit ? (const void*)cg_resident_kernel<IDX, 2, true, NoIonic>
                      : (const void*)cg_resident_kernel<IDX, 2, false, NoIonic>;
    return asplit ? (const void*)cg_resident_kernel<IDX, 1, true, NoIonic>
                  : (const void*)cg_resident_kernel<IDX, 1, false, NoIonic>;
}

// the fused step instances (int16 column offsets only)
template <class M, class Q>
const void* pick_fused(int per_sm, bool asplit) {
    using I = WithIonic<M, Q>;
    if (per_sm == 2)
        return asplit ? (const void*)cg_resident_kernel<int16_t, 2, true, I>
                      : (const void*)cg_resident_kernel<int16_t, 2, false, I>;
    return asplit ? (const void*)cg_resident_kernel<int16_t, 1, true, I>
                  : (const void*)cg_resident_kernel<int16_t, 1, false, I>;
}

// division policy of each model's fused step: TTP and MS under the 64-register
// budget of two 512-thread blocks per SM take IEEE division (far fewer spills
// there); CRN, whose update needs more registers in any case, the hardware forms
const PickFn kFusedPick[4] = {nullptr, pick_fused<MS, QExact>, pick_fused<TTP, QExact>, pick_fused<CRN, QFast>};

PickFn cg_pick(bool i16) { return i16 ? pick<int16_t> : pick<int32_t>; }

struct ResidentInfo {
    int sms = 0;
    int max_smem = 0;
    bool configured = false;
};

ResidentInfo& resident_info() {
    static ResidentInfo infos[64];
    int dev = 0;
    cudaGetDevice(&dev);
    ResidentInfo& ri = infos[dev & 63];
    if (!ri.configured) {
        cudaDeviceGetAttribute(&ri.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&ri.max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        int reserve = (int)(sizeof(double) * (kCgWarps * 2 + 2)) + 1024;
        ri.max_smem -= reserve;
        const PickFn picks[5] = {pick<int16_t>, pick<int32_t>, kFusedPick[1], kFusedPick[2], kFusedPick[3]};
        for (PickFn pk : picks)
            for (int ps = 1; ps <= 2; ++ps)
                for (int as = 0; as < 2; ++as)
                    cudaFuncSetAttribute(pk(ps, as), cudaFuncAttributeMaxDynamicSharedMemorySize, ri.max_smem);
        ri.configured = true;
    }
    return ri;
}

constexpr int kResidentBytesPerRow = 6 * sizeof(float);

// Grid of the resident kernel: the most blocks per SM (2, else 1) whose rows fit.
bool resident_plan(const MonoDev& d, unsigned* nb_out, int* cap_out, size_t* smem_out, int* per_sm_out, PickFn pk) {
    ResidentInfo& ri = resident_info();
    // d.cg_per_sm = 1 or 2 pins the blocks per SM (a tuning choice); 0: 2 if the rows fit, else 1
    const int hi = d.cg_per_sm == 1 ? 1 : 2, lo = d.cg_per_sm == 2 ? 2 : 1;
    for (int per_sm = hi; per_sm >= lo; --per_sm) {
        int64_t want = ceil_div(d.n_slices, kMinSlicesPerBlock);
        int64_t nb = std::min<int64_t>(want, (int64_t)ri.sms * per_sm);
        if (nb < 1) nb = 1;
        int64_t cap = ceil_div(d.n_slices, nb) * TCB_SLICE;
        size_t smem = (size_t)cap * kResidentBytesPerRow;
        if ((int64_t)smem > (int64_t)ri.max_smem) continue;
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pk(per_sm, d.a_split != 0), kCgThreads, smem);
        if (occ < per_sm) continue;
        *nb_out = (unsigned)nb;
        *cap_out = (int)cap;
        *smem_out = smem;
        *per_sm_out = per_sm;
        return true;
    }
    return false;
}

template <class ION>
int launch_resident(const MonoDev& d, cudaStream_t s, PickFn pk, const void* colp, const ION& ion) {
    unsigned nb = 0;
    int cap = 0;
    size_t smem = 0;
    int per_sm = 0;
    if (!resident_plan(d, &nb, &cap, &smem, &per_sm, pk)) return 0;
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
    void* args[] = {const_cast<MonoDev*>(&d), const_cast<const void**>(&colp), &cap, const_cast<ION*>(&ion)};
    cudaError_t e = cudaLaunchKernelExC(&cfg, pk(per_sm, d.a_split != 0), args);
    if (e != cudaSuccess) return cuda_fail(e, "resident CG launch");
    return 1;
}

template <class M, class Q>
int launch_fused(const tcb_mono* m, const MonoDev& d, cudaStream_t s) {
    WithIonic<M, Q> ion;
    ion.c = M::derive(m->params);
    ion.T = M::tables(m->tables, m->params);
    return launch_resident(d, s, pick_fused<M, Q>, (const void*)d.dcol, ion);
}

}  // namespace

int resident_blocks(const MonoDev& d) {
    unsigned nb = 0;
    int cap = 0;
    size_t smem = 0;
    int per_sm = 0;
    return resident_plan(d, &nb, &cap, &smem, &per_sm, cg_pick(d.dcol != nullptr)) ? (int)nb : 0;
}

// 1 = launched, 0 = does not fit (caller falls back), <0 = error
int launch_cg_resident(const MonoDev& d, cudaStream_t s) {
    const bool i16 = d.dcol != nullptr;
    return launch_resident(d, s, cg_pick(i16), i16 ? (const void*)d.dcol : (const void*)d.col, NoIonic{});
}

// The whole step as one launch (ionic update fused into the resident CG kernel):
// 1 = launched, 0 = not applicable here (32-bit columns, rows that do not fit in
// shared memory): the caller runs the two kernels; <0 = error.
int launch_mono_step(const tcb_mono* m, const MonoDev& d, cudaStream_t s) {
    if (!d.dcol) return 0;
    switch (m->model) {
        case TCB_MODEL_MS: return launch_fused<MS, QExact>(m, d, s);
        case TCB_MODEL_TTP: return launch_fused<TTP, QExact>(m, d, s);
        case TCB_MODEL_CRN: return launch_fused<CRN, QFast>(m, d, s);
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

// 1 if launch_mono_step would run the fused kernel for this simulation
int mono_step_fusable(const tcb_mono* m, const MonoDev& d) {
    if (!d.dcol || m->model < TCB_MODEL_MS || m->model > TCB_MODEL_CRN) return 0;
    unsigned nb = 0;
    int cap = 0;
    size_t smem = 0;
    int per_sm = 0;
    return resident_plan(d, &nb, &cap, &smem, &per_sm, kFusedPick[m->model]) ? 1 : 0;
}

}  // namespace tcb
