// Batched persistent cooperative CG: every simulation of a batch takes its
// right-hand side, guess and Jacobi-PCG solve (torchcor/core/solver.py:40-76)
// in one launch, with its own alpha, beta, norms, stopping test and iteration
// count (per-simulation convergence masks).
//
// The simulations' 32-row slices form one virtual slice space split evenly
// over the blocks.  Vectors live in global memory (a batch is larger than
// what shared memory holds); the arithmetic is that of the resident
// single-simulation kernel (fused p-update with a double-buffered p, float64
// row sums and inner products, int16 column offsets and A rebuilt from M and K'
// where the simulation allows).
//
// Reductions are per simulation and deterministic: a warp reduces each slice's
// rows and adds the result to its per-simulation slot in slice order, the
// block adds its warps' slots in warp order into its partial for each
// simulation it overlaps, and after the grid barrier every block sums each
// simulation's partials in block order (a warp per simulation, strided lanes
// and a fixed shuffle tree), so all blocks hold identical scalars and take
// identical control-flow decisions.
#include <cuda_runtime.h>
#include <math.h>

#include "batch.cuh"
#include "cg_common.cuh"
#include "tcb_internal.h"

namespace tcb {
namespace {

using namespace cgk;
static_assert(sizeof(MonoDev) % 8 == 0, "MonoDev is copied as words and followed by int64 data");

__device__ __forceinline__ float p_update(float z, float p_old, double beta, bool first) {
    return first ? z : (float)(beta * (double)p_old + (double)z);
}

__device__ __forceinline__ int col_of(const MonoDev& d, int64_t e, int64_t row) {
    return d.dcol ? (int)row + (int)__ldg(d.dcol + e) : __ldg(d.col + e);
}

struct BatchShared {
    double *rz, *bn, *al, *be, *wp;  // per simulation; wp = [warps][kBatchMaxPerBlock][2]
    MonoDev* dev;                    // descriptors of the block's simulations
    int64_t* lsp;                    // their first virtual slice, [kBatchMaxPerBlock + 1]
    int *it, *act, *step;
};

__device__ __forceinline__ BatchShared carve(double* smd, int n) {
    BatchShared s;
    s.rz = smd;
    s.bn = s.rz + n;
    s.al = s.bn + n;
    s.be = s.al + n;
    s.wp = s.be + n;
    s.dev = reinterpret_cast<MonoDev*>(s.wp + kCgWarps * kBatchMaxPerBlock * 2);
    s.lsp = reinterpret_cast<int64_t*>(s.dev + kBatchMaxPerBlock);
    s.it = reinterpret_cast<int*>(s.lsp + kBatchMaxPerBlock + 1);
    s.act = s.it + n;
    s.step = s.act + n;
    return s;
}

// copy the descriptors and slice offsets of the block's simulations into shared memory
__device__ __forceinline__ void stage_descriptors(const BatchWS* W, BatchShared& S, int first, int cnt) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(W->dev + first);
    uint32_t* dst = reinterpret_cast<uint32_t*>(S.dev);
    const int words = cnt * (int)(sizeof(MonoDev) / 4);
    for (int t = threadIdx.x; t < words; t += blockDim.x) dst[t] = src[t];
    for (int t = threadIdx.x; t <= cnt; t += blockDim.x) S.lsp[t] = W->slice_prefix[first + t];
}

// warp-reduce two values and add them to this warp's slot of local simulation j
__device__ __forceinline__ void warp_add(BatchShared& S, int warp, int lane, int j, double a, double b) {
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        S.wp[(warp * kBatchMaxPerBlock + j) * 2 + 0] += a;
        S.wp[(warp * kBatchMaxPerBlock + j) * 2 + 1] += b;
    }
}

__device__ __forceinline__ void clear_slots(BatchShared& S, int cnt) {
    for (int t = threadIdx.x; t < kCgWarps * kBatchMaxPerBlock * 2; t += blockDim.x) S.wp[t] = 0.0;
    __syncthreads();
}

// block partials (NV values) of the block's simulations -> parts[value][blk_off + j]
template <int NV>
__device__ __forceinline__ void publish(const BatchWS* W, BatchShared& S, double* parts, int cnt, int off) {
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x)
        for (int v = 0; v < NV; ++v) {
            double acc = 0.0;
            for (int w = 0; w < kCgWarps; ++w) acc += S.wp[(w * kBatchMaxPerBlock + j) * 2 + v];
            parts[(size_t)v * W->parts_stride + off + j] = acc;
        }
}

// every block: totals of every simulation (warp per simulation)
template <int NV, class F>
__device__ __forceinline__ void totals(const BatchWS* W, const double* parts, F&& consume) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < W->n; i += kCgWarps) {
        const int b0 = W->inst_b0[i], b1 = W->inst_b1[i];
        double acc[NV];
        for (int v = 0; v < NV; ++v) acc[v] = 0.0;
        for (int b = b0 + lane; b <= b1; b += 32) {
            const int slot = W->blk_off[b] + (i - W->blk_first[b]);
            for (int v = 0; v < NV; ++v) acc[v] += __ldcg(parts + (size_t)v * W->parts_stride + slot);
        }
        for (int v = 0; v < NV; ++v) acc[v] = warp_sum(acc[v]);
        if (lane == 0) consume(i, acc);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kCgThreads) batch_cg_kernel(const BatchWS* __restrict__ W) {
    extern __shared__ double smd[];
    __shared__ int s_any;
    const int n = W->n;
    BatchShared S = carve(smd, n);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nb = gridDim.x, b = blockIdx.x;
    const int64_t vb = (int64_t)b * W->total_slices / nb, ve = (int64_t)(b + 1) * W->total_slices / nb;
    const int first = W->blk_first[b], cnt = W->blk_count[b], off = W->blk_off[b];
    double* parts0 = W->parts;
    double* parts1 = W->parts + 2 * (size_t)W->parts_stride;
    int32_t* err = W->err;

    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int64_t st = W->dev[i].counter[0];
        S.step[i] = (st >= 1 && st <= W->dev[i].nt) ? (int)st : 0;   // 0 = not stepping
    }
    stage_descriptors(W, S, first, cnt);
    clear_slots(S, cnt);

    // ---- right-hand side, guess, r0, z0
    {
        int js = 0;
        for (int64_t vs = vb + warp; vs < ve; vs += kCgWarps) {
            while (S.lsp[js + 1] <= vs) ++js;
            const int i = first + js;
            const int step = S.step[i];
            if (!step) continue;
            const MonoDev& d = S.dev[js];
            const int64_t ls = vs - S.lsp[js];
            const int64_t row = ls * TCB_SLICE + lane;
            double bb = 0.0, rzl = 0.0;
            if (row < d.n) {
                const float* u = d.x + ring_cur(step) * d.n_pad;
                const float* xp = d.x + ring_prev(step) * d.n_pad;
                float* xn = d.x + ring_next(step) * d.n_pad;
                const bool lg = d.linear_guess != 0, as = d.a_split != 0;
                const int64_t base = d.slice_ptr[ls] + lane;
                const int w = (int)((d.slice_ptr[ls + 1] - d.slice_ptr[ls]) / TCB_SLICE);
                double mb = 0.0, ku = 0.0, ax = 0.0;
                for (int k0 = 0; k0 < w; k0 += 4) {
                    int c[4];
                    float mv[4], kv[4], av[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const bool ok = k0 + j < w;
                        const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
                        c[j] = ok ? col_of(d, e, row) : (int)row;
                        mv[j] = ok ? __ldg(d.mv + e) : 0.0f;
                        kv[j] = ok ? __ldg(d.kv + e) : 0.0f;
                        av[j] = ok ? (as ? __fadd_rn(__fmul_rn(mv[j], d.cm), kv[j]) : __ldg(d.av + e)) : 0.0f;
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float uc = u[c[j]];
                        const float xg = lg ? 2.0f * uc - xp[c[j]] : uc;
                        mb += (double)mv[j] * (double)d.bp[c[j]];
                        ku += (double)kv[j] * (double)uc;
                        ax += (double)av[j] * (double)xg;
                    }
                }
                const float rhs = (float)mb - (float)ku;
                const float ui = u[row];
                xn[row] = lg ? 2.0f * ui - xp[row] : ui;
                const float r32 = (float)((double)rhs - ax);
                const float di = d.dinv[row];
                const float z32 = (float)((double)di * (double)r32);
                d.r[row] = r32;
                d.z[row] = z32;
                const double db = (double)di * (double)rhs;
                bb = db * db;
                rzl = (double)r32 * (double)z32;
            }
            warp_add(S, warp, lane, js, bb, rzl);
        }
    }
    publish<2>(W, S, parts0, cnt, off);
    if (!grid_barrier(W->bar, err)) return;
    totals<2>(W, parts0, [&](int i, double* t) {
        S.bn[i] = sqrt(t[0]);
        S.rz[i] = t[1];
        S.be[i] = 0.0;
        S.it[i] = 0;
        S.act[i] = S.step[i] != 0 && W->dev[i].max_iter > 0;
    });

    for (int pass = 0;; ++pass) {
        if (threadIdx.x == 0) {
            int any = 0;
            for (int i = 0; i < n; ++i) any |= S.act[i];
            s_any = any;
        }
        __syncthreads();
        if (!s_any) break;
        const bool first_pass = pass == 0;
        // ---- p = z + beta p (on the fly), Ap, p.Ap
        clear_slots(S, cnt);
        {
            int js = 0;
            for (int64_t vs = vb + warp; vs < ve; vs += kCgWarps) {
                while (S.lsp[js + 1] <= vs) ++js;
                const int i = first + js;
                if (!S.act[i]) continue;
                const MonoDev& d = S.dev[js];
                const float* pin = (pass & 1) ? d.p2 : d.p;
                float* pout = (pass & 1) ? d.p : d.p2;
                const double beta = S.be[i];
                const int64_t ls = vs - S.lsp[js];
                const int64_t row = ls * TCB_SLICE + lane;
                double pap = 0.0;
                if (row < d.n) {
                    const int64_t base = d.slice_ptr[ls] + lane;
                    const int w = (int)((d.slice_ptr[ls + 1] - d.slice_ptr[ls]) / TCB_SLICE);
                    double a = 0.0;
                    for (int k0 = 0; k0 < w; k0 += 8) {
                        int c[8];
                        float av[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const bool ok = k0 + j < w;
                            const int64_t e = base + (int64_t)(k0 + j) * TCB_SLICE;
                            c[j] = ok ? col_of(d, e, row) : (int)row;
                            av[j] = ok ? __ldg(d.av + e) : 0.0f;
                        }
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const float pc = first_pass ? 0.0f : pin[c[j]];
                            a += (double)av[j] * (double)p_update(d.z[c[j]], pc, beta, first_pass);
                        }
                    }
                    const float pn = p_update(d.z[row], first_pass ? 0.0f : pin[row], beta, first_pass);
                    pout[row] = pn;
                    const float a32 = (float)a;
                    d.ap[row] = a32;
                    pap = (double)pn * (double)a32;
                }
                warp_add(S, warp, lane, js, pap, 0.0);
            }
        }
        publish<1>(W, S, parts1, cnt, off);
        if (!grid_barrier(W->bar, err)) return;
        totals<1>(W, parts1, [&](int i, double* t) {
            if (S.act[i]) S.al[i] = S.rz[i] / t[0];
        });

        // ---- x += alpha p, r -= alpha Ap, z = D r; ||z||^2, r.z
        clear_slots(S, cnt);
        {
            int js = 0;
            for (int64_t vs = vb + warp; vs < ve; vs += kCgWarps) {
                while (S.lsp[js + 1] <= vs) ++js;
                const int i = first + js;
                if (!S.act[i]) continue;
                const MonoDev& d = S.dev[js];
                const float* pnew = (pass & 1) ? d.p : d.p2;
                const double alpha = S.al[i];
                const int64_t row = (vs - S.lsp[js]) * TCB_SLICE + lane;
                double zz = 0.0, rzn = 0.0;
                if (row < d.n) {
                    float* x = d.x + ring_next(S.step[i]) * d.n_pad;
                    x[row] = (float)((double)x[row] + alpha * (double)pnew[row]);
                    const float r32 = (float)((double)d.r[row] - alpha * (double)d.ap[row]);
                    d.r[row] = r32;
                    const float z32 = (float)((double)d.dinv[row] * (double)r32);
                    d.z[row] = z32;
                    zz = (double)z32 * (double)z32;
                    rzn = (double)r32 * (double)z32;
                }
                warp_add(S, warp, lane, js, zz, rzn);
            }
        }
        publish<2>(W, S, parts0, cnt, off);
        if (!grid_barrier(W->bar, err)) return;
        totals<2>(W, parts0, [&](int i, double* t) {
            if (!S.act[i]) return;
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
    // each simulation's first block records its iterations and advances its step
    if (threadIdx.x == 0)
        for (int i = first; i < first + cnt; ++i)
            if (W->inst_b0[i] == b && S.step[i]) {
                W->dev[i].step_iters[S.step[i]] = S.it[i];
                W->dev[i].counter[0] = S.step[i] + 1;
            }
}

}  // namespace

size_t batch_cg_smem(int n) {
    return (size_t)n * (4 * sizeof(double) + 3 * sizeof(int)) + sizeof(double) * kCgWarps * kBatchMaxPerBlock * 2 +
           sizeof(MonoDev) * kBatchMaxPerBlock + sizeof(int64_t) * (kBatchMaxPerBlock + 1) + 64;
}

int batch_cg_max_blocks(size_t smem) {
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(batch_cg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_cg_kernel, kCgThreads, smem);
    int cap = sms * occ;
    return cap > kMaxBlocks ? kMaxBlocks : cap;
}

int launch_batch_cg(const BatchWS* ws_dev, int nb, size_t smem, cudaStream_t s) {
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
    TCB_CHECK_CUDA(cudaLaunchKernelEx(&cfg, batch_cg_kernel, ws_dev));
    return TCB_OK;
}

}  // namespace tcb
