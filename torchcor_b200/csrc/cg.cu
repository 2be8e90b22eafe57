// The electric half of a monodomain step as one persistent cooperative
// kernel: right-hand side b = M b' - ((1-theta) dt K/chi) u, the linear
// extrapolation guess, and the Jacobi-preconditioned CG of
// torchcor/core/solver.py:40-76 with the device-side stopping test.
//
// Matrix, vectors and values are float32 (sliced ELL, one warp per 32-row
// slice); row sums, inner products and the stopping test are float64.  Every
// block owns a fixed range of slices for the whole solve, so a thread always
// revisits the rows it wrote; cross-block dependencies are the search
// direction p (read with ld.global.cg after a grid barrier) and the scalar
// reductions (per-block partials, summed by every block in the same fixed
// order, so all blocks take identical control-flow decisions).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "cg_common.cuh"
#include "l2_hint.cuh"
#include "mono.cuh"
#include "tcb_internal.h"

namespace tcb {
namespace {

using namespace cgk;

__global__ void __launch_bounds__(kCgThreads, 2) cg_kernel(MonoDev d) {
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
    float* __restrict__ x = d.x + ring_next(n) * d.n_pad;
    const float* __restrict__ bp = d.bp;
    float* __restrict__ r = d.r;
    float* __restrict__ p = d.p;
    float* __restrict__ ap = d.ap;
    const float* __restrict__ dinv = d.dinv;
    double* parts0 = d.scratch;
    double* parts1 = d.scratch + 2 * kMaxBlocks;
    const bool lg = d.linear_guess != 0;
    const uint64_t once = l2_once();   // M, K and A: first to leave L2

    // ---- right-hand side, initial guess, r0, z0 = p0 (solver.py:46-55; monodomain.py:130-131)
    double acc2[2] = {0.0, 0.0};  // ||D b||^2, r.z
    for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
        const int64_t row = s * TCB_SLICE + lane;
        if (row >= d.n) continue;
        const int64_t base = d.slice_ptr[s] + lane;
        const int w = (int)((d.slice_ptr[s + 1] - d.slice_ptr[s]) / TCB_SLICE);
        // M b' and K u in float32 (the reference's float32 products), A x0 in float64
        float mb = 0.0f, ku = 0.0f;
        double ax = 0.0;
        for (int k = 0; k < w; ++k) {
            const int64_t e = base + (int64_t)k * TCB_SLICE;
            const int c = __ldg(d.col + e);
            const float uc = u[c];
            const float xg = lg ? 2.0f * uc - xp[c] : uc;
            mb = __fmaf_rn(ld_hint(d.mv + e, once), bp[c], mb);
            ku = __fmaf_rn(ld_hint(d.kv + e, once), uc, ku);
            ax += (double)ld_hint(d.av + e, once) * (double)xg;
        }
        const float rhs = mb - ku;
        const float ui = u[row];
        x[row] = lg ? 2.0f * ui - xp[row] : ui;
        const float r32 = (float)((double)rhs - ax);
        const double di = (double)dinv[row];
        const double z = di * (double)r32;
        r[row] = r32;
        p[row] = (float)z;
        const double db = di * (double)rhs;
        acc2[0] += db * db;
        acc2[1] += (double)r32 * z;
    }
    block_partial<2>(acc2, parts0, sh_part);
    if (!grid_barrier(d.bar, err, d.wait)) return;
    double tot[2];
    grid_total<2>(parts0, tot, sh_tot);
    const double b_norm = sqrt(tot[0]);
    double rz = tot[1];

    int it = 0;
    while (it < d.max_iter) {
        // ---- Ap = A p, p.Ap
        double acc1[1] = {0.0};
        for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
            const int64_t row = s * TCB_SLICE + lane;
            if (row >= d.n) continue;
            const int64_t base = d.slice_ptr[s] + lane;
            const int w = (int)((d.slice_ptr[s + 1] - d.slice_ptr[s]) / TCB_SLICE);
            double a = 0.0;
            for (int k = 0; k < w; ++k) {
                const int64_t e = base + (int64_t)k * TCB_SLICE;
                a += (double)ld_hint(d.av + e, once) * (double)__ldcg(p + __ldg(d.col + e));
            }
            const float a32 = (float)a;
            ap[row] = a32;
            acc1[0] += (double)p[row] * (double)a32;
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
            x[row] = (float)((double)x[row] + alpha * (double)p[row]);
            const float r32 = (float)((double)r[row] - alpha * (double)ap[row]);
            r[row] = r32;
            const double z = (double)dinv[row] * (double)r32;
            acc2[0] += z * z;
            acc2[1] += (double)r32 * z;
        }
        __syncthreads();
        block_partial<2>(acc2, parts0, sh_part);
        if (!grid_barrier(d.bar, err, d.wait)) return;
        grid_total<2>(parts0, tot, sh_tot);
        const double zn = sqrt(tot[0]);
        if (zn < d.a_tol || (zn / b_norm) < d.r_tol) break;   // solver.py:66-69
        const double beta = tot[1] / rz;
        rz = tot[1];

        // ---- p = beta p + z
        for (int64_t s = s_begin + warp; s < s_end; s += kCgWarps) {
            const int64_t row = s * TCB_SLICE + lane;
            if (row >= d.n) continue;
            p[row] = (float)(beta * (double)p[row] + (double)dinv[row] * (double)r[row]);
        }
        if (!grid_barrier(d.bar, err, d.wait)) return;
        ++it;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d.step_iters[n] = it;
        d.counter[0] = (int32_t)(n + 1);
    }
}

struct DeviceInfo {
    int sms = 0;
    int cg_blocks_per_sm = 0;
};

DeviceInfo& device_info() {
    static std::mutex mu;
    static std::vector<DeviceInfo> infos;
    std::lock_guard<std::mutex> g(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if ((int)infos.size() <= dev) infos.resize(dev + 1);
    DeviceInfo& di = infos[dev];
    if (di.sms == 0) {
        cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&di.cg_blocks_per_sm, cg_kernel, kCgThreads, 0);
    }
    return di;
}

}  // namespace

int num_sms() { return device_info().sms; }

// TCB_CG_KERNEL=streaming forces the streaming kernel, TCB_CG_INDEX=int32 the
// 32-bit column stream (both for testing the paths large meshes take).
static bool env_is(const char* name, const char* value) {
    const char* v = getenv(name);
    return v && strcmp(v, value) == 0;
}

// Number of blocks launch_cg uses for this simulation on the current device.
int cg_blocks(const MonoDev& d) {
    int r = env_is("TCB_CG_KERNEL", "streaming") ? 0 : resident_blocks(d);
    if (r > 0) return r;
    DeviceInfo& di = device_info();
    int64_t want = ceil_div(d.n_slices, kMinSlicesPerBlock);
    int64_t cap = (int64_t)di.sms * di.cg_blocks_per_sm;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    int64_t nb = want < cap ? want : cap;
    return (int)(nb < 1 ? 1 : nb);
}

// the test variables that force the streaming kernel or 32-bit columns (these also rule out the fused step)
bool cg_forced_fallback() { return env_is("TCB_CG_KERNEL", "streaming") || env_is("TCB_CG_INDEX", "int32"); }

// 1 if launch_cg runs the shared-memory-resident kernel for this simulation, 0 if the streaming one
int cg_uses_resident(const MonoDev& d) { return !env_is("TCB_CG_KERNEL", "streaming") && resident_blocks(d) > 0; }

int launch_cg(const MonoDev& d, cudaStream_t s) {
    if (!env_is("TCB_CG_KERNEL", "streaming")) {
        MonoDev dd = d;
        if (env_is("TCB_CG_INDEX", "int32")) dd.dcol = nullptr;
        int r = launch_cg_resident(dd, s);
        if (r < 0) return r;
        if (r == 1) return TCB_OK;
    }
    DeviceInfo& di = device_info();
    if (di.cg_blocks_per_sm <= 0) return fail(TCB_ECUDA, "CG kernel cannot be resident on this device");
    int64_t want = ceil_div(d.n_slices, kMinSlicesPerBlock);
    int64_t cap = (int64_t)di.sms * di.cg_blocks_per_sm;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    unsigned nb = (unsigned)(want < cap ? want : cap);
    if (nb < 1) nb = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nb);
    cfg.blockDim = dim3(kCgThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TCB_CHECK_CUDA(cudaLaunchKernelEx(&cfg, cg_kernel, d));
    return TCB_OK;
}

}  // namespace tcb

extern "C" int64_t tcb_mono_scratch_doubles(void) { return 4 * (int64_t)tcb::kMaxBlocks; }
