// Status handling and the time-loop entry points of the C ABI.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "mono.cuh"
#include "tcb_internal.h"

namespace tcb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return TCB_ECUDA;
}

MonoDev make_dev(const tcb_mono* m) {
    MonoDev d;
    d.n = m->n_nodes;
    d.n_pad = m->n_pad;
    d.n_slices = m->n_slices;
    d.nt = m->nt;
    d.slice_ptr = m->slice_ptr;
    d.col = m->col;
    d.dcol = m->col_delta;
    d.mv = m->m_val;
    d.kv = m->k_val;
    d.av = m->a_val;
    d.dinv = m->d_inv;
    d.state = m->state;
    d.tables = m->tables;
    d.x = m->x;
    d.bp = m->bprime;
    d.r = m->r;
    d.p = m->p;
    d.ap = m->ap;
    d.z = m->z;
    d.p2 = m->p2;
    d.at = m->at;
    d.rt = m->rt;
    d.snap = m->snapshots;
    d.snap_ring = m->snap_ring;
    d.cg_per_sm = m->cg_per_sm;
    d.stim_bits = m->stim_bits;
    d.node_params = m->node_params;
    d.step_t = m->step_t;
    d.step_stim = m->step_stim;
    d.step_iters = m->step_iters;
    d.counter = m->counter;
    d.scratch = m->scratch;
    d.bar = m->barrier;
    d.a_tol = m->a_tol;
    d.r_tol = m->r_tol;
    d.max_iter = m->max_iter;
    d.linear_guess = m->linear_guess;
    d.at_rt = m->at_rt;
    d.per_frame = m->per_frame;
    d.a_split = m->a_split;
    d.cm = m->cm;
    d.dt = m->dt;
    for (int k = 0; k < TCB_MAX_STIMULI; ++k) d.amp[k] = m->stim_amp[k];
    d.wait = wait_limit();
    return d;
}

// TCB_TEST_WAIT_STALL=grid|copy makes a bounded wait run out after 10 ms (the
// failure-detection tests); unset, the waits only guard against a lost block.
cgk::WaitLimit wait_limit() {
    cgk::WaitLimit w = {cgk::kBarrierTimeoutNs, 0u, 0u};
    const char* v = getenv("TCB_TEST_WAIT_STALL");
    if (v && (strcmp(v, "grid") == 0 || strcmp(v, "copy") == 0)) {
        w.timeout_ns = 10000000ull;
        w.extra_arrivals = strcmp(v, "grid") == 0 ? 1u : 0u;
        w.drop_first_copy = strcmp(v, "copy") == 0 ? 1u : 0u;
    }
    return w;
}

namespace {
int validate(const tcb_mono* m) {
    if (!m) return fail(TCB_EINVAL, "null tcb_mono");
    if (m->n_nodes <= 0 || m->n_pad < m->n_nodes || m->n_pad % 128 != 0 ||
        m->n_slices != ceil_div(m->n_nodes, TCB_SLICE) || m->nt < 0)
        return fail(TCB_EINVAL, "tcb_mono: inconsistent sizes");
    if (m->nt >= INT32_MAX) return fail(TCB_ERANGE, "tcb_mono: more than 2^31 - 2 time steps");
    if (!m->slice_ptr || !m->col || !m->m_val || !m->k_val || !m->a_val || !m->d_inv || !m->state || !m->x ||
        !m->bprime || !m->r || !m->p || !m->ap || !m->at || !m->rt || !m->stim_bits || !m->step_t ||
        !m->step_stim || !m->step_iters || !m->counter || !m->scratch || !m->barrier || !m->params)
        return fail(TCB_EINVAL, "tcb_mono: null pointer");
    if (m->model != TCB_MODEL_MS && !m->tables) return fail(TCB_EINVAL, "tcb_mono: null tables");
    // the grid barrier's count and generation are one 64-bit word
    if ((uintptr_t)m->barrier & 7u) return fail(TCB_EINVAL, "tcb_mono: barrier words not 8-byte aligned");
    // the ionic kernels read table column pairs as 8-byte vectors
    if (m->model != TCB_MODEL_MS && ((uintptr_t)m->tables & 15u))
        return fail(TCB_EINVAL, "tcb_mono: tables not 16-byte aligned");
    if (m->max_iter < 0 || m->per_frame < 0 || m->snap_ring < 0)
        return fail(TCB_EINVAL, "tcb_mono: negative max_iter/per_frame/snap_ring");
    if (m->ionic_variant < 0 || m->cg_per_sm < 0 || m->cg_per_sm > 2)
        return fail(TCB_EINVAL, "tcb_mono: ionic_variant < 0 or cg_per_sm outside 0..2");
    return TCB_OK;
}
}  // namespace

int validate_mono(const tcb_mono* m) { return validate(m); }

}  // namespace tcb

using namespace tcb;

extern "C" int tcb_version(void) { return 1; }

extern "C" const char* tcb_status_string(int status) {
    switch (status) {
        case TCB_OK: return "ok";
        case TCB_EINVAL: return "invalid argument";
        case TCB_ECUDA: return "CUDA error";
        case TCB_ETIMEOUT: return "device wait timed out";
        case TCB_ENOMEM: return "out of host memory";
        case TCB_ERANGE: return "size out of range";
    }
    return "unknown status";
}

extern "C" int tcb_last_error(char* buf, int64_t len) {
    if (!buf || len <= 0) return TCB_EINVAL;
    const std::string& s = g_last_error;
    int64_t n = (int64_t)s.size() < len - 1 ? (int64_t)s.size() : len - 1;
    memcpy(buf, s.data(), (size_t)n);
    buf[n] = 0;
    return TCB_OK;
}

extern "C" int tcb_mono_run(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream) {
    int st = validate(m);
    if (st) return st;
    if (step_begin < 1 || step_end > m->nt + 1 || step_begin > step_end)
        return fail(TCB_EINVAL, "tcb_mono_run: step range outside [1, nt]");
    cudaStream_t s = as_stream(stream);
    MonoDev d = make_dev(m);
    const bool fused = step_begin < step_end && uses_fused_step(m, d);
    for (int64_t n = step_begin; n < step_end; ++n) {
        if (fused) {
            st = launch_mono_step(m, d, s);
            if (st < 0) return st;
            if (st == 1) continue;
        }
        st = launch_mono_ionic(m, d, s);
        if (st) return st;
        st = launch_cg(d, s);
        if (st) return st;
    }
    return TCB_OK;
}

extern "C" int tcb_mono_cg_run(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream) {
    int st = validate(m);
    if (st) return st;
    if (step_begin < 1 || step_end > m->nt + 1 || step_begin > step_end)
        return fail(TCB_EINVAL, "tcb_mono_cg_run: step range outside [1, nt]");
    cudaStream_t s = as_stream(stream);
    MonoDev d = make_dev(m);
    for (int64_t n = step_begin; n < step_end; ++n) {
        st = launch_cg(d, s);
        if (st) return st;
    }
    return TCB_OK;
}

extern "C" int tcb_mono_profile(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream,
                                double* ms_ionic, double* ms_cg) {
    int st = validate(m);
    if (st) return st;
    if (!ms_ionic || !ms_cg) return fail(TCB_EINVAL, "tcb_mono_profile: null output");
    if (step_begin < 1 || step_end > m->nt + 1 || step_begin > step_end)
        return fail(TCB_EINVAL, "tcb_mono_profile: step range outside [1, nt]");
    cudaStream_t s = as_stream(stream);
    MonoDev d = make_dev(m);
    const int64_t count = step_end - step_begin;
    if (count == 0) return TCB_OK;
    std::vector<cudaEvent_t> ev(3 * count);
    for (auto& e : ev) TCB_CHECK_CUDA(cudaEventCreate(&e));
    int rc = TCB_OK;
    const bool fused = uses_fused_step(m, d);
    for (int64_t i = 0; i < count && rc == TCB_OK; ++i) {
        cudaEventRecord(ev[3 * i], s);
        if (!fused) {
            rc = launch_mono_ionic(m, d, s);
            if (rc) break;
        }
        cudaEventRecord(ev[3 * i + 1], s);
        if (fused) {
            rc = launch_mono_step(m, d, s);
            rc = rc == 1 ? TCB_OK : rc < 0 ? rc : fail(TCB_EINVAL, "fused step not applicable");
        } else {
            rc = launch_cg(d, s);
        }
        cudaEventRecord(ev[3 * i + 2], s);
    }
    if (rc == TCB_OK) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "tcb_mono_profile sync");
    }
    for (int64_t i = 0; i < count && rc == TCB_OK; ++i) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]);
        cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]);
        *ms_ionic += a;
        *ms_cg += b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

extern "C" int tcb_mono_cg_kernel(const tcb_mono* m) {
    int st = validate(m);
    if (st) return st;
    const MonoDev d = make_dev(m);
    if (uses_fused_step(m, d)) return 2;
    return cg_uses_resident(d) ? 1 : 0;
}

extern "C" int tcb_mono_finish(const tcb_mono* m, void* stream) {
    int st = validate(m);
    if (st) return st;
    return launch_mono_finish(make_dev(m), as_stream(stream));
}

extern "C" int tcb_mono_check(const tcb_mono* m, void* stream) {
    if (!m || !m->counter) return fail(TCB_EINVAL, "tcb_mono_check: null");
    cudaStream_t s = as_stream(stream);
    int32_t host[2] = {0, 0};
    TCB_CHECK_CUDA(cudaMemcpyAsync(host, m->counter, sizeof host, cudaMemcpyDeviceToHost, s));
    TCB_CHECK_CUDA(cudaStreamSynchronize(s));
    if (host[1] == TCB_ETIMEOUT) return fail(TCB_ETIMEOUT, "a bounded wait (grid barrier) of the CG kernel timed out");
    if (host[1] != 0) return fail(host[1], "device error word set");
    return TCB_OK;
}
