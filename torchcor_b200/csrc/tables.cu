// Lookup-table construction and initial state of the ionic models
// (construct_tables / initialize of TenTusscherPanfilov.py:197-351,
// CourtemancheRamirezNattel.py:212-357, ModifiedMS2v.py:31-34).
//
// Compiled with -fmad=false and IEEE division: the table formulas are
// evaluated in the reference's float32 operation order with separate
// roundings, on the reference's float32 grid, because the grids pass through
// removable singularities where the last ulp decides between a finite entry
// and NaN.  The per-step kernels that read the tables are in ionic.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "ionic_crn.cuh"
#include "ionic_ms.cuh"
#include "ionic_ttp.cuh"
#include "tcb_internal.h"

namespace tcb {

int64_t LutSpec::rows() const { return (int64_t)ceil((mx - mn) / res); }
int32_t LutSpec::mx_idx() const { return (int32_t)((mx - mn) * (1.0 / res)) - 1; }
Lut LutSpec::make(const float* tab) const {
    Lut L;
    L.tab = tab;
    L.mn = (float)mn;
    L.mx = (float)mx;
    L.res = (float)res;
    L.step = (float)(1.0 / res);
    L.mx_idx = mx_idx();
    return L;
}

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) {
    int64_t b = ceil_div(n, kThreads);
    return (unsigned)(b > 148 * 64 ? 148 * 64 : b);
}

// ------------------------------------------------------------- tables
// Grid value of row i of a table built on torch.arange(mn, mx, res) in
// float32 on the CPU, as PyTorch's CPU kernel forms it: the range is split
// into chunks of max(32768, ceil(rows/8)) (its parallel grain on the 8-thread
// host the reference fixtures come from); inside a chunk, whole 16-element
// groups are vectorised as 8-wide vectors whose first element is
// float(fma(res, i0, mn)) and whose element k is float(fma(k, res, first));
// the remaining elements take float(fma(res, i, mn)).  The exact grid matters
// at removable singularities of the table formulas (e.g. V = 7.9 in CRN tau_w).
__device__ inline float grid_value(double mn, double res, int64_t i, int64_t rows) {
    const int64_t chunk = rows / 8 + (rows % 8 != 0) > 32768 ? rows / 8 + (rows % 8 != 0) : 32768;
    const int64_t cb = (i / chunk) * chunk;
    const int64_t ce = cb + chunk < rows ? cb + chunk : rows;
    const int64_t vec_end = cb + ((ce - cb) / 16) * 16;
    if (i < vec_end) {
        const int64_t i0 = cb + ((i - cb) / 8) * 8;
        const float base = (float)__fma_rn(res, (double)i0, mn);
        return (float)__fma_rn((double)(i - i0), res, (double)base);
    }
    return (float)__fma_rn(res, (double)i, mn);
}

__global__ void ttp_v_table(TTP::C c, float* tab, int64_t rows, double mn, double res) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
        float o[TV_NCOL];
        TTP::v_row(grid_value(mn, res, i, rows), c, o);
        constexpr int S = lut_stride(TV_NCOL);
        for (int k = 0; k < S; ++k) tab[i * S + k] = k < TV_NCOL ? o[k] : 0.0f;
    }
}
__global__ void ttp_cass_table(TTP::C c, float* tab, int64_t rows, double mn, double res) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
        float o[3];
        TTP::cass_row(grid_value(mn, res, i, rows), c, o);
        constexpr int S = lut_stride(3);
        for (int k = 0; k < S; ++k) tab[i * S + k] = k < 3 ? o[k] : 0.0f;
    }
}
__global__ void ttp_vek_table(float* tab, int64_t rows, double mn, double res) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x)
        tab[i] = TTP::vek_row(grid_value(mn, res, i, rows));
}
__global__ void crn_v_table(CRN::C c, float* tab, int64_t rows, double mn, double res) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
        float o[CV_NCOL];
        CRN::v_row(grid_value(mn, res, i, rows), c, o);
        constexpr int S = lut_stride(CV_NCOL);
        for (int k = 0; k < S; ++k) tab[i * S + k] = k < CV_NCOL ? o[k] : 0.0f;
    }
}
__global__ void crn_cai_table(CRN::C c, float* tab, int64_t rows, double mn, double res) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
        float o[CC_NCOL];
        CRN::cai_row(grid_value(mn, res, i, rows), c, o);
        constexpr int S = lut_stride(CC_NCOL);
        for (int k = 0; k < S; ++k) tab[i * S + k] = k < CC_NCOL ? o[k] : 0.0f;
    }
}
__global__ void crn_fn_table(CRN::C c, float* tab, int64_t rows, double mn, double res) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
        float o[3];
        CRN::fn_row(grid_value(mn, res, i, rows), c, o);
        constexpr int S = lut_stride(3);
        for (int k = 0; k < S; ++k) tab[i * S + k] = k < 3 ? o[k] : 0.0f;
    }
}

// ------------------------------------------------------------- initial state
template <class M>
__global__ void init_kernel(typename M::C c, float* state, int64_t n_pad, float* v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += (int64_t)gridDim.x * blockDim.x) {
        float s[M::kStates];
        float V;
        M::init(c, s, V);
        for (int k = 0; k < M::kStates; ++k) state[k * n_pad + i] = s[k];
        if (v) v[i] = V;
    }
}

template <class M>
int run_init(const double* params, float* state, int64_t n_pad, float* v, cudaStream_t s) {
    init_kernel<M><<<grid_for(n_pad), kThreads, 0, s>>>(M::derive(params), state, n_pad, v);
    TCB_CHECK_LAUNCH("init kernel");
    return TCB_OK;
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" const char* tcb_model_params(int32_t model) {
    switch (model) {
        case TCB_MODEL_MS: return TCB_MS_PARAMS;
        case TCB_MODEL_TTP: return TCB_TTP_PARAMS;
        case TCB_MODEL_CRN: return TCB_CRN_PARAMS;
    }
    return nullptr;
}

extern "C" const char* tcb_model_states(int32_t model) {
    switch (model) {
        case TCB_MODEL_MS: return TCB_MS_STATES;
        case TCB_MODEL_TTP: return TCB_TTP_STATES;
        case TCB_MODEL_CRN: return TCB_CRN_STATES;
    }
    return nullptr;
}

extern "C" int tcb_model_layout(int32_t model, const double* params, int64_t* n_states, int64_t* table_floats) {
    if (!n_states || !table_floats) return fail(TCB_EINVAL, "tcb_model_layout: null output");
    switch (model) {
        case TCB_MODEL_MS:
            *n_states = MS::kStates;
            *table_floats = MS::table_floats(params);
            return TCB_OK;
        case TCB_MODEL_TTP:
            *n_states = TTP::kStates;
            *table_floats = TTP::table_floats(params);
            return TCB_OK;
        case TCB_MODEL_CRN:
            *n_states = CRN::kStates;
            *table_floats = CRN::table_floats(params);
            return TCB_OK;
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

extern "C" int tcb_model_table_info(int32_t model, int32_t index, int64_t* rows, int32_t* ncol, int32_t* stride,
                                    int64_t* offset) {
    if (!rows || !ncol || !stride || !offset) return fail(TCB_EINVAL, "tcb_model_table_info: null output");
    const LutSpec* specs[3] = {nullptr, nullptr, nullptr};
    if (model == TCB_MODEL_TTP) {
        specs[0] = &TTP::kV;
        specs[1] = &TTP::kCaSS;
        specs[2] = &TTP::kVEk;
    } else if (model == TCB_MODEL_CRN) {
        specs[0] = &CRN::kV;
        specs[1] = &CRN::kCai;
        specs[2] = &CRN::kFn;
    } else if (model != TCB_MODEL_MS) {
        return fail(TCB_EINVAL, "unknown ionic model");
    }
    if (index < 0 || index > 2 || !specs[index]) return fail(TCB_ERANGE, "no such lookup table");
    int64_t off = 0;
    for (int i = 0; i < index; ++i) off += specs[i]->floats();
    *rows = specs[index]->rows();
    *ncol = specs[index]->ncol;
    *stride = specs[index]->stride();
    *offset = off;
    return TCB_OK;
}

extern "C" int tcb_model_tables(int32_t model, const double* params, float* tables, void* stream) {
    if (!params) return fail(TCB_EINVAL, "tcb_model_tables: null params");
    cudaStream_t s = as_stream(stream);
    if (model == TCB_MODEL_MS) return TCB_OK;
    if (!tables) return fail(TCB_EINVAL, "tcb_model_tables: null tables");
    if ((uintptr_t)tables & 15u) return fail(TCB_EINVAL, "tcb_model_tables: tables not 16-byte aligned");
    if (model == TCB_MODEL_TTP) {
        TTP::C c = TTP::derive(params);
        TTP::Tables T = TTP::tables(tables, params);
        ttp_v_table<<<grid_for(TTP::kV.rows()), kThreads, 0, s>>>(c, const_cast<float*>(T.V.tab), TTP::kV.rows(),
                                                                    TTP::kV.mn, TTP::kV.res);
        ttp_cass_table<<<grid_for(TTP::kCaSS.rows()), kThreads, 0, s>>>(c, const_cast<float*>(T.CaSS.tab),
                                                                          TTP::kCaSS.rows(), TTP::kCaSS.mn,
                                                                          TTP::kCaSS.res);
        ttp_vek_table<<<grid_for(TTP::kVEk.rows()), kThreads, 0, s>>>(const_cast<float*>(T.VEk.tab),
                                                                        TTP::kVEk.rows(), TTP::kVEk.mn, TTP::kVEk.res);
        TCB_CHECK_LAUNCH("TTP table kernels");
        return TCB_OK;
    }
    if (model == TCB_MODEL_CRN) {
        CRN::C c = CRN::derive(params);
        CRN::Tables T = CRN::tables(tables, params);
        crn_v_table<<<grid_for(CRN::kV.rows()), kThreads, 0, s>>>(c, const_cast<float*>(T.V.tab), CRN::kV.rows(),
                                                                    CRN::kV.mn, CRN::kV.res);
        crn_cai_table<<<grid_for(CRN::kCai.rows()), kThreads, 0, s>>>(c, const_cast<float*>(T.Cai.tab),
                                                                        CRN::kCai.rows(), CRN::kCai.mn, CRN::kCai.res);
        crn_fn_table<<<grid_for(CRN::kFn.rows()), kThreads, 0, s>>>(c, const_cast<float*>(T.Fn.tab), CRN::kFn.rows(),
                                                                      CRN::kFn.mn, CRN::kFn.res);
        TCB_CHECK_LAUNCH("CRN table kernels");
        return TCB_OK;
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

extern "C" int tcb_model_init(int32_t model, const double* params, float* state, int64_t n_pad, float* v,
                              void* stream) {
    if (!params || !state || n_pad <= 0) return fail(TCB_EINVAL, "tcb_model_init: bad arguments");
    cudaStream_t s = as_stream(stream);
    switch (model) {
        case TCB_MODEL_MS: return run_init<MS>(params, state, n_pad, v, s);
        case TCB_MODEL_TTP: return run_init<TTP>(params, state, n_pad, v, s);
        case TCB_MODEL_CRN: return run_init<CRN>(params, state, n_pad, v, s);
    }
    return fail(TCB_EINVAL, "unknown ionic model");
}

