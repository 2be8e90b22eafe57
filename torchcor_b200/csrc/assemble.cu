// P1 assembly on the device: element matrices, deterministic gather into CSR
// values, the monodomain system values and the sliced-ELL repack.
//
// Element kernels follow torchcor/core/assemble.py (Matrices3D :148-248,
// Matrices3DSurface :99-145).  The reference forms the local matrices in the
// simulation dtype with batched LU-based det/inv; here each element is one
// thread working in float64 from the float32 coordinates (closed-form
// determinant and adjugate), rounded to float32 once at the end.
#include <cuda_runtime.h>

#include "tcb_internal.h"

namespace {

constexpr int kThreads = 256;

// sigma = st*I + ((sl - st)*f_a)*f_b in float32, as conductivity.py:64-67
// (the outer product there is a batched matmul of single products).
__device__ inline void conductivity_tensor(float sl, float st, const float* f, double s[3][3]) {
    float d = sl - st;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            float o = __fmul_rn(__fmul_rn(d, f[a]), f[b]);
            float v = __fadd_rn(a == b ? st : 0.0f, o);
            s[a][b] = (double)v;
        }
}

__global__ void tet_local_kernel(const float* __restrict__ nodes, const int32_t* __restrict__ elems, int64_t E,
                                 const float* __restrict__ sl, const float* __restrict__ st,
                                 const float* __restrict__ fib, float* __restrict__ ke, float* __restrict__ mw) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double x[4][3];
    for (int a = 0; a < 4; ++a) {
        int32_t v = elems[e * 4 + a];
        for (int c = 0; c < 3; ++c) x[a][c] = (double)nodes[(int64_t)v * 3 + c];
    }
    // J[:, c] = x_{c+1} - x_0  (assemble.py:163-169)
    double J[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) J[r][c] = x[c + 1][r] - x[0][r];
    double C00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    double C01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    double C02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    double det = J[0][0] * C00 + J[0][1] * C01 + J[0][2] * C02;
    // inverse = adj / det
    double inv[3][3];
    inv[0][0] = C00 / det;
    inv[1][0] = C01 / det;
    inv[2][0] = C02 / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    // G = dN @ inv(J): row 0 = -(sum of rows), row a = inv row a-1
    double G[4][3];
    for (int c = 0; c < 3; ++c) {
        G[1][c] = inv[0][c];
        G[2][c] = inv[1][c];
        G[3][c] = inv[2][c];
        G[0][c] = -(inv[0][c] + inv[1][c] + inv[2][c]);
    }
    double s[3][3];
    conductivity_tensor(sl[e], st[e], fib + e * 3, s);
    double adet = fabs(det);
    // vol = |det([1|X])|/6 equals |det J|/6 (assemble.py:194-200); Me = vol/20 * (1 + delta)
    float vol = __fdiv_rn((float)adet, 6.0f);
    mw[e] = __fdiv_rn(vol, 20.0f);
    double scale = adet / 6.0;
    double GS[4][3];
    for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 3; ++c) GS[a][c] = G[a][0] * s[0][c] + G[a][1] * s[1][c] + G[a][2] * s[2][c];
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
            double v = GS[a][0] * G[b][0] + GS[a][1] * G[b][1] + GS[a][2] * G[b][2];
            ke[e * 16 + a * 4 + b] = (float)(scale * v);
        }
}

__global__ void tri_local_kernel(const float* __restrict__ nodes, const int32_t* __restrict__ elems, int64_t E,
                                 const float* __restrict__ sl, const float* __restrict__ st,
                                 const float* __restrict__ fib, float* __restrict__ ke, float* __restrict__ mw) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double x[3][3];
    for (int a = 0; a < 3; ++a) {
        int32_t v = elems[e * 3 + a];
        for (int c = 0; c < 3; ++c) x[a][c] = (double)nodes[(int64_t)v * 3 + c];
    }
    double u1[3], u2[3];
    for (int c = 0; c < 3; ++c) {
        u1[c] = x[1][c] - x[0][c];
        u2[c] = x[2][c] - x[0][c];
    }
    // area = |u1 x u2| / 2 (assemble.py:123-130); Me = area/12 * (1 + delta)
    double cr0 = u1[1] * u2[2] - u1[2] * u2[1];
    double cr1 = u1[2] * u2[0] - u1[0] * u2[2];
    double cr2 = u1[0] * u2[1] - u1[1] * u2[0];
    float area = (float)(0.5 * sqrt(cr0 * cr0 + cr1 * cr1 + cr2 * cr2));
    mw[e] = __fdiv_rn(area, 12.0f);
    // in-plane orthonormal frame (assemble.py:103-113)
    double n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    double al[3] = {u1[0] / n1, u1[1] / n1, u1[2] / n1};
    double pr = u2[0] * al[0] + u2[1] * al[1] + u2[2] * al[2];
    double be[3] = {u2[0] - pr * al[0], u2[1] - pr * al[1], u2[2] - pr * al[2]};
    double n2 = sqrt(be[0] * be[0] + be[1] * be[1] + be[2] * be[2]);
    for (int c = 0; c < 3; ++c) be[c] /= n2;
    double s[3][3];
    conductivity_tensor(sl[e], st[e], fib + e * 3, s);
    // sigma2 = R sigma R^T (2x2), R rows = (alpha, beta)  (assemble.py:134)
    const double* R[2] = {al, be};
    double s2[2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
            double acc = 0.0;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) acc += R[i][a] * s[a][b] * R[j][b];
            s2[i][j] = acc;
        }
    // J = R X^T dN: columns are the edges in the local frame (assemble.py:115-121)
    double J[2][2];
    J[0][0] = al[0] * u1[0] + al[1] * u1[1] + al[2] * u1[2];
    J[1][0] = be[0] * u1[0] + be[1] * u1[1] + be[2] * u1[2];
    J[0][1] = al[0] * u2[0] + al[1] * u2[1] + al[2] * u2[2];
    J[1][1] = be[0] * u2[0] + be[1] * u2[1] + be[2] * u2[2];
    double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    double inv[2][2] = {{J[1][1] / det, -J[0][1] / det}, {-J[1][0] / det, J[0][0] / det}};
    double G[3][2];
    for (int c = 0; c < 2; ++c) {
        G[1][c] = inv[0][c];
        G[2][c] = inv[1][c];
        G[0][c] = -(inv[0][c] + inv[1][c]);
    }
    double scale = 0.5 * det;  // signed, as assemble.py:143
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double v = 0.0;
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j) v += G[a][i] * s2[i][j] * G[b][j];
            ke[e * 9 + a * 3 + b] = (float)(scale * v);
        }
}

// slot-parallel, contributions summed in float32 in the reference COO order
template <int K>
__global__ void gather_kernel(const int32_t* __restrict__ slot_ptr, const int32_t* __restrict__ slot_src,
                              int64_t nnz, const float* __restrict__ ke, const float* __restrict__ mw,
                              float* __restrict__ kval, float* __restrict__ mval) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nnz) return;
    int32_t q0 = slot_ptr[s], q1 = slot_ptr[s + 1];
    float ks = 0.0f, ms = 0.0f;
    for (int32_t q = q0; q < q1; ++q) {
        int32_t src = slot_src[q];
        int32_t e = src / (K * K);
        int32_t ab = src - e * (K * K);
        float m = mw[e];
        float mv = (ab / K == ab % K) ? __fmul_rn(m, 2.0f) : m;
        if (q == q0) {
            ks = ke[src];
            ms = mv;
        } else {
            ks = __fadd_rn(ks, ke[src]);
            ms = __fadd_rn(ms, mv);
        }
    }
    kval[s] = ks;
    mval[s] = ms;
}

__global__ void system_kernel(int64_t nnz, float* __restrict__ kval, const float* __restrict__ mval, float chi,
                              float cm, float dt, float theta, float rhs_scale, float* __restrict__ aval,
                              float* __restrict__ krhs, int32_t* a_split) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nnz) return;
    float k = __fdiv_rn(kval[s], chi);                                    // K / chi   (monodomain.py:93)
    kval[s] = k;
    const float mc = __fmul_rn(mval[s], cm);
    const float a = __fadd_rn(mc, __fmul_rn(__fmul_rn(k, dt), theta));  // :96
    const float kr = __fmul_rn(k, rhs_scale);                             // ((1-theta)*dt)*K  (:131)
    aval[s] = a;
    krhs[s] = kr;
    if (a_split && __fadd_rn(mc, kr) != a) atomicAnd(a_split, 0);
}

__global__ void jacobi_kernel(int64_t n, int64_t n_pad, const int32_t* __restrict__ diag,
                              const float* __restrict__ aval, float* __restrict__ dinv) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    dinv[i] = i < n ? __fdiv_rn(1.0f, aval[diag[i]]) : 0.0f;   // preconditioner.py:27
}

struct SellVals {
    const float* in[4];
    float* out[4];
};

__global__ void sell_pack_kernel(int64_t n_rows, int64_t n_slices, const int32_t* __restrict__ rowptr,
                                 const int32_t* __restrict__ col, const int64_t* __restrict__ slice_ptr, int nv,
                                 SellVals v, int32_t* __restrict__ scol) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t s = t / TCB_SLICE;
    int lane = (int)(t % TCB_SLICE);
    if (s >= n_slices) return;
    int64_t row = s * TCB_SLICE + lane;
    int64_t base = slice_ptr[s];
    int32_t w = (int32_t)((slice_ptr[s + 1] - base) / TCB_SLICE);
    int32_t b = 0, len = 0;
    if (row < n_rows) {
        b = rowptr[row];
        len = rowptr[row + 1] - b;
    }
    for (int32_t k = 0; k < w; ++k) {
        int64_t e = base + (int64_t)k * TCB_SLICE + lane;
        bool real = k < len;
        scol[e] = real ? col[b + k] : (row < n_rows ? (int32_t)row : 0);
        for (int j = 0; j < nv; ++j) v.out[j][e] = real ? v.in[j][b + k] : 0.0f;
    }
}

__global__ void sell_delta_kernel(int64_t n_rows, int64_t n_slices, const int64_t* __restrict__ slice_ptr,
                                  const int32_t* __restrict__ scol, int16_t* __restrict__ delta, int32_t* max_abs) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t s = t / TCB_SLICE;
    int lane = (int)(t % TCB_SLICE);
    if (s >= n_slices) return;
    int64_t row = s * TCB_SLICE + lane;
    int64_t base = slice_ptr[s];
    int32_t w = (int32_t)((slice_ptr[s + 1] - base) / TCB_SLICE);
    int32_t m = 0;
    for (int32_t k = 0; k < w; ++k) {
        int64_t e = base + (int64_t)k * TCB_SLICE + lane;
        int64_t dlt = row < n_rows ? (int64_t)scol[e] - row : 0;
        int64_t a = dlt < 0 ? -dlt : dlt;
        if (a > m) m = a > INT32_MAX ? INT32_MAX : (int32_t)a;
        delta[e] = (int16_t)(a < 32768 ? dlt : 0);
    }
    atomicMax(max_abs, m);   // integer maximum: order-independent
}

inline unsigned blocks_for(int64_t n) { return (unsigned)tcb::ceil_div(n, kThreads); }

}  // namespace

extern "C" int tcb_assemble_local(int32_t k, const float* nodes, const int32_t* elems, int64_t E, const float* sl,
                                  const float* st, const float* fibres, float* ke, float* mw, void* stream) {
    if ((k != 3 && k != 4) || !nodes || !elems || !sl || !st || !fibres || !ke || !mw || E <= 0)
        return tcb::fail(TCB_EINVAL, "tcb_assemble_local: bad arguments");
    cudaStream_t s = tcb::as_stream(stream);
    if (k == 4)
        tet_local_kernel<<<blocks_for(E), kThreads, 0, s>>>(nodes, elems, E, sl, st, fibres, ke, mw);
    else
        tri_local_kernel<<<blocks_for(E), kThreads, 0, s>>>(nodes, elems, E, sl, st, fibres, ke, mw);
    TCB_CHECK_LAUNCH("element kernel");
    return TCB_OK;
}

extern "C" int tcb_assemble_gather(int32_t k, const int32_t* slot_ptr, const int32_t* slot_src, int64_t nnz,
                                   const float* ke, const float* mw, float* k_val, float* m_val, void* stream) {
    if ((k != 3 && k != 4) || !slot_ptr || !slot_src || !ke || !mw || !k_val || !m_val || nnz <= 0)
        return tcb::fail(TCB_EINVAL, "tcb_assemble_gather: bad arguments");
    cudaStream_t s = tcb::as_stream(stream);
    if (k == 4)
        gather_kernel<4><<<blocks_for(nnz), kThreads, 0, s>>>(slot_ptr, slot_src, nnz, ke, mw, k_val, m_val);
    else
        gather_kernel<3><<<blocks_for(nnz), kThreads, 0, s>>>(slot_ptr, slot_src, nnz, ke, mw, k_val, m_val);
    TCB_CHECK_LAUNCH("gather kernel");
    return TCB_OK;
}

extern "C" int tcb_assemble_system(int64_t nnz, int64_t n, int64_t n_pad, const int32_t* diag, float* k_val,
                                   const float* m_val, double chi, double cm, double dt, double theta, float* a_val,
                                   float* k_rhs, float* d_inv, int32_t* a_split, void* stream) {
    if (!diag || !k_val || !m_val || !a_val || !k_rhs || !d_inv || nnz <= 0 || n <= 0 || n_pad < n)
        return tcb::fail(TCB_EINVAL, "tcb_assemble_system: bad arguments");
    cudaStream_t s = tcb::as_stream(stream);
    // Python-level scalars meet float32 tensors: each is rounded to float32 first
    system_kernel<<<blocks_for(nnz), kThreads, 0, s>>>(nnz, k_val, m_val, (float)chi, (float)cm, (float)dt,
                                                        (float)theta, (float)((1.0 - theta) * dt), a_val, k_rhs,
                                                        a_split);
    TCB_CHECK_LAUNCH("system kernel");
    jacobi_kernel<<<blocks_for(n_pad), kThreads, 0, s>>>(n, n_pad, diag, a_val, d_inv);
    TCB_CHECK_LAUNCH("jacobi kernel");
    return TCB_OK;
}

extern "C" int tcb_sell_delta(int64_t n_rows, const int64_t* slice_ptr, int64_t n_slices, const int32_t* sell_col,
                              int16_t* delta, int32_t* max_abs, void* stream) {
    if (!slice_ptr || !sell_col || !delta || !max_abs || n_rows <= 0 || n_slices != tcb::ceil_div(n_rows, TCB_SLICE))
        return tcb::fail(TCB_EINVAL, "tcb_sell_delta: bad arguments");
    sell_delta_kernel<<<blocks_for(n_slices * TCB_SLICE), kThreads, 0, tcb::as_stream(stream)>>>(
        n_rows, n_slices, slice_ptr, sell_col, delta, max_abs);
    TCB_CHECK_LAUNCH("sell delta kernel");
    return TCB_OK;
}

extern "C" int tcb_sell_pack(int64_t n_rows, const int32_t* rowptr, const int32_t* col, const int64_t* slice_ptr,
                             int64_t n_slices, int32_t n_vals, const float* const* vals, int32_t* sell_col,
                             float* const* sell_vals, void* stream) {
    if (!rowptr || !col || !slice_ptr || !sell_col || n_vals < 0 || n_vals > 4 || n_rows <= 0 ||
        n_slices != tcb::ceil_div(n_rows, TCB_SLICE))
        return tcb::fail(TCB_EINVAL, "tcb_sell_pack: bad arguments");
    SellVals v{};
    for (int j = 0; j < n_vals; ++j) {
        if (!vals[j] || !sell_vals[j]) return tcb::fail(TCB_EINVAL, "tcb_sell_pack: null value array");
        v.in[j] = vals[j];
        v.out[j] = sell_vals[j];
    }
    cudaStream_t s = tcb::as_stream(stream);
    sell_pack_kernel<<<blocks_for(n_slices * TCB_SLICE), kThreads, 0, s>>>(n_rows, n_slices, rowptr, col, slice_ptr,
                                                                           n_vals, v, sell_col);
    TCB_CHECK_LAUNCH("sell pack kernel");
    return TCB_OK;
}
