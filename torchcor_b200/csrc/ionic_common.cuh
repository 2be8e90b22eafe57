// Arithmetic helpers shared by the ionic-model kernels.
//
// Two fidelity levels.  The lookup tables (built once per simulation; tables.cu,
// compiled with -fmad=false) reproduce the float32 operation order of the
// reference's PyTorch expressions with separate roundings:
//  * a Python float meeting a float32 tensor is rounded to float32 first;
//  * `python_float / tensor` is evaluated by PyTorch as
//    `tensor.reciprocal() * python_float` -> sdiv() below;
//  * `tensor / python_float` is a true division by the rounded float.
// Their grids pass through removable singularities where the last ulp decides
// between a finite value and NaN, so they keep IEEE division.
// The per-step updates (every node, every step) keep the reference's order of
// operations but let the compiler fuse multiply-adds, and take their division
// and logarithm from a policy (QFast or QExact below): a few ulp per operation,
// far inside the 1e-3 membrane-potential tolerance.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace tcb {

// number of comma-separated names in a parameter list (compile-time check
// that a model's raw-parameter struct matches the names the host passes)
constexpr int count_names(const char* s) {
    int n = 1;
    for (; *s; ++s) n += (*s == ',');
    return n;
}

#define TCB_HD __host__ __device__ __forceinline__

// python_float / tensor
TCB_HD float sdiv(float s, float t) { return (1.0f / t) * s; }

// Division and logarithm of the per-step updates, as a compile-time policy of
// each kernel instance:
//  * QFast: __fdividef (a times the hardware reciprocal of b, within 2 ulp for
//    |b| below 2^126; every denominator here is far smaller) and __logf
//    (absolute error below 2^-21.4 on [0.5, 2], a few ulp elsewhere; the
//    arguments are positive concentration ratios).  Fewest instructions, but the
//    compiler then schedules the table gathers far ahead, so it pays only with a
//    large register budget.
//  * QExact: IEEE division and logf, python_float / tensor as reciprocal times
//    the float (PyTorch's order).  Under a tight register budget it spills far
//    less.
struct QFast {
    static TCB_HD float div(float a, float b) {
#ifdef __CUDA_ARCH__
        return __fdividef(a, b);
#else
        return a / b;
#endif
    }
    static TCB_HD float sdiv(float s, float t) { return div(s, t); }
    static TCB_HD float log(float x) {
#ifdef __CUDA_ARCH__
        return __logf(x);
#else
        return logf(x);
#endif
    }
};
struct QExact {
    static TCB_HD float div(float a, float b) { return a / b; }
    static TCB_HD float sdiv(float s, float t) { return (1.0f / t) * s; }
    static TCB_HD float log(float x) { return logf(x); }
};

// torch.clamp(X, mn, mx) with NaN propagation
TCB_HD float tclamp(float x, float mn, float mx) {
    x = (x < mn) ? mn : x;
    return (x > mx) ? mx : x;
}

// Lookup table with the reference's linear interpolation
// (TenTusscherPanfilov.py:188-195, CourtemancheRamirezNattel.py:203-210).
struct Lut {
    const float* tab;   // rows x stride floats, row-major (stride = ncol rounded up to 4, or 1)
    float mn, mx, res, step;
    int32_t mx_idx;
};

struct LutPos {
    int32_t lo;
    float w, w1;  // w, 1 - w
};

template <class Q>
TCB_HD LutPos lut_pos(float X, const Lut& L) {
    X = tclamp(X, L.mn, L.mx);
    float f = (X - L.mn) * L.step;   // X is clamped, so 0 <= f <= rows: 32-bit is enough
    int idx = (f != f) ? 0 : (int)f;  // .to(torch.long) truncates
    idx = idx < 0 ? 0 : idx;
    idx = idx > L.mx_idx - 1 ? L.mx_idx - 1 : idx;
    float lo_pos = (float)idx * L.res + L.mn;
    float w = Q::div(X - lo_pos, L.res);
    LutPos p;
    p.lo = (int32_t)idx;
    p.w = w;
    p.w1 = 1.0f - w;
    return p;
}

TCB_HD float ldro(const float* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

__host__ __device__ constexpr int lut_stride(int ncol) { return ncol == 1 ? 1 : (ncol + 3) / 4 * 4; }

// one column of the interpolated row: (1 - w) * T[lo] + w * T[lo + 1]
template <int NCOL>
TCB_HD float lut_col(const Lut& L, const LutPos& p, int c) {
    constexpr int S = lut_stride(NCOL);
    const float* r0 = L.tab + (int64_t)p.lo * S;
    return p.w1 * ldro(r0 + c) + p.w * ldro(r0 + S + c);
}

// columns c and c + 1 (c even) of the interpolated row, each table row read as one
// 8-byte vector; the table starts 16-byte aligned and its stride is even, so the
// pair is 8-byte aligned.  Same arithmetic as two lut_col calls.
template <int NCOL>
TCB_HD float2 lut_pair(const Lut& L, const LutPos& p, int c) {
    constexpr int S = lut_stride(NCOL);
    static_assert(S % 2 == 0, "paired columns need an even stride");
    const float* r0 = L.tab + (int64_t)p.lo * S + c;
#ifdef __CUDA_ARCH__
    const float2 a = __ldg(reinterpret_cast<const float2*>(r0));
    const float2 b = __ldg(reinterpret_cast<const float2*>(r0 + S));
#else
    const float2 a = make_float2(r0[0], r0[1]);
    const float2 b = make_float2(r0[S], r0[S + 1]);
#endif
    return make_float2(p.w1 * a.x + p.w * b.x, p.w1 * a.y + p.w * b.y);
}

// host-side helpers describing a table the way the reference does
struct LutSpec {
    double mn, mx, res;
    int ncol;
    int stride() const { return lut_stride(ncol); }
    int64_t floats() const { return rows() * stride(); }
    int64_t rows() const;       // torch.arange(mn, mx, res).shape[0]
    int32_t mx_idx() const;     // int((mx - mn) * (1/res)) - 1
    Lut make(const float* tab) const;
};

}  // namespace tcb
