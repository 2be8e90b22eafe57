// ModifiedMS2v: dimensional two-variable Mitchell-Schaeffer model
// (torchcor/ionic/ModifiedMS2v.py:4-44).  The product's MitchellSchaeffer
// class uses this arithmetic (the CellML-based MitchellSchaeffer of the
// reference cannot run inside Monodomain).
#pragma once
#include "ionic_common.cuh"

namespace tcb {

struct MSRaw {  // order of tcb_model_params(TCB_MODEL_MS)
    double tau_in, tau_out, tau_open, tau_close, u_gate, u_crit, vmin, vmax, dt;
};
#define TCB_MS_PARAMS "tau_in,tau_out,tau_open,tau_close,u_gate,u_crit,vmin,vmax,dt"
#define TCB_MS_STATES "H"
static_assert(sizeof(MSRaw) == count_names(TCB_MS_PARAMS) * sizeof(double), "MSRaw layout");

struct MS {
    static constexpr int kStates = 1;
    struct C {
        float tau_in, tau_out, tau_open, tau_close, u_gate, u_crit, vmin, DV, dt, H_init, V_init;
    };
    struct Tables {};

    static C derive(const double* p) {
        MSRaw r;
        memcpy(&r, p, sizeof r);
        C c;
        c.tau_in = (float)r.tau_in;
        c.tau_out = (float)r.tau_out;
        c.tau_open = (float)r.tau_open;
        c.tau_close = (float)r.tau_close;
        c.u_gate = (float)r.u_gate;
        c.u_crit = (float)r.u_crit;
        c.vmin = (float)r.vmin;
        c.DV = (float)(r.vmax - r.vmin);
        c.dt = (float)r.dt;
        c.H_init = 1.0f;
        c.V_init = (float)r.vmin;
        return c;
    }
    // no per-node parameters
    static constexpr int kNodeParams = 0;
    struct NodeG {};
    __host__ __device__ static NodeG node_g(const C&, const float*, int64_t, int64_t) { return NodeG{}; }

    static int64_t table_floats(const double*) { return 0; }
    static Tables tables(const float*, const double*) { return Tables{}; }

    __host__ __device__ static void init(const C& c, float* s, float& V) {
        s[0] = c.H_init;
        V = c.V_init;
    }

    // ModifiedMS2v.differentiate (:36-44); returns dU and updates H
    template <class Q>
    __host__ __device__ static float step(float U, float* s, const C& c, const Tables&, const NodeG&) {
        float H = s[0];
        float Uad = (U - c.vmin) / c.DV;
        float J_in = ((((-1.0f * H) * Uad) * (Uad - c.u_crit)) * (1.0f - Uad)) / c.tau_in;
        float J_out = ((1.0f - H) * Uad) / c.tau_out;
        float dU = -(c.DV * (J_in + J_out));
        float dH = (Uad > c.u_gate) ? ((-H) / c.tau_close) : ((1.0f - H) / c.tau_open);
        s[0] = H + c.dt * dH;
        return dU;
    }
};

}  // namespace tcb
