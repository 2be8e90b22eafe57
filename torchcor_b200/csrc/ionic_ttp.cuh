// ten Tusscher-Panfilov 2006 (torchcor/ionic/TenTusscherPanfilov.py:6-454):
// 18 states besides V (6 forward-Euler, 12 Rush-Larsen gates) and three
// lookup tables (V: 27 columns, CaSS: 3, V-Ek: 1).  The conductances GCaL,
// GKr, GKs, Gto are per-node arrays in the reference, filled uniformly by
// initialize(); here they are the scalar parameters *_init.
#pragma once
#include "ionic_common.cuh"

namespace tcb {

struct TTPRaw {  // order of tcb_model_params(TCB_MODEL_TTP)
    double CaSR_init, CaSS_init, Cai_init, EC, F2_init, FCaSS_init, F_init, H_init, J_init, Ki_init, M_init,
        Nai_init, R__init, R_init, S_init, V_init, Vxfer, Xr1_init, Xr2_init, Xs_init, d_init, k1_, k2_, k3, k4,
        maxsr, minsr, Bufc, Bufsr, Bufss, CAPACITANCE, Cao, D_CaL_off, Fconst, GK1, GNa, GbCa, GbNa, GpCa, GpK,
        Kbufc, Kbufsr, Kbufss, KmCa, KmK, KmNa, KmNai, Ko, KpCa, Kup, Nao, Rconst, T, Vc, Vleak, Vmaxup, Vrel,
        Vsr, Vss, knaca, knak, ksat, n, pKNa, scl_tau_f, vHalfXs, xr2_off, GCaL_init, GKr_init, GKs_init,
        Gto_init, endo, dt;
};
#define TCB_TTP_PARAMS                                                                                           \
    "CaSR_init,CaSS_init,Cai_init,EC,F2_init,FCaSS_init,F_init,H_init,J_init,Ki_init,M_init,Nai_init,R__init,"  \
    "R_init,S_init,V_init,Vxfer,Xr1_init,Xr2_init,Xs_init,d_init,k1_,k2_,k3,k4,maxsr,minsr,Bufc,Bufsr,Bufss,"   \
    "CAPACITANCE,Cao,D_CaL_off,Fconst,GK1,GNa,GbCa,GbNa,GpCa,GpK,Kbufc,Kbufsr,Kbufss,KmCa,KmK,KmNa,KmNai,Ko,"   \
    "KpCa,Kup,Nao,Rconst,T,Vc,Vleak,Vmaxup,Vrel,Vsr,Vss,knaca,knak,ksat,n,pKNa,scl_tau_f,vHalfXs,xr2_off,"      \
    "GCaL_init,GKr_init,GKs_init,Gto_init,endo,dt"
#define TCB_TTP_STATES "CaSR,CaSS,Cai,D,F,F2,FCaSS,H,J,Ki,M,Nai,R,R_,S,Xr1,Xr2,Xs"
static_assert(sizeof(TTPRaw) == count_names(TCB_TTP_PARAMS) * sizeof(double), "TTPRaw layout");

// V-table columns (TenTusscherPanfilov.py:98-125)
enum TTPV {
    TV_D_A, TV_D_B, TV_F2_A, TV_F2_B, TV_F_A, TV_F_B, TV_H_A, TV_H_B, TV_INaCa_A, TV_INaCa_B, TV_J_A, TV_J_B,
    TV_M_A, TV_M_B, TV_R_A, TV_R_B, TV_S_A, TV_S_B, TV_Xr1_A, TV_Xr1_B, TV_Xr2_A, TV_Xr2_B, TV_Xs_A, TV_Xs_B,
    TV_a2, TV_rec_iNaK, TV_rec_ipK, TV_NCOL
};
// columns read as pairs (lut_pair): (X_A, X_B) of every V gate, (INaCa_A, INaCa_B) and
// (a2, rec_iNaK); each pair starts at an even column with its partner next to it
static_assert(TV_D_A % 2 == 0 && TV_F2_A % 2 == 0 && TV_F_A % 2 == 0 && TV_H_A % 2 == 0 && TV_INaCa_A % 2 == 0 &&
              TV_J_A % 2 == 0 && TV_M_A % 2 == 0 && TV_R_A % 2 == 0 && TV_S_A % 2 == 0 && TV_Xr1_A % 2 == 0 &&
              TV_Xr2_A % 2 == 0 && TV_Xs_A % 2 == 0 && TV_a2 % 2 == 0 && TV_rec_iNaK == TV_a2 + 1,
              "paired V-table columns");

// Rush-Larsen update x' = A + B * x from the interpolated (A, B) pair
TCB_HD float rl_gate(float2 ab, float x) { return ab.x + ab.y * x; }
enum TTPS { S_CaSR, S_CaSS, S_Cai, S_D, S_F, S_F2, S_FCaSS, S_H, S_J, S_Ki, S_M, S_Nai, S_R, S_R_, S_S, S_Xr1,
            S_Xr2, S_Xs, TTP_NS };

struct TTP {
    static constexpr int kStates = TTP_NS;
    static constexpr LutSpec kV{-800.0, 800.0, 0.05, TV_NCOL};
    static constexpr LutSpec kCaSS{0.00001, 10.0, 0.00001, 3};
    static constexpr LutSpec kVEk{-800.0, 800.0, 0.05, 1};

    struct C {
        // differentiate constants (Python-level expressions rounded to float32 once)
        float halfRTONF, RTONF, Cao, Ko, Nao, KoNa, pKNa, GpCa, KpCa, ga1, halfFRT, F_RT, GKr_sqrtKo, GKs, GNa,
            pmf_INaK, KmNa, GbCa, GbNa, GpK, Gto, GK1, Vleak, Vmaxup, KupKup, Vxfer, invVcF_Cm, maxsr, dsr, EC,
            inverseVcF2, CAP, Vsr_Vc, BufcKbufc, Kbufc, k4, k2_, k1_, k3, Vrel, BufsrKbufsr, Kbufsr, Vc_Vss,
            Vsr_Vss, inverseVssF2, BufssKbufss, Kbufss, dt;
        // per-node conductances from their arrays: ga1 = ((GCaL * Fconst) * F_RT) * 4, GKr * sqrt(Ko/5.4)
        float Fconst, sqrt_Ko;
        // table constants
        float mdt, D_off, xr2c, mvHalf, nm1_FRT_dummy, n_, nm1, ksat, pmf_INaCa, Nao3, scl_tau_f;
        int endo;
        float init[TTP_NS];
        float V_init;
    };
    struct Tables {
        Lut V, CaSS, VEk;
    };

    static C derive(const double* p) {
        TTPRaw r;
        memcpy(&r, p, sizeof r);
        C c;
        double RTONF = (r.Rconst * r.T) / r.Fconst;
        double inverseVcF = 1. / (r.Vc * r.Fconst);
        double inverseVcF2 = 1. / ((2. * r.Vc) * r.Fconst);
        double inverseVssF2 = 1. / ((2. * r.Vss) * r.Fconst);
        double pmf_INaK = r.knak * (r.Ko / (r.Ko + r.KmK));
        double sqrt_Ko = sqrt(r.Ko / 5.4);
        double F_RT = 1. / RTONF;
        double invVcF_Cm = inverseVcF * r.CAPACITANCE;
        c.halfRTONF = (float)(0.5 * RTONF);
        c.RTONF = (float)RTONF;
        c.Cao = (float)r.Cao;
        c.Ko = (float)r.Ko;
        c.Nao = (float)r.Nao;
        c.KoNa = (float)(r.Ko + r.pKNa * r.Nao);
        c.pKNa = (float)r.pKNa;
        c.GpCa = (float)r.GpCa;
        c.KpCa = (float)r.KpCa;
        // ((GCaL*Fconst)*F_RT)*4 with GCaL a float32 tensor: three float32 roundings
        c.ga1 = ((float)r.GCaL_init * (float)r.Fconst * (float)F_RT) * 4.0f;
        c.halfFRT = (float)((1. / 2.) * F_RT);
        c.F_RT = (float)F_RT;
        c.GKr_sqrtKo = (float)r.GKr_init * (float)sqrt_Ko;
        c.Fconst = (float)r.Fconst;
        c.sqrt_Ko = (float)sqrt_Ko;
        c.GKs = (float)r.GKs_init;
        c.GNa = (float)r.GNa;
        c.pmf_INaK = (float)pmf_INaK;
        c.KmNa = (float)r.KmNa;
        c.GbCa = (float)r.GbCa;
        c.GbNa = (float)r.GbNa;
        c.GpK = (float)r.GpK;
        c.Gto = (float)r.Gto_init;
        c.GK1 = (float)r.GK1;
        c.Vleak = (float)r.Vleak;
        c.Vmaxup = (float)r.Vmaxup;
        c.KupKup = (float)(r.Kup * r.Kup);
        c.Vxfer = (float)r.Vxfer;
        c.invVcF_Cm = (float)invVcF_Cm;
        c.maxsr = (float)r.maxsr;
        c.dsr = (float)(r.maxsr - r.minsr);
        c.EC = (float)r.EC;
        c.inverseVcF2 = (float)inverseVcF2;
        c.CAP = (float)r.CAPACITANCE;
        c.Vsr_Vc = (float)(r.Vsr / r.Vc);
        c.BufcKbufc = (float)(r.Bufc * r.Kbufc);
        c.Kbufc = (float)r.Kbufc;
        c.k4 = (float)r.k4;
        c.k2_ = (float)r.k2_;
        c.k1_ = (float)r.k1_;
        c.k3 = (float)r.k3;
        c.Vrel = (float)r.Vrel;
        c.BufsrKbufsr = (float)(r.Bufsr * r.Kbufsr);
        c.Kbufsr = (float)r.Kbufsr;
        c.Vc_Vss = (float)(r.Vc / r.Vss);
        c.Vsr_Vss = (float)(r.Vsr / r.Vss);
        c.inverseVssF2 = (float)inverseVssF2;
        c.BufssKbufss = (float)(r.Bufss * r.Kbufss);
        c.Kbufss = (float)r.Kbufss;
        c.dt = (float)r.dt;
        // construct_tables constants (:198-204)
        double KmNai3 = (r.KmNai * r.KmNai) * r.KmNai;
        double Nao3 = (r.Nao * r.Nao) * r.Nao;
        double invKmCa_Cao = 1. / (r.KmCa + r.Cao);
        double invKmNai3_Nao3 = 1. / (KmNai3 + Nao3);
        c.pmf_INaCa = (float)((r.knaca * invKmNai3_Nao3) * invKmCa_Cao);
        c.Nao3 = (float)Nao3;
        c.mdt = (float)(-r.dt);
        c.D_off = (float)(-8. + r.D_CaL_off);
        c.xr2c = (float)(-88. + r.xr2_off);
        c.mvHalf = (float)(-r.vHalfXs);
        c.n_ = (float)r.n;
        c.nm1 = (float)(r.n - 1.);
        c.ksat = (float)r.ksat;
        c.scl_tau_f = (float)r.scl_tau_f;
        c.endo = r.endo != 0.0;
        c.nm1_FRT_dummy = 0.0f;
        // initial values (:322-351)
        const double init[TTP_NS] = {r.CaSR_init, r.CaSS_init, r.Cai_init, r.d_init, r.F_init, r.F2_init,
                                     r.FCaSS_init, r.H_init, r.J_init, r.Ki_init, r.M_init, r.Nai_init,
                                     r.R_init, r.R__init, r.S_init, r.Xr1_init, r.Xr2_init, r.Xs_init};
        for (int i = 0; i < TTP_NS; ++i) c.init[i] = (float)init[i];
        c.V_init = (float)r.V_init;
        return c;
    }

    // Per-node conductances (the reference's GCaL, GKr, GKs, Gto tensors,
    // TenTusscherPanfilov.py:327-330): rows of tcb_mono.node_params when a caller
    // set them node by node, else the uniform values of the parameters.
    static constexpr int kNodeParams = 4;   // GCaL, GKr, GKs, Gto
    struct NodeG {
        float ga1, GKr_sqrtKo, GKs, Gto;
    };
    __host__ __device__ static NodeG node_g(const C& c, const float* np, int64_t n_pad, int64_t i) {
        if (!np) return NodeG{c.ga1, c.GKr_sqrtKo, c.GKs, c.Gto};
        NodeG g;
        // ((GCaL * Fconst) * F_RT) * 4. and GKr * sqrt_Ko: float32 tensor times Python floats (:374, :377)
        g.ga1 = ((np[i] * c.Fconst) * c.F_RT) * 4.0f;
        g.GKr_sqrtKo = np[n_pad + i] * c.sqrt_Ko;
        g.GKs = np[2 * n_pad + i];
        g.Gto = np[3 * n_pad + i];
        return g;
    }

    static int64_t table_floats(const double*) {
        return kV.floats() + kCaSS.floats() + kVEk.floats();
    }
    static Tables tables(const float* t, const double*) {
        Tables T;
        T.V = kV.make(t);
        T.CaSS = kCaSS.make(t + kV.floats());
        T.VEk = kVEk.make(t + kV.floats() + kCaSS.floats());
        return T;
    }

    // -------------------------------------------------------- tables (:197-318)
    __host__ __device__ static void cass_row(float cs, const C& c, float* out) {
        float q = cs / 0.05f;
        float q2 = q * q;
        float FCaSS_inf = sdiv(0.6f, 1.0f + q2) + 0.4f;
        float tau = sdiv(80.0f, 1.0f + q2) + 2.0f;
        float e = sdiv(c.mdt, tau);
        out[0] = 0.0f;  // CaSS2 column: never written by the reference (stays zero)
        out[2] = expf(e);
        out[1] = (-FCaSS_inf) * expm1f(e);
    }

    __host__ __device__ static void v_row(float V, const C& c, float* o) {
        float D_inf = sdiv(1.0f, 1.0f + expf((c.D_off - V) / 7.5f));
        float F2_inf = sdiv(0.67f, 1.0f + expf((V + 35.0f) / 7.0f)) + 0.33f;
        float F_inf = sdiv(1.0f, 1.0f + expf((V + 20.0f) / 7.0f));
        float eh = 1.0f + expf((V + 71.55f) / 7.43f);
        float H_inf = sdiv(1.0f, eh * eh);
        float em = 1.0f + expf((-56.86f - V) / 9.03f);
        float M_inf = sdiv(1.0f, em * em);
        float R_inf = sdiv(1.0f, 1.0f + expf((20.0f - V) / 6.0f));
        float S_inf = sdiv(1.0f, 1.0f + expf((V + 20.0f) / 5.0f));
        float Xr1_inf = sdiv(1.0f, 1.0f + expf((-26.0f - V) / 7.0f));
        float Xr2_inf = sdiv(1.0f, 1.0f + expf((V - c.xr2c) / 24.0f));
        float Xs_inf = sdiv(1.0f, 1.0f + expf((c.mvHalf - V) / 14.0f));
        o[TV_a2] = 0.25f * expf((2.0f * (V - 15.0f)) * c.F_RT);
        float aa_D = sdiv(1.4f, 1.0f + expf((-35.0f - V) / 13.0f)) + 0.25f;
        float v27 = V + 27.0f;
        float aa_F = 1102.5f * expf(((-v27) * v27) / 225.0f);
        float aa_F2 = 562.0f * expf(((-v27) * v27) / 240.0f);
        float aa_H = (V >= -40.0f) ? 0.0f : 0.057f * expf((-(V + 80.0f)) / 6.8f);
        float aa_J = (V >= -40.0f)
                         ? 0.0f
                         : (((-2.5428e4f * expf(0.2444f * V)) - (6.948e-6f * expf(-0.04391f * V))) * (V + 37.78f)) /
                               (1.0f + expf(0.311f * (V + 79.23f)));
        float aa_M = sdiv(1.0f, 1.0f + expf((-60.0f - V) / 5.0f));
        float aa_Xr1 = sdiv(450.0f, 1.0f + expf((-45.0f - V) / 10.0f));
        float aa_Xr2 = sdiv(3.0f, 1.0f + expf((-60.0f - V) / 20.0f));
        float aa_Xs = sdiv(1400.0f, sqrtf(1.0f + expf((5.0f - V) / 6.0f)));
        float bb_D = sdiv(1.4f, 1.0f + expf((V + 5.0f) / 5.0f));
        float bb_F = sdiv(200.0f, 1.0f + expf((13.0f - V) / 10.0f));
        float bb_F2 = sdiv(31.0f, 1.0f + expf((25.0f - V) / 10.0f));
        float bb_H = (V >= -40.0f) ? sdiv(0.77f, 0.13f * (1.0f + expf((-(V + 10.66f)) / 11.1f)))
                                   : (2.7f * expf(0.079f * V)) + (3.1e5f * expf(0.3485f * V));
        float bb_J = (V >= -40.0f) ? (0.6f * expf(0.057f * V)) / (1.0f + expf(-0.1f * (V + 32.0f)))
                                   : (0.02424f * expf(-0.01052f * V)) / (1.0f + expf(-0.1378f * (V + 40.14f)));
        float bb_M = sdiv(0.1f, 1.0f + expf((V + 35.0f) / 5.0f)) + sdiv(0.10f, 1.0f + expf((V - 50.0f) / 200.0f));
        float bb_Xr1 = sdiv(6.0f, 1.0f + expf((V - (-30.0f)) / 11.5f));
        float bb_Xr2 = sdiv(1.12f, 1.0f + expf((V - 60.0f) / 20.0f));
        float bb_Xs = sdiv(1.0f, 1.0f + expf((V - 35.0f) / 15.0f));
        float cc_D = sdiv(1.0f, 1.0f + expf((50.0f - V) / 20.0f));
        float cc_F = sdiv(180.0f, 1.0f + expf((V + 30.0f) / 10.0f)) + 20.0f;
        float cc_F2 = sdiv(80.0f, 1.0f + expf((V + 30.0f) / 10.0f));
        float den = sdiv(c.pmf_INaCa, 1.0f + (c.ksat * expf((c.nm1 * V) * c.F_RT)));
        o[TV_rec_iNaK] = sdiv(1.0f, (1.0f + (0.1245f * expf((-0.1f * V) * c.F_RT))) + (0.0353f * expf((-V) * c.F_RT)));
        o[TV_rec_ipK] = sdiv(1.0f, 1.0f + expf((25.0f - V) / 5.98f));
        float v40 = V + 40.0f;
        float tau_R = (9.5f * expf(((-v40) * v40) / 1800.0f)) + 0.8f;
        float tau_S;
        if (c.endo) {
            float v67 = V + 67.0f;
            tau_S = (1000.0f * expf(((-v67) * v67) / 1000.0f)) + 8.0f;
        } else {
            float v45 = V + 45.0f;
            tau_S = ((85.0f * expf(((-v45) * v45) / 320.0f)) + sdiv(5.0f, 1.0f + expf((V - 20.0f) / 5.0f))) + 3.0f;
        }
        o[TV_INaCa_A] = (den * c.Cao) * expf((c.n_ * V) * c.F_RT);
        o[TV_INaCa_B] = ((den * expf((c.nm1 * V) * c.F_RT)) * c.Nao3) * 2.5f;
        float J_inf = H_inf;
        float tau_D = (aa_D * bb_D) + cc_D;
        float tau_F2 = (aa_F2 + bb_F2) + cc_F2;
        float tau_Ff = (aa_F + bb_F) + cc_F;
        float tau_H = sdiv(1.0f, aa_H + bb_H);
        float tau_J = sdiv(1.0f, aa_J + bb_J);
        float tau_M = aa_M * bb_M;
        float tau_Xr1 = aa_Xr1 * bb_Xr1;
        float tau_Xr2 = aa_Xr2 * bb_Xr2;
        float tau_Xs = (aa_Xs * bb_Xs) + 80.0f;
        float tau_F = (V > 0.0f) ? tau_Ff * c.scl_tau_f : tau_Ff;
        gate(o, TV_D_A, D_inf, tau_D, c);
        gate(o, TV_F2_A, F2_inf, tau_F2, c);
        gate(o, TV_F_A, F_inf, tau_F, c);
        gate(o, TV_H_A, H_inf, tau_H, c);
        gate(o, TV_J_A, J_inf, tau_J, c);
        gate(o, TV_M_A, M_inf, tau_M, c);
        gate(o, TV_R_A, R_inf, tau_R, c);
        gate(o, TV_S_A, S_inf, tau_S, c);
        gate(o, TV_Xr1_A, Xr1_inf, tau_Xr1, c);
        gate(o, TV_Xr2_A, Xr2_inf, tau_Xr2, c);
        gate(o, TV_Xs_A, Xs_inf, tau_Xs, c);
    }
    // Rush-Larsen pair: B = exp(-dt/tau), A = -inf * expm1(-dt/tau)
    __host__ __device__ static void gate(float* o, int a_col, float inf, float tau, const C& c) {
        float e = sdiv(c.mdt, tau);
        o[a_col + 1] = expf(e);
        o[a_col] = (-inf) * expm1f(e);
    }

    __host__ __device__ static float vek_row(float V) {
        float a_K1 = sdiv(0.1f, 1.0f + expf(0.06f * (V - 200.0f)));
        float b_K1 = ((3.0f * expf(0.0002f * (V + 100.0f))) + expf(0.1f * (V - 10.0f))) / (1.0f + expf(-0.5f * V));
        return a_K1 / (a_K1 + b_K1);
    }

    __host__ __device__ static void init(const C& c, float* s, float& V) {
        for (int i = 0; i < TTP_NS; ++i) s[i] = c.init[i];
        V = c.V_init;
    }

    // ---------------------------------------------------- differentiate (:353-454)
    // The reference's order of operations; division and logarithm from the
    // policy Q (QFast or QExact, ionic_common.cuh).
    template <class Q>
    __host__ __device__ static float step(float V, float* s, const C& c, const Tables& T, const NodeG& g) {
        LutPos pv = lut_pos<Q>(V, T.V);
        const float CaSR = s[S_CaSR], CaSS = s[S_CaSS], Cai = s[S_Cai], Ki = s[S_Ki], Nai = s[S_Nai];
        LutPos pc = lut_pos<Q>(CaSS, T.CaSS);
        float Eca = c.halfRTONF * Q::log(Q::sdiv(c.Cao, Cai));
        float Ek = c.RTONF * Q::log(Q::sdiv(c.Ko, Ki));
        float Eks = c.RTONF * Q::log(Q::sdiv(c.KoNa, Ki + (c.pKNa * Nai)));
        float Ena = c.RTONF * Q::log(Q::sdiv(c.Nao, Nai));
        float IpCa = Q::div(c.GpCa * Cai, Cai + c.KpCa);
        float v15 = V - 15.0f;
        float a1 = g.ga1 * ((V == 15.0f) ? c.halfFRT : Q::div(v15, expm1f((2.0f * v15) * c.F_RT)));
        const float2 a2_iNaK = lut_pair<TV_NCOL>(T.V, pv, TV_a2);  // TV_a2, TV_rec_iNaK
        float ICaL_A = a1 * a2_iNaK.x;
        float ICaL_B = a1 * c.Cao;
        float VmEk = V - Ek;
        float IKr = ((g.GKr_sqrtKo * s[S_Xr1]) * s[S_Xr2]) * VmEk;
        float IKs = ((g.GKs * s[S_Xs]) * s[S_Xs]) * (V - Eks);
        float m = s[S_M];
        float INa = (((((c.GNa * m) * m) * m) * s[S_H]) * s[S_J]) * (V - Ena);
        float INaK = (c.pmf_INaK * Q::div(Nai, Nai + c.KmNa)) * a2_iNaK.y;
        float IbCa = c.GbCa * (V - Eca);
        float IbNa = c.GbNa * (V - Ena);
        float IpK = (c.GpK * lut_col<TV_NCOL>(T.V, pv, TV_rec_ipK)) * VmEk;
        float Ito = ((g.Gto * s[S_R]) * s[S_S]) * VmEk;
        LutPos pe = lut_pos<Q>(VmEk, T.VEk);
        float ICaL = (((s[S_D] * s[S_F]) * s[S_F2]) * s[S_FCaSS]) * ((ICaL_A * CaSS) - ICaL_B);
        const float2 naca = lut_pair<TV_NCOL>(T.V, pv, TV_INaCa_A);
        float INaCa = (((naca.x * Nai) * Nai) * Nai) - (naca.y * Cai);
        float IK1 = (c.GK1 * lut_col<1>(T.VEk, pe, 0)) * VmEk;
        float Iion = ((((((((((IKr + IKs) + IK1) + Ito) + INa) + IbNa) + ICaL) + IbCa) + INaK) + INaCa) + IpCa) + IpK;

        float Ileak = c.Vleak * (CaSR - Cai);
        float Iup = Q::sdiv(c.Vmaxup, 1.0f + Q::sdiv(c.KupKup, Cai * Cai));
        float Ixfer = c.Vxfer * (CaSS - Cai);
        float diff_Ki = (-((((IK1 + Ito) + IKr) + IKs) - (2.0f * INaK) + IpK)) * c.invVcF_Cm;
        float diff_Nai = (-(((INa + IbNa) + (3.0f * INaK)) + (3.0f * INaCa))) * c.invVcF_Cm;
        float ec = Q::sdiv(c.EC, CaSR);
        float kCaSR = c.maxsr - Q::sdiv(c.dsr, 1.0f + (ec * ec));
        float bc = Cai + c.Kbufc;
        float diff_Cai = Q::div((Ixfer - ((((IbCa + IpCa) - (2.0f * INaCa)) * c.inverseVcF2) * c.CAP)) -
                                  ((Iup - Ileak) * c.Vsr_Vc),
                              1.0f + Q::div(Q::sdiv(c.BufcKbufc, bc), bc));
        float R_ = s[S_R_];
        float diff_R_ = (c.k4 * (1.0f - R_)) - (((c.k2_ * kCaSR) * CaSS) * R_);
        float k1 = Q::sdiv(c.k1_, kCaSR);
        float cass2 = lut_col<3>(T.CaSS, pc, 0);
        float O = Q::div((k1 * cass2) * R_, (k1 * cass2) + c.k3);
        float Irel = (c.Vrel * O) * (CaSR - CaSS);
        float bsr = CaSR + c.Kbufsr;
        float diff_CaSR = Q::div((Iup - Irel) - Ileak, 1.0f + Q::div(Q::sdiv(c.BufsrKbufsr, bsr), bsr));
        float bss = CaSS + c.Kbufss;
        float diff_CaSS = Q::div((((-Ixfer) * c.Vc_Vss) + (Irel * c.Vsr_Vss)) + (((-ICaL) * c.inverseVssF2) * c.CAP),
                               1.0f + Q::div(Q::sdiv(c.BufssKbufss, bss), bss));
        s[S_CaSR] = CaSR + diff_CaSR * c.dt;
        s[S_CaSS] = CaSS + diff_CaSS * c.dt;
        s[S_Cai] = Cai + diff_Cai * c.dt;
        s[S_Ki] = Ki + diff_Ki * c.dt;
        s[S_Nai] = Nai + diff_Nai * c.dt;
        s[S_R_] = R_ + diff_R_ * c.dt;
        // Rush-Larsen (:439-450)
        s[S_D] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_D_A), s[S_D]);
        s[S_F] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_F_A), s[S_F]);
        s[S_F2] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_F2_A), s[S_F2]);
        s[S_FCaSS] = lut_col<3>(T.CaSS, pc, 1) + lut_col<3>(T.CaSS, pc, 2) * s[S_FCaSS];
        s[S_H] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_H_A), s[S_H]);
        s[S_J] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_J_A), s[S_J]);
        s[S_M] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_M_A), m);
        s[S_R] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_R_A), s[S_R]);
        s[S_S] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_S_A), s[S_S]);
        s[S_Xr1] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_Xr1_A), s[S_Xr1]);
        s[S_Xr2] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_Xr2_A), s[S_Xr2]);
        s[S_Xs] = rl_gate(lut_pair<TV_NCOL>(T.V, pv, TV_Xs_A), s[S_Xs]);
        return -Iion;
    }
};

}  // namespace tcb
