// Courtemanche-Ramirez-Nattel 1998 (torchcor/ionic/CourtemancheRamirezNattel.py:5-444):
// 19 states besides V (4 forward-Euler, 15 Rush-Larsen; Nai is a constant),
// lookup tables over V (32 columns), Cai (5) and the release flux fn (3).
#pragma once
#include "ionic_common.cuh"

namespace tcb {

struct CRNRaw {  // order of tcb_model_params(TCB_MODEL_CRN)
    double C_B1a, C_B1b, C_B1c, C_B1d, C_B1e, C_Fn1, C_Fn2, C_dCa_rel, C_dCaup, Ca_rel_init, Ca_up_init,
        Cai_init, F, K_Q10, K_up, Ki_init, KmCa, KmCmdn, KmCsqn, KmKo, KmNa, KmNa3, KmNai, KmTrpn, Nai, R, T,
        V_init, Volcell, Voli, Volrel, Volup, d_init, f_Ca_init, f_init, gamma, h_init, j_init, k_rel, k_sat,
        m_init, maxCmdn, maxCsqn, maxTrpn, oa_init, oi_init, tau_f_Ca, tau_tr, tau_u, u_init, ua_init, ui_init,
        v_init, w_init, xr_init, xs_init, ACh, Cao, Cm, GACh, GCaL, GK1, GKr, GKs, GNa, GbCa, GbNa, Gto, Ko, Nao,
        factorGKur, factorGrel, factorGtr, factorGup, factorhGate, factormGate, factoroaGate, factorxrGate,
        maxCaup, maxINaCa, maxINaK, maxIpCa, maxIup, dt;
};
#define TCB_CRN_PARAMS                                                                                          \
    "C_B1a,C_B1b,C_B1c,C_B1d,C_B1e,C_Fn1,C_Fn2,C_dCa_rel,C_dCaup,Ca_rel_init,Ca_up_init,Cai_init,F,K_Q10,K_up," \
    "Ki_init,KmCa,KmCmdn,KmCsqn,KmKo,KmNa,KmNa3,KmNai,KmTrpn,Nai,R,T,V_init,Volcell,Voli,Volrel,Volup,d_init,"  \
    "f_Ca_init,f_init,gamma,h_init,j_init,k_rel,k_sat,m_init,maxCmdn,maxCsqn,maxTrpn,oa_init,oi_init,tau_f_Ca,"  \
    "tau_tr,tau_u,u_init,ua_init,ui_init,v_init,w_init,xr_init,xs_init,ACh,Cao,Cm,GACh,GCaL,GK1,GKr,GKs,GNa,"   \
    "GbCa,GbNa,Gto,Ko,Nao,factorGKur,factorGrel,factorGtr,factorGup,factorhGate,factormGate,factoroaGate,"      \
    "factorxrGate,maxCaup,maxINaCa,maxINaK,maxIpCa,maxIup,dt"
#define TCB_CRN_STATES "Ca_rel,Ca_up,Cai,Ki,d,f,f_Ca,h,j,m,oa,oi,u,ua,ui,v,w,xr,xs"
static_assert(sizeof(CRNRaw) == count_names(TCB_CRN_PARAMS) * sizeof(double), "CRNRaw layout");

// V-table columns (CourtemancheRamirezNattel.py:104-137)
enum CRNV {
    CV_GKur, CV_INaK, CV_IbNa, CV_d_A, CV_d_B, CV_f_A, CV_f_B, CV_h_A, CV_h_B, CV_j_A, CV_j_B, CV_m_A, CV_m_B,
    CV_oa_A, CV_oa_B, CV_oi_A, CV_oi_B, CV_ua_A, CV_ua_B, CV_ui_A, CV_ui_B, CV_vrow_29, CV_vrow_31, CV_vrow_32,
    CV_vrow_36, CV_vrow_7, CV_w_A, CV_w_B, CV_xr_A, CV_xr_B, CV_xs_A, CV_xs_B, CV_NCOL
};
enum CRNC { CC_carow_1, CC_carow_2, CC_carow_3, CC_conCa, CC_f_Ca_A, CC_NCOL };
enum CRNS { R_Ca_rel, R_Ca_up, R_Cai, R_Ki, R_d, R_f, R_f_Ca, R_h, R_j, R_m, R_oa, R_oi, R_u, R_ua, R_ui, R_v, R_w,
            R_xr, R_xs, CRN_NS };

struct CRN {
    static constexpr int kStates = CRN_NS;
    static constexpr LutSpec kCai{3e-4, 30.0, 3e-4, CC_NCOL};
    static constexpr LutSpec kV{-200.0, 200.0, 0.1, CV_NCOL};
    static constexpr LutSpec kFn{-2e-11, 10.0e-11, 2e-15, 3};

    struct C {
        // differentiate
        float RTF, Ko, ACh_term, tauf_k, Gto, factorGKur, GKr, GKs, GK1, factorGtr, tau_tr, factorGrel, k_rel,
            maxIup_maxCaup, C_dCa_rel, KmCsqn, FVoli, C_dCaup, C_B1d, C_B1e, fCa_B, u_B, C_Fn1, C_Fn2, dt;
        // tables
        float mdt, f_Ca_C, u_C, E_Na, GbNa, fGup_maxIup, K_up, maxTrpnKmTrpn, KmTrpn, maxCmdnKmCmdn, KmCmdn,
            C_B1c, maxIpCa, GbCaRT2F, Cao, factorhGate, factormGate, factoroaGate, factorxrGate, inv_fxr, mF_R,
            m01F_R, sig0365, GCaL, gF_R, gm1F_R, maxINaCa, Nai, NaCaDen, KmCa_Cao, k_sat, Nao, GbCa, GNa, INaK_c,
            KoKmKo, K_Q10, R, T, maxINaK, tau_d10, bh0;
        float init[CRN_NS];
        float V_init;
    };
    struct Tables {
        Lut V, Cai, Fn;
    };

    static C derive(const double* p) {
        CRNRaw r;
        memcpy(&r, p, sizeof r);
        C c;
        c.RTF = (float)((r.R * r.T) / r.F);
        c.Ko = (float)r.Ko;
        // (GACh*(10.0/(1.0+(9.13652/pow(ACh,0.477811))))) is a Python float (:365)
        c.ACh_term = (float)(r.GACh * (10.0 / (1.0 + (9.13652 / pow(r.ACh, 0.477811)))));
        c.tauf_k = (float)(-0.0337 * 0.0337);
        c.Gto = (float)r.Gto;
        c.factorGKur = (float)r.factorGKur;
        c.GKr = (float)r.GKr;
        c.GKs = (float)r.GKs;
        c.GK1 = (float)r.GK1;
        c.factorGtr = (float)r.factorGtr;
        c.tau_tr = (float)r.tau_tr;
        c.factorGrel = (float)r.factorGrel;
        c.k_rel = (float)r.k_rel;
        c.maxIup_maxCaup = (float)(r.maxIup / r.maxCaup);
        c.C_dCa_rel = (float)r.C_dCa_rel;
        c.KmCsqn = (float)r.KmCsqn;
        c.FVoli = (float)(r.F * r.Voli);
        c.C_dCaup = (float)r.C_dCaup;
        c.C_B1d = (float)r.C_B1d;
        c.C_B1e = (float)r.C_B1e;
        c.fCa_B = (float)exp((-r.dt) / r.tau_f_Ca);   // :199-200
        c.u_B = (float)exp((-r.dt) / r.tau_u);
        c.C_Fn1 = (float)r.C_Fn1;
        c.C_Fn2 = (float)r.C_Fn2;
        c.dt = (float)r.dt;
        // construct_tables (:213-216)
        double E_Na = ((r.R * r.T) / r.F) * log(r.Nao / r.Nai);
        double sigma = (exp(r.Nao / 67.3) - 1.) / 7.;
        c.mdt = (float)(-r.dt);
        c.f_Ca_C = (float)expm1((-r.dt) / r.tau_f_Ca);
        c.u_C = (float)expm1((-r.dt) / r.tau_u);
        c.E_Na = (float)E_Na;
        c.GbNa = (float)r.GbNa;
        c.fGup_maxIup = (float)(r.factorGup * r.maxIup);
        c.K_up = (float)r.K_up;
        c.maxTrpnKmTrpn = (float)(r.maxTrpn * r.KmTrpn);
        c.KmTrpn = (float)r.KmTrpn;
        c.maxCmdnKmCmdn = (float)(r.maxCmdn * r.KmCmdn);
        c.KmCmdn = (float)r.KmCmdn;
        c.C_B1c = (float)r.C_B1c;
        c.maxIpCa = (float)r.maxIpCa;
        c.GbCaRT2F = (float)((((r.GbCa * r.R) * r.T) / 2.) / r.F);
        c.Cao = (float)r.Cao;
        c.factorhGate = (float)r.factorhGate;
        c.factormGate = (float)r.factormGate;
        c.factoroaGate = (float)r.factoroaGate;
        c.factorxrGate = (float)r.factorxrGate;
        c.inv_fxr = (float)(1.0 / r.factorxrGate);
        c.mF_R = (float)(-r.F);
        c.m01F_R = (float)(-0.1 * r.F);
        c.sig0365 = (float)(0.0365 * sigma);
        c.GCaL = (float)r.GCaL;
        c.gF_R = (float)(r.gamma * r.F);
        c.gm1F_R = (float)((r.gamma - 1.) * r.F);
        c.maxINaCa = (float)r.maxINaCa;
        c.Nai = (float)r.Nai;
        c.NaCaDen = (float)(r.KmNa3 + ((r.Nao * r.Nao) * r.Nao));
        c.KmCa_Cao = (float)(r.KmCa + r.Cao);
        c.k_sat = (float)r.k_sat;
        c.Nao = (float)r.Nao;
        c.GbCa = (float)r.GbCa;
        c.GNa = (float)r.GNa;
        c.INaK_c = (float)(1. + pow(r.KmNai / r.Nai, 1.5));
        c.KoKmKo = (float)(r.Ko + r.KmKo);
        c.K_Q10 = (float)r.K_Q10;
        c.R = (float)r.R;
        c.T = (float)r.T;
        c.maxINaK = (float)r.maxINaK;
        c.tau_d10 = (float)(((1. / 6.24) / 0.035) / 2.);
        c.bh0 = (float)(1. / 0.13);
        const double init[CRN_NS] = {r.Ca_rel_init, r.Ca_up_init, r.Cai_init, r.Ki_init, r.d_init, r.f_init,
                                     r.f_Ca_init, r.h_init, r.j_init, r.m_init, r.oa_init, r.oi_init, r.u_init,
                                     r.ua_init, r.ui_init, r.v_init, r.w_init, r.xr_init, r.xs_init};
        for (int i = 0; i < CRN_NS; ++i) c.init[i] = (float)init[i];
        c.V_init = (float)r.V_init;
        return c;
    }

    // no per-node parameters
    static constexpr int kNodeParams = 0;
    struct NodeG {};
    __host__ __device__ static NodeG node_g(const C&, const float*, int64_t, int64_t) { return NodeG{}; }

    static int64_t table_floats(const double*) {
        return kV.floats() + kCai.floats() + kFn.floats();
    }
    static Tables tables(const float* t, const double*) {
        Tables T;
        T.V = kV.make(t);
        T.Cai = kCai.make(t + kV.floats());
        T.Fn = kFn.make(t + kV.floats() + kCai.floats());
        return T;
    }

    // ------------------------------------------------------ tables (:212-328)
    __host__ __device__ static void cai_row(float cai, const C& c, float* o) {
        float con = cai / 1000.0f;
        o[CC_conCa] = con;
        o[CC_carow_1] = sdiv(c.fGup_maxIup, 1.0f + sdiv(c.K_up, con));
        float a = con + c.KmTrpn, b = con + c.KmCmdn;
        o[CC_carow_2] = ((((sdiv(c.maxTrpnKmTrpn, a) / a) + (sdiv(c.maxCmdnKmCmdn, b) / b)) + 1.0f) / c.C_B1c) / 1000.0f;
        o[CC_carow_3] = ((c.maxIpCa * con) / (con + 0.0005f)) - (c.GbCaRT2F * logf(sdiv(c.Cao, con)));
        float f_Ca_inf = sdiv(1.0f, 1.0f + (con / 0.00035f));
        o[CC_f_Ca_A] = (-f_Ca_inf) * c.f_Ca_C;
    }

    __host__ __device__ static void fn_row(float fn, const C& c, float* o) {
        float eu = expf((3.4175e-13f - fn) / 13.67e-16f);
        float tau_v = sdiv(2.09f, 1.0f + eu) + 1.91f;
        float u_inf = sdiv(1.0f, 1.0f + eu);
        float v_inf = 1.0f - sdiv(1.0f, 1.0f + expf((6.835e-14f - fn) / 13.67e-16f));
        o[0] = (-u_inf) * c.u_C;
        float e = sdiv(c.mdt, tau_v);
        o[2] = expf(e);
        o[1] = (-v_inf) * expm1f(e);
    }

    __host__ __device__ static void rl_tau(float* o, int a_col, float inf, float tau, const C& c) {
        float e = sdiv(c.mdt, tau);
        o[a_col + 1] = expf(e);
        o[a_col] = (-inf) * expm1f(e);
    }
    __host__ __device__ static void rl_ab(float* o, int a_col, float a, float b, const C& c) {
        float ab = a + b;
        o[a_col] = ((-a) / ab) * expm1f(ab * c.mdt);
        o[a_col + 1] = expf(ab * c.mdt);
    }

    __host__ __device__ static void v_row(float V, const C& c, float* o) {
        o[CV_GKur] = sdiv(0.05f, 1.0f + expf((15.0f - V) / 13.0f)) + 0.005f;
        o[CV_IbNa] = c.GbNa * (V - c.E_Na);
        float a_h = (V >= -40.0f) ? 0.0f : 0.135f * expf(((V + 80.0f) - c.factorhGate) / -6.8f);
        float a_j = (V < -40.0f)
                        ? (((-127140.0f * expf(0.2444f * V)) - (3.474e-5f * expf(-0.04391f * V))) * (V + 37.78f)) /
                              (1.0f + expf(0.311f * (V + 79.23f)))
                        : 0.0f;
        float a_m = (V == -47.13f) ? 3.2f : (0.32f * (V + 47.13f)) / (1.0f - expf(-0.1f * (V + 47.13f)));
        float aa_oa = sdiv(0.65f, expf((V + 10.0f) / -8.5f) + expf((30.0f - V) / 59.0f));
        float aa_oi = sdiv(1.0f, expf((V + 113.7f) / 10.95f) + 18.53f);
        float aa_ua = sdiv(0.65f, expf((V + 10.0f) / -8.5f) + expf((V - 30.0f) / -59.0f));
        float aa_ui = sdiv(1.0f, expf((V - 185.0f) / -28.0f) + 21.0f);
        float aa_xr = ((0.0003f * (V + 14.1f)) / (1.0f - expf((V + 14.1f) / -5.0f))) * c.factorxrGate;
        float aa_xs = (4.e-5f * (V - 19.9f)) / (1.0f - expf((19.9f - V) / 17.0f));
        float b_h = (V >= -40.0f) ? sdiv(c.bh0, 1.0f + expf((-(V + 10.66f)) / 11.1f))
                                  : (3.56f * expf(0.079f * V)) + (3.1e5f * expf(0.35f * V));
        float b_j = (V >= -40.0f) ? (0.3f * expf(-2.535e-7f * V)) / (1.0f + expf(-0.1f * (V + 32.0f)))
                                  : (0.1212f * expf(-0.01052f * V)) / (1.0f + expf(-0.1378f * (V + 40.14f)));
        float b_m = 0.08f * expf((-(V - c.factormGate)) / 11.0f);
        float bb_oa = sdiv(0.65f, expf((V + 82.0f) / 17.0f) + 2.5f);
        float bb_oi = sdiv(1.0f, expf((-(V + 1.26f)) / 7.44f) + 35.56f);
        float bb_ua = sdiv(0.65f, expf((V + 82.0f) / 17.0f) + 2.5f);
        float bb_ui = expf((V - 158.0f) / 16.0f);
        float bb_xr = ((7.3898e-5f * (V - 3.3328f)) / (expf((V - 3.3328f) / 5.1237f) - 1.0f)) * c.inv_fxr;
        float bb_xs = (3.5e-5f * (V - 19.9f)) / (expf((V - 19.9f) / 9.0f) - 1.0f);
        float d_inf = sdiv(1.0f, 1.0f + expf((-(V + 10.0f)) / 8.0f));
        float f_NaK = sdiv(1.0f, (1.0f + (0.1245f * expf(((c.m01F_R * V) / c.R) / c.T))) +
                                     (c.sig0365 * expf(((c.mF_R * V) / c.R) / c.T)));
        float f_inf = sdiv(1.0f, 1.0f + expf((V + 28.0f) / 6.9f));
        float oa_inf = sdiv(1.0f, 1.0f + expf((-((V + 20.47f) - c.factoroaGate)) / 17.54f));
        float oi_inf = sdiv(1.0f, 1.0f + expf((V + 43.1f) / 5.3f));
        float ed = expf((-(V + 10.0f)) / 6.24f);
        float tau_d = (V == -10.0f) ? c.tau_d10 : (((1.0f - ed) / 0.035f) / (V + 10.0f)) / (1.0f + ed);
        float v10 = V + 10.0f;
        float tau_f = sdiv(9.0f, (0.0197f * expf((c.tauf_k * v10) * v10)) + 0.02f);
        float ew = expf((7.9f - V) / 5.0f);
        float tau_w = ((6.0f * (1.0f - ew)) / (1.0f + (0.3f * ew))) / (V - 7.9f);
        float ua_inf = sdiv(1.0f, 1.0f + expf((V + 30.3f) / -9.6f));
        float ui_inf = sdiv(1.0f, 1.0f + expf((V - 99.45f) / 27.48f));
        o[CV_vrow_29] = c.GCaL * (V - 65.0f);
        float eg1 = expf(((c.gm1F_R * V) / c.R) / c.T);
        o[CV_vrow_31] = ((((((c.maxINaCa * expf(((c.gF_R * V) / c.R) / c.T)) * c.Nai) * c.Nai) * c.Nai) * c.Cao) /
                         c.NaCaDen / c.KmCa_Cao) /
                        (1.0f + (c.k_sat * eg1));
        o[CV_vrow_32] = (((((c.maxINaCa * eg1) * c.Nao) * c.Nao) * c.Nao) / c.NaCaDen / c.KmCa_Cao /
                         (1.0f + (c.k_sat * eg1))) /
                        1000.0f;
        o[CV_vrow_36] = V * c.GbCa;
        o[CV_vrow_7] = c.GNa * (V - c.E_Na);
        float w_inf = 1.0f - sdiv(1.0f, 1.0f + expf((40.0f - V) / 17.0f));
        float xr_inf = sdiv(1.0f, 1.0f + expf((V + 14.1f) / -6.5f));
        float xs_inf = sdiv(1.0f, sqrtf(1.0f + expf((V - 19.9f) / -12.7f)));
        o[CV_INaK] = (((c.maxINaK * f_NaK) / c.INaK_c) * c.Ko) / c.KoKmKo;
        rl_tau(o, CV_d_A, d_inf, tau_d, c);
        rl_tau(o, CV_f_A, f_inf, tau_f, c);
        rl_ab(o, CV_h_A, a_h, b_h, c);
        rl_ab(o, CV_j_A, a_j, b_j, c);
        rl_ab(o, CV_m_A, a_m, b_m, c);
        float tau_oa = sdiv(1.0f, aa_oa + bb_oa) / c.K_Q10;
        float tau_oi = sdiv(1.0f, aa_oi + bb_oi) / c.K_Q10;
        float tau_ua = sdiv(1.0f, aa_ua + bb_ua) / c.K_Q10;
        float tau_ui = sdiv(1.0f, aa_ui + bb_ui) / c.K_Q10;
        float tau_xr = sdiv(1.0f, aa_xr + bb_xr);
        float tau_xs = sdiv(0.5f, aa_xs + bb_xs);
        rl_tau(o, CV_w_A, w_inf, tau_w, c);
        rl_tau(o, CV_oa_A, oa_inf, tau_oa, c);
        rl_tau(o, CV_oi_A, oi_inf, tau_oi, c);
        rl_tau(o, CV_ua_A, ua_inf, tau_ua, c);
        rl_tau(o, CV_ui_A, ui_inf, tau_ui, c);
        rl_tau(o, CV_xr_A, xr_inf, tau_xr, c);
        rl_tau(o, CV_xs_A, xs_inf, tau_xs, c);
    }

    __host__ __device__ static void init(const C& c, float* s, float& V) {
        for (int i = 0; i < CRN_NS; ++i) s[i] = c.init[i];
        V = c.V_init;
    }

    // ------------------------------------------------ differentiate (:358-444)
    // The reference's order of operations; division and logarithm from the
    // policy Q (QFast or QExact, ionic_common.cuh).
    template <class Q>
    __host__ __device__ static float step(float V, float* s, const C& c, const Tables& T, const NodeG&) {
        LutPos pv = lut_pos<Q>(V, T.V);
        LutPos pc = lut_pos<Q>(s[R_Cai], T.Cai);
#define VR(col) lut_col<CV_NCOL>(T.V, pv, col)
#define CR(col) lut_col<CC_NCOL>(T.Cai, pc, col)
        float E_K = c.RTF * Q::log(Q::sdiv(c.Ko, s[R_Ki]));
        float VmK = V - E_K;
        float ICaL = ((VR(CV_vrow_29) * s[R_d]) * s[R_f]) * s[R_f_Ca];
        float IKACh = (c.ACh_term * (Q::sdiv(0.4516f, 1.0f + expf(Q::div(V + 59.53f, 17.18f))) + 0.0517f)) * VmK;
        float m = s[R_m];
        float INa = ((((VR(CV_vrow_7) * m) * m) * m) * s[R_h]) * s[R_j];
        float INaCa = VR(CV_vrow_31) - (s[R_Cai] * VR(CV_vrow_32));
        float vrow_13 = c.Gto * VmK;
        float vrow_18 = (c.factorGKur * VR(CV_GKur)) * VmK;
        float vrow_21 = Q::div(c.GKr * VmK, 1.0f + expf(Q::div(V + 15.0f, 22.4f)));
        float vrow_24 = c.GKs * VmK;
        float IK1 = Q::div(c.GK1 * VmK, 1.0f + expf(0.07f * (V + 80.0f)));
        float IKr = vrow_21 * s[R_xr];
        float IKs = (vrow_24 * s[R_xs]) * s[R_xs];
        float ua = s[R_ua], oa = s[R_oa];
        float IKur = (((vrow_18 * ua) * ua) * ua) * s[R_ui];
        float IpCa = CR(CC_carow_3) + VR(CV_vrow_36);
        float Ito = (((vrow_13 * oa) * oa) * oa) * s[R_oi];
        float INaK = VR(CV_INaK);
        float Iion = INa + IK1 + Ito + IKur + IKr + IKs + ICaL + IpCa + INaCa + VR(CV_IbNa) + INaK + IKACh;

        float Ca_rel = s[R_Ca_rel], Ca_up = s[R_Ca_up], u = s[R_u];
        float Itr = Q::div(c.factorGtr * (Ca_up - Ca_rel), c.tau_tr);
        float Irel = (((((c.factorGrel * u) * u) * s[R_v]) * c.k_rel) * s[R_w]) * (Ca_rel - CR(CC_conCa));
        float dIups = CR(CC_carow_1) - (c.maxIup_maxCaup * Ca_up);
        float cs = Ca_rel + c.KmCsqn;
        float diff_Ca_rel = Q::div(Itr - Irel, 1.0f + Q::div(Q::sdiv(c.C_dCa_rel, cs), cs));
        float diff_Ki = Q::div(-((((((Ito + IKr) + IKur) + IKs) + IK1) + IKACh) - (2.0f * INaK)), c.FVoli);
        float diff_Ca_up = dIups - (Itr * c.C_dCaup);
        float diff_Cai = Q::div(((c.C_B1d * (((INaCa + INaCa) - IpCa) - ICaL)) - (c.C_B1e * dIups)) + Irel, CR(CC_carow_2));
        s[R_Ca_rel] = Ca_rel + diff_Ca_rel * c.dt;
        s[R_Ca_up] = Ca_up + diff_Ca_up * c.dt;
        float fCaA = CR(CC_f_Ca_A);
        s[R_Cai] = s[R_Cai] + diff_Cai * c.dt;
        s[R_Ki] = s[R_Ki] + diff_Ki * c.dt;

        float fn = (c.C_Fn1 * Irel) - (c.C_Fn2 * (ICaL - (0.4f * INaCa)));
        LutPos pf = lut_pos<Q>(fn, T.Fn);
        s[R_d] = VR(CV_d_A) + VR(CV_d_B) * s[R_d];
        s[R_f] = VR(CV_f_A) + VR(CV_f_B) * s[R_f];
        s[R_f_Ca] = fCaA + c.fCa_B * s[R_f_Ca];
        s[R_h] = VR(CV_h_A) + VR(CV_h_B) * s[R_h];
        s[R_j] = VR(CV_j_A) + VR(CV_j_B) * s[R_j];
        s[R_m] = VR(CV_m_A) + VR(CV_m_B) * m;
        s[R_oa] = VR(CV_oa_A) + VR(CV_oa_B) * oa;
        s[R_oi] = VR(CV_oi_A) + VR(CV_oi_B) * s[R_oi];
        s[R_u] = lut_col<3>(T.Fn, pf, 0) + c.u_B * u;
        s[R_ua] = VR(CV_ua_A) + VR(CV_ua_B) * ua;
        s[R_ui] = VR(CV_ui_A) + VR(CV_ui_B) * s[R_ui];
        s[R_v] = lut_col<3>(T.Fn, pf, 1) + lut_col<3>(T.Fn, pf, 2) * s[R_v];
        s[R_w] = VR(CV_w_A) + VR(CV_w_B) * s[R_w];
        s[R_xr] = VR(CV_xr_A) + VR(CV_xr_B) * s[R_xr];
        s[R_xs] = VR(CV_xs_A) + VR(CV_xs_B) * s[R_xs];
#undef VR
#undef CR
        return -Iion;
    }
};

}  // namespace tcb
