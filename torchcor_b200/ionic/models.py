"""The ionic models with the reference's class names, constructors and defaults.

* ``ModifiedMS2v(dt, device, dtype)`` - torchcor/ionic/ModifiedMS2v.py:4-44;
* ``MitchellSchaeffer`` - the same dimensional two-variable model.  The
  reference class of that name wraps the dimensionless CellML model and cannot
  run inside ``Monodomain`` (its ``initialize`` takes two arguments); this one
  accepts both ``MitchellSchaeffer(dt, device=..., dtype=...)`` and the
  reference form ``MitchellSchaeffer(device, dtype)``, taking dt from the
  simulator (or from ``initialize(n_nodes, dt)``);
* ``TenTusscherPanfilov(cell_type, dt, device, dtype)`` - TenTusscherPanfilov.py:6-454;
* ``CourtemancheRamirezNattel(dt, device, dtype)`` - CourtemancheRamirezNattel.py:5-444.
"""
from __future__ import annotations

import torch

from torchcor_b200._lib import MODEL_CRN, MODEL_MS, MODEL_TTP
from torchcor_b200.ionic.base import DeviceIonicModel


class ModifiedMS2v(DeviceIonicModel):
    model_id = MODEL_MS
    name = "ModifiedMS2v"

    def __init__(self, dt, device=None, dtype=torch.float32):
        super().__init__(dt, device, dtype)
        self.tau_in = 0.1          # ModifiedMS2v.py:9-18
        self.tau_out = 9.0
        self.tau_open = 100.0
        self.tau_close = 120.0
        self.u_gate = 0.13
        self.u_crit = 0.13
        self.vmin = -80.0
        self.vmax = 20.0

    @property
    def DV(self):
        return self.vmax - self.vmin


class MitchellSchaeffer(ModifiedMS2v):
    name = "MitchellSchaeffer"

    def __init__(self, dt=None, device=None, dtype=torch.float32):
        if isinstance(dt, (torch.device, str)):   # reference form MitchellSchaeffer(device, dtype)
            if isinstance(device, torch.dtype):
                dtype = device
            device, dt = dt, None
        super().__init__(dt, device, dtype)

    def initialize(self, n_nodes, dt=None):
        if dt is not None:
            self.dt = dt
        return super().initialize(n_nodes)


_TTP_DEFAULTS = dict(  # TenTusscherPanfilov.py:12-89
    CaSR_init=1.3, CaSS_init=0.00007, Cai_init=0.00007, EC=1.5, ENDO=2., EPI=0., F2_init=1., FCaSS_init=1.,
    F_init=1., H_init=0.75, J_init=0.75, Ki_init=138.3, MCELL=1., M_init=0., Nai_init=7.67, O_init=0.,
    R__init=1., R_init=0., S_init=1., V_init=-86.2, Vxfer=0.0038, Xr1_init=0., Xr2_init=1., Xs_init=0.,
    d_init=0., k1_=0.15, k2_=0.045, k3=0.060, k4=0.005, maxsr=2.5, minsr=1.,
    Bufc=0.2, Bufsr=10., Bufss=0.4, CAPACITANCE=0.185, Cao=2.0, D_CaL_off=0., Fconst=96485.3415, GK1=5.405,
    GNa=14.838, GbCa=0.000592, GbNa=0.00029, GpCa=0.1238, GpK=0.0146, Kbufc=0.001, Kbufsr=0.3,
    Kbufss=0.00025, KmCa=1.38, KmK=1.0, KmNa=40.0, KmNai=87.5, Ko=5.4, KpCa=0.0005, Kup=0.00025, Nao=140.0,
    Rconst=8314.472, T=310.0, Vc=0.016404, Vleak=0.00036, Vmaxup=0.006375, Vrel=0.102, Vsr=0.001094,
    Vss=0.00005468, knaca=1000., knak=2.724, ksat=0.1, n=0.35, pKNa=0.03, scl_tau_f=1., vHalfXs=5.,
    xr2_off=0., GCaL_init=0.00003980, GKr_init=0.153)


class TenTusscherPanfilov(DeviceIonicModel):
    model_id = MODEL_TTP
    name = "TenTusscherPanfilov"

    def __init__(self, cell_type, dt, device=None, dtype=torch.float32):
        super().__init__(dt, device, dtype)
        self.cell_type = "EPI" if cell_type is None else cell_type
        for k, v in _TTP_DEFAULTS.items():
            setattr(self, k, v)
        self.GKs_init = 0.392 if cell_type == "EPI" else 0.098 if cell_type == "MCELL" else 0.392
        self.Gto_init = 0.294 if cell_type == "EPI" else 0.294 if cell_type == "MCELL" else 0.073

    def _param_value(self, name):
        if name == "endo":
            return 1.0 if self.cell_type == "ENDO" else 0.0
        return super()._param_value(name)


_CRN_DEFAULTS = dict(  # CourtemancheRamirezNattel.py:9-94
    C_B1a=3.79138232501097e-05, C_B1b=0.0811764705882353, C_B1c=0.00705882352941176,
    C_B1d=0.00537112496043221, C_B1e=11.5, C_Fn1=9.648e-13, C_Fn2=2.5910306809e-13, C_dCa_rel=8.,
    C_dCaup=0.0869565217391304, Ca_rel_init=1.49, Ca_up_init=1.49, Cai_init=1.02e-1, F=96.4867, K_Q10=3.,
    K_up=0.00092, Ki_init=139.0, KmCa=1.38, KmCmdn=0.00238, KmCsqn=0.8, KmKo=1.5, KmNa=87.5,
    KmNa3=669921.875, KmNai=10., KmTrpn=0.0005, Nai=11.2, R=8.3143, T=310., V_init=-81.2, Volcell=20100.,
    Voli=13668., Volrel=96.48, Volup=1109.52, d_init=1.37e-4, f_Ca_init=0.775, f_init=0.999, gamma=0.35,
    h_init=0.965, j_init=0.978, k_rel=30., k_sat=0.1, m_init=2.91e-3, maxCmdn=0.05, maxCsqn=10.,
    maxTrpn=0.07, oa_init=3.04e-2, oi_init=0.999, tau_f_Ca=2., tau_tr=180., tau_u=8., u_init=0.,
    ua_init=4.96e-3, ui_init=0.999, v_init=1., w_init=0.999, xr_init=3.29e-5, xs_init=1.87e-2,
    ACh=0.000001, Cao=1.8, Cm=100., GACh=0., GCaL=0.1238, GK1=0.09, GKr=0.0294, GKs=0.129, GNa=7.8,
    GbCa=0.00113, GbNa=0.000674, Gto=0.1652, Ko=5.4, Nao=140., factorGKur=1., factorGrel=1., factorGtr=1.,
    factorGup=1., factorhGate=0., factormGate=0., factoroaGate=0., factorxrGate=1., maxCaup=15.,
    maxINaCa=1600., maxINaK=0.60, maxIpCa=0.275, maxIup=0.005)


class CourtemancheRamirezNattel(DeviceIonicModel):
    model_id = MODEL_CRN
    name = "CourtemancheRamirezNattel"

    def __init__(self, dt, device=None, dtype=torch.float32):
        super().__init__(dt, device, dtype)
        for k, v in _CRN_DEFAULTS.items():
            setattr(self, k, v)
