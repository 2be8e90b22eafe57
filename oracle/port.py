"""CPU restatement of TorchCor 0.1.8's monodomain path (the oracle).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline legs, never by the product package.

Each block restates the reference function it cites (paths relative to the
TorchCor repository) with plain PyTorch CPU ops, keeping the reference's
operation order and dtype promotion so that, on one machine, the results agree
with the reference bit for bit.  Two facts of PyTorch arithmetic that the
restatement (and the CUDA kernels) rely on:

* ``python_float / tensor`` is evaluated as ``tensor.reciprocal() * python_float``
  (both eagerly and under ``torch.jit.script``), not as a true division;
* ``tensor op python_float`` rounds the Python float to the tensor dtype first.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

CPU = torch.device("cpu")


# --------------------------------------------------------------------------
# mesh input  (torchcor/core/mesh.py:5-63)
# --------------------------------------------------------------------------
def find_mesh_files(mesh_dir):
    """Pick the ``.pts/.elem/.lon`` files of a mesh directory (mesh.py:7-19)."""
    files = {}
    for p in Path(mesh_dir).iterdir():
        if p.suffix in (".pts", ".elem", ".lon"):
            files[p.suffix] = p
    return files


def read_mesh(mesh_dir, unit_conversion=1000):
    """Return (nodes, elems, regions, fibres) as numpy arrays (mesh.py:26-63).

    nodes are divided by ``unit_conversion`` (um -> mm); elems/regions/fibres
    are per element; a count mismatch raises ``ValueError``.
    """
    f = find_mesh_files(mesh_dir)
    with f[".pts"].open("r") as fh:
        n_expected = int(fh.readline().strip())
    nodes = np.loadtxt(f[".pts"], dtype=float, skiprows=1)
    if nodes.shape[0] != n_expected:
        raise ValueError(f"Mismatch in number of nodes: expected {n_expected}, but found {nodes.shape[0]}")
    nodes = nodes / unit_conversion
    with f[".elem"].open("r") as fh:
        e_expected = int(fh.readline().strip())
        first = fh.readline().strip().split()
        usecols = list(range(1, len(first)))
    data = np.loadtxt(f[".elem"], dtype=int, skiprows=1, usecols=usecols)
    if data.shape[0] != e_expected:
        raise ValueError(f"Mismatch: expected {e_expected}, but found {data.shape[0]}")
    elems, regions = data[:, :-1], data[:, -1]
    fibres = np.loadtxt(f[".lon"], dtype=np.float64, skiprows=1)
    return nodes, elems, regions, fibres


def read_vtx(path):
    """Node indices of a ``.vtx`` stimulus file (stimulation.py:20-29)."""
    with Path(path).open("r") as fh:
        n = int(fh.readline().strip())
    region = np.loadtxt(path, dtype=int, skiprows=2)
    if len(region) != n:
        raise Exception(f"Error loading {path}")
    return torch.from_numpy(region).to(torch.long)


# --------------------------------------------------------------------------
# conductivity  (torchcor/core/conductivity.py:4-69)
# --------------------------------------------------------------------------
class Conductivity:
    """Per-element sigma_l / sigma_t and the (E,3,3) tensor (conductivity.py:4-69)."""

    def __init__(self, regions: torch.Tensor, dtype):
        self.regions = regions
        self.dtype = dtype
        z = lambda: torch.zeros_like(regions, dtype=dtype)  # noqa: E731
        self.il, self.it, self.el, self.et = z(), z(), z(), z()
        self.sl, self.st = z(), z()

    def add(self, region_ids, il, it, el=None, et=None):
        # conductivity.py:18-47: without el/et the bulk value is il/it and the
        # intra/extra arrays are dropped; with them, the harmonic mean.
        if el is None and et is None:
            self.il = self.it = self.el = self.et = None
            lv, tv = il, it
            for rid in region_ids:
                m = self.regions == rid
                self.sl[m] = lv
                self.st[m] = tv
        else:
            lv = il * el * (1 / (il + el))
            tv = it * et * (1 / (it + et))
            for rid in region_ids:
                m = self.regions == rid
                self.il[m] = il
                self.it[m] = it
                self.el[m] = el
                self.et[m] = et
                self.sl[m] = lv
                self.st[m] = tv

    def _tensor(self, l, t, fibres):
        # conductivity.py:64-67: sigma = t*I + (l - t) * f f^T
        E = fibres.shape[0]
        lv = l.view(E, 1, 1)
        tv = t.view(E, 1, 1)
        s = tv * torch.eye(3, dtype=self.dtype).unsqueeze(0).expand(E, 3, 3)
        s += (lv - tv) * fibres.unsqueeze(2) @ fibres.unsqueeze(1)
        return s

    def sigma(self, fibres):
        """(sigma_i, sigma_e, sigma_m) as in conductivity.py:49-69."""
        if self.il is None and self.it is None and self.el is None and self.et is None:
            si = se = None
        else:
            si = self._tensor(self.il, self.it, fibres)
            se = self._tensor(self.el, self.et, fibres)
        return si, se, self._tensor(self.sl, self.st, fibres)


# --------------------------------------------------------------------------
# P1 assembly  (torchcor/core/assemble.py)
# --------------------------------------------------------------------------
def tet_local_matrices(vertices, tets, sigma, dtype):
    """Batched (Me, Ke) of P1 tetrahedra (assemble.py:156-215)."""
    coords = vertices[tets]                                   # (E,4,3)
    E = coords.shape[0]
    aug = torch.cat([torch.ones(E, 4, 1, dtype=dtype), coords], dim=2)
    vol = torch.abs(torch.linalg.det(aug)) / 6                # :194-200
    pattern = torch.tensor([[2, 1, 1, 1], [1, 2, 1, 1], [1, 1, 2, 1], [1, 1, 1, 2]], dtype=dtype)
    Me = (vol / 20).unsqueeze(1).unsqueeze(2) * pattern.unsqueeze(0)   # :171-178
    dN = torch.tensor([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=dtype)
    J = coords.transpose(1, 2) @ dN                           # :163-169
    detJ = torch.abs(torch.linalg.det(J))
    invJ = torch.linalg.inv(J)
    G = dN @ invJ
    Ke = (detJ / 6).view(-1, 1, 1) * (G @ (sigma @ G.transpose(1, 2)))  # :180-192
    return Me, Ke


def _surface_rotation(c):
    # assemble.py:103-113: orthonormal in-plane frame (alpha, beta)
    u1 = c[:, 1, :] - c[:, 0, :]
    u2 = c[:, 2, :] - c[:, 0, :]
    alpha = u1 / torch.linalg.norm(u1, dim=1, keepdim=True)
    beta = u2 - torch.sum(u2 * alpha, dim=1, keepdim=True) * alpha
    beta = beta / torch.linalg.norm(beta, dim=1, keepdim=True)
    return torch.stack([alpha, beta], dim=1)                  # (E,2,3)


def tri_surface_local_matrices(vertices, tris, sigma, dtype):
    """Batched (Me, Ke) of P1 triangles embedded in 3-D (assemble.py:4-145)."""
    c = vertices[tris]                                        # (E,3,3)
    a = c[:, 1] - c[:, 0]
    b = c[:, 2] - c[:, 0]
    area = 0.5 * torch.norm(torch.linalg.cross(a, b), dim=1)  # :123-130
    pattern = torch.tensor([[2, 1, 1], [1, 2, 1], [1, 1, 2]], dtype=dtype)
    Me = (area / 12).unsqueeze(1).unsqueeze(2) * pattern.unsqueeze(0)  # :27-31
    dN = torch.tensor([[-1, -1], [1, 0], [0, 1]], dtype=dtype)
    R = _surface_rotation(c)
    s2 = R @ sigma @ R.transpose(1, 2)                        # :134
    J = _surface_rotation(c) @ c.transpose(1, 2) @ dN         # :115-121
    detJ = torch.linalg.det(J)
    invJ = torch.linalg.inv(J)
    G = dN @ invJ
    Ke = (0.5 * detJ).view(-1, 1, 1) * G @ (s2 @ G.transpose(1, 2))   # :143
    return Me, Ke


def scatter_coo(elems, Me, Ke, n_nodes, dtype):
    """Global K, M as coalesced COO (assemble.py:217-248 / :67-96).

    The reference lists entries (i, j)-major over all elements, converts the
    values through Python floats (so they become default-dtype float32), casts
    to ``dtype`` and coalesces.
    """
    k = elems.shape[1]
    el = elems.to(torch.long)
    rows = torch.cat([el[:, i] for i in range(k) for _ in range(k)])
    cols = torch.cat([el[:, j] for _ in range(k) for j in range(k)])
    kv = torch.cat([Ke[:, i, j] for i in range(k) for j in range(k)]).to(torch.float32)
    mv = torch.cat([Me[:, i, j] for i in range(k) for j in range(k)]).to(torch.float32)
    idx = torch.stack([rows, cols])
    K = torch.sparse_coo_tensor(idx, kv, size=(n_nodes, n_nodes)).to(dtype=dtype)
    M = torch.sparse_coo_tensor(idx, mv, size=(n_nodes, n_nodes)).to(dtype=dtype)
    return K.coalesce(), M.coalesce()


def jacobi(A_coo):
    """PC = 1/diag(A) from a COO matrix (preconditioner.py:9-27)."""
    A = A_coo.coalesce()
    ind, val = A.indices(), A.values()
    diag = ind[0] == ind[1]
    pc = torch.zeros(A.shape[0], dtype=A.dtype)
    pc[ind[0][diag]] = val[diag]
    return 1.0 / pc


@dataclass
class System:
    M: torch.Tensor       # CSR, dtype
    K: torch.Tensor       # CSR, dtype, already divided by chi
    A: torch.Tensor       # CSR, dtype (the CG casts it to float64)
    PC: torch.Tensor      # (N,) dtype
    A_coo: torch.Tensor = None


def build_system(vertices, elems, sigma_m, dt, dtype, chi=140, cm=0.01, theta=0.5):
    """Monodomain.assemble (monodomain.py:83-106)."""
    if elems.shape[1] == 3:
        Me, Ke = tri_surface_local_matrices(vertices, elems, sigma_m, dtype)
    else:
        Me, Ke = tet_local_matrices(vertices, elems, sigma_m, dtype)
    K, M = scatter_coo(elems, Me, Ke, vertices.shape[0], dtype)
    K = K / chi
    K = K.to(dtype=dtype)
    M = M.to(dtype=dtype)
    A = M * cm + K * dt * theta
    A = A.coalesce()
    pc = jacobi(A)
    return System(M=M.to_sparse_csr(), K=K.to_sparse_csr(), A=A.to_sparse_csr(), PC=pc, A_coo=A)


# --------------------------------------------------------------------------
# Jacobi-PCG  (torchcor/core/solver.py:5-76)
# --------------------------------------------------------------------------
class PCG:
    """Jacobi-preconditioned CG in float64 with the linear-extrapolation guess."""

    def __init__(self, pc, A_csr, dtype=torch.float64):
        self.pc = pc
        self.dtype = dtype
        self.A = A_csr

    def initialize(self, x, linear_guess=True):            # solver.py:23-33
        self.A = self.A.to(self.dtype)
        self.x = x.to(self.dtype).clone()
        self.x_prev = x.clone()
        self.linear_guess = linear_guess

    def solve(self, b, a_tol=1e-6, r_tol=1e-6, max_iter=100):   # solver.py:40-76
        b_dtype = b.dtype
        b = b.to(self.dtype)
        n_iter = 0
        if self.linear_guess:                               # :35-38
            xc = self.x.clone()
            self.x.mul_(2).sub_(self.x_prev)
            self.x_prev.copy_(xc)
        r = b - self.A @ self.x
        z = self.pc * r
        p = z.clone()
        b_norm = torch.linalg.vector_norm(self.pc * b)
        for _ in range(max_iter):
            Ap = self.A @ p
            rz = torch.dot(r, z)
            alpha = rz / torch.dot(p, Ap)
            self.x.add_(alpha * p)
            r.sub_(alpha * Ap)
            z = self.pc * r
            zn = torch.linalg.vector_norm(z)
            if zn.item() < a_tol or (zn.item() / b_norm.item()) < r_tol:
                break
            beta = torch.dot(r, z) / rz
            p.mul_(beta).add_(z)
            n_iter += 1
        return self.x.to(b_dtype), n_iter


# --------------------------------------------------------------------------
# stimuli  (torchcor/core/stimulation.py:6-63)
# --------------------------------------------------------------------------
@dataclass
class Stim:
    region: torch.Tensor
    stimulus: torch.Tensor
    start: float
    duration: float
    intensity: float
    period: float
    count: float


class Stimuli:
    def __init__(self, n_nodes, dtype):
        self.items: list[Stim] = []
        self.n = n_nodes
        self.dtype = dtype
        self.zero = torch.zeros((n_nodes,), dtype=dtype)

    def add(self, region, start, duration, intensity, period=None, count=1):   # :39-48
        if period is None:
            raise Exception("period is unspecified.")
        mask = torch.zeros((self.n,), dtype=self.dtype)
        mask[region] = 1.0
        self.items.append(Stim(region, mask * intensity, start, duration, intensity, period, count))

    @staticmethod
    def active(s: Stim, t: float) -> bool:                  # :51-58
        p_t = t % s.period
        t_t = t / s.period
        return t_t <= s.count and (p_t >= s.start and p_t <= s.start + s.duration)

    def apply(self, t):                                     # :51-63
        act = [s.stimulus for s in self.items if self.active(s, t)]
        if act:
            return torch.stack(act).sum(dim=0)
        return self.zero


# --------------------------------------------------------------------------
# LUT interpolation shared by TTP and CRN (TenTusscherPanfilov.py:188-195)
# --------------------------------------------------------------------------
def interpolate(X, table, mn, mx, res, step, mx_idx):
    X = torch.clamp(X, mn, mx)
    idx = ((X - mn) * step).to(torch.long)
    lo = torch.clamp(idx, 0, mx_idx - 1)
    hi = lo + 1
    lo_pos = lo * res + mn
    w = ((X - lo_pos) / res).unsqueeze(1)
    return (1 - w) * table[lo] + w * table[hi]


def lut_grid(mn, mx, res, dtype):
    """The fp32 ``torch.arange`` grid the reference tables are built on."""
    return torch.arange(mn, mx, res).to(dtype)


# --------------------------------------------------------------------------
# ModifiedMS2v  (torchcor/ionic/ModifiedMS2v.py:4-44)
# --------------------------------------------------------------------------
class ModifiedMS2v:
    """Dimensional two-variable Mitchell-Schaeffer model, forward-Euler gate."""

    name = "ModifiedMS2v"

    def __init__(self, dt, dtype=torch.float32):
        self.tau_in, self.tau_out = 0.1, 9.0
        self.tau_open, self.tau_close = 100.0, 120.0
        self.u_gate, self.u_crit = 0.13, 0.13
        self.vmin, self.vmax = -80.0, 20.0
        self.dt = dt
        self.dtype = dtype

    @property
    def DV(self):
        return self.vmax - self.vmin

    def initialize(self, n):                                # :31-34
        self.H = torch.full((n,), 1.0, dtype=self.dtype)
        return torch.full((n,), self.vmin, dtype=self.dtype)

    def states(self):
        return {"H": self.H}

    def differentiate(self, U):                             # :36-44
        DV = self.vmax - self.vmin
        Uad = (U - self.vmin) / DV
        J_in = -1.0 * self.H * Uad * (Uad - self.u_crit) * (1.0 - Uad) / self.tau_in
        J_out = (1.0 - self.H) * Uad / self.tau_out
        dU = -(DV * (J_in + J_out))
        dH = torch.where(Uad > self.u_gate, -self.H / self.tau_close, (1 - self.H) / self.tau_open)
        self.H += self.dt * dH
        return dU


# --------------------------------------------------------------------------
# TenTusscherPanfilov  (torchcor/ionic/TenTusscherPanfilov.py:6-454)
# --------------------------------------------------------------------------
TTP_STATES = ["CaSR", "CaSS", "Cai", "D", "F", "F2", "FCaSS", "H", "J", "Ki",
              "M", "Nai", "R", "R_", "S", "Xr1", "Xr2", "Xs"]
TTP_V_COLS = ["D_A", "D_B", "F2_A", "F2_B", "F_A", "F_B", "H_A", "H_B", "INaCa_A", "INaCa_B",
              "J_A", "J_B", "M_A", "M_B", "R_A", "R_B", "S_A", "S_B", "Xr1_A", "Xr1_B",
              "Xr2_A", "Xr2_B", "Xs_A", "Xs_B", "a2", "rec_iNaK", "rec_ipK"]     # :98-125
TTP_CASS_COLS = ["CaSS2", "FCaSS_A", "FCaSS_B"]                                    # :92-95


class TenTusscherPanfilov:
    name = "TenTusscherPanfilov"

    def __init__(self, cell_type, dt, dtype=torch.float32):
        self.cell_type = "EPI" if cell_type is None else cell_type
        P = dict(  # parameters and constants, :12-89
            CaSR_init=1.3, CaSS_init=0.00007, Cai_init=0.00007, EC=1.5, F2_init=1., FCaSS_init=1.,
            F_init=1., H_init=0.75, J_init=0.75, Ki_init=138.3, M_init=0., Nai_init=7.67, R__init=1.,
            R_init=0., S_init=1., V_init=-86.2, Vxfer=0.0038, Xr1_init=0., Xr2_init=1., Xs_init=0.,
            d_init=0., k1_=0.15, k2_=0.045, k3=0.060, k4=0.005, maxsr=2.5, minsr=1.,
            Bufc=0.2, Bufsr=10., Bufss=0.4, CAPACITANCE=0.185, Cao=2.0, D_CaL_off=0., Fconst=96485.3415,
            GK1=5.405, GNa=14.838, GbCa=0.000592, GbNa=0.00029, GpCa=0.1238, GpK=0.0146, Kbufc=0.001,
            Kbufsr=0.3, Kbufss=0.00025, KmCa=1.38, KmK=1.0, KmNa=40.0, KmNai=87.5, Ko=5.4, KpCa=0.0005,
            Kup=0.00025, Nao=140.0, Rconst=8314.472, T=310.0, Vc=0.016404, Vleak=0.00036,
            Vmaxup=0.006375, Vrel=0.102, Vsr=0.001094, Vss=0.00005468, knaca=1000., knak=2.724,
            ksat=0.1, n=0.35, pKNa=0.03, scl_tau_f=1., vHalfXs=5., xr2_off=0., GCaL_init=0.00003980,
            GKr_init=0.153)
        P["GKs_init"] = 0.392 if cell_type == "EPI" else 0.098 if cell_type == "MCELL" else 0.392
        P["Gto_init"] = 0.294 if cell_type == "EPI" else 0.294 if cell_type == "MCELL" else 0.073
        self.__dict__.update(P)
        self.dt = dt
        self.dtype = dtype
        # table parameters, :131-150
        self.CaSS_T = (0.00001, 10.0, 0.00001)
        self.V_T = (-800., 800., 0.05)
        self.VEk_T = (-800., 800., 0.05)

    @staticmethod
    def _tparams(T):
        mn, mx, res = T
        step = 1 / res
        return mn, mx, res, step, int((mx - mn) * step) - 1

    def construct_tables(self):                             # :197-318
        dt, dtype = self.dt, self.dtype
        E = torch.exp
        KmNai3 = ((self.KmNai * self.KmNai) * self.KmNai)
        Nao3 = ((self.Nao * self.Nao) * self.Nao)
        RTONF = ((self.Rconst * self.T) / self.Fconst)
        invKmCa_Cao = (1. / (self.KmCa + self.Cao))
        F_RT = (1. / RTONF)
        invKmNai3_Nao3 = (1. / (KmNai3 + Nao3))
        pmf_INaCa = ((self.knaca * invKmNai3_Nao3) * invKmCa_Cao)

        CaSS = lut_grid(*self.CaSS_T, dtype)
        ct = torch.zeros((CaSS.shape[0], 3)).to(dtype)
        FCaSS_inf = ((0.6 / (1. + ((CaSS / 0.05) * (CaSS / 0.05)))) + 0.4)
        tau_FCaSS = ((80. / (1. + ((CaSS / 0.05) * (CaSS / 0.05)))) + 2.)
        ct[:, 2] = E(((-dt) / tau_FCaSS))
        ct[:, 1] = ((-FCaSS_inf) * torch.expm1(((-dt) / tau_FCaSS)))
        self.CaSS_tab = ct

        V = lut_grid(*self.V_T, dtype)
        vt = torch.zeros((V.shape[0], 27)).to(dtype)
        c = {n: i for i, n in enumerate(TTP_V_COLS)}
        D_inf = (1. / (1. + (E((((-8. + self.D_CaL_off) - (V)) / 7.5)))))
        F2_inf = ((0.67 / (1. + (E(((V + 35.) / 7.))))) + 0.33)
        F_inf = (1. / (1. + (E(((V + 20.) / 7.)))))
        H_inf = (1. / ((1. + (E(((V + 71.55) / 7.43)))) * (1. + (E(((V + 71.55) / 7.43))))))
        M_inf = (1. / ((1. + (E(((-56.86 - (V)) / 9.03)))) * (1. + (E(((-56.86 - (V)) / 9.03))))))
        R_inf = (1. / (1. + (E(((20. - (V)) / 6.)))))
        S_inf = (1. / (1. + (E(((V + 20.) / 5.)))))
        Xr1_inf = (1. / (1. + (E(((-26. - (V)) / 7.)))))
        Xr2_inf = (1. / (1. + (E(((V - ((-88. + self.xr2_off))) / 24.)))))
        Xs_inf = (1. / (1. + (E((((-self.vHalfXs) - (V)) / 14.)))))
        vt[:, c["a2"]] = (0.25 * (E(((2. * (V - (15.))) * F_RT))))
        aa_D = ((1.4 / (1. + (E(((-35. - (V)) / 13.))))) + 0.25)
        aa_F = (1102.5 * (E((((-(V + 27.)) * (V + 27.)) / 225.))))
        aa_F2 = (562. * (E((((-(V + 27.)) * (V + 27.)) / 240.))))
        aa_H = torch.where((V >= -40.), 0., (0.057 * (E(((-(V + 80.)) / 6.8)))))
        aa_J = torch.where((V >= -40.), 0., ((((-2.5428e4 * (E((0.2444 * V)))) - ((6.948e-6 * (E((-0.04391 * V)))))) * (V + 37.78)) / (1. + (E((0.311 * (V + 79.23)))))))
        aa_M = (1. / (1. + (E(((-60. - (V)) / 5.)))))
        aa_Xr1 = (450. / (1. + (E(((-45. - (V)) / 10.)))))
        aa_Xr2 = (3. / (1. + (E(((-60. - (V)) / 20.)))))
        aa_Xs = (1400. / (torch.sqrt((1. + (E(((5. - (V)) / 6.)))))))
        bb_D = (1.4 / (1. + (E(((V + 5.) / 5.)))))
        bb_F = (200. / (1. + (E(((13. - (V)) / 10.)))))
        bb_F2 = (31. / (1. + (E(((25. - (V)) / 10.)))))
        bb_H = torch.where((V >= -40.), (0.77 / (0.13 * (1. + (E(((-(V + 10.66)) / 11.1)))))), ((2.7 * (E((0.079 * V)))) + (3.1e5 * (E((0.3485 * V))))))
        bb_J = torch.where((V >= -40.), ((0.6 * (E((0.057 * V)))) / (1. + (E((-0.1 * (V + 32.)))))), ((0.02424 * (E((-0.01052 * V)))) / (1. + (E((-0.1378 * (V + 40.14)))))))
        bb_M = ((0.1 / (1. + (E(((V + 35.) / 5.))))) + (0.10 / (1. + (E(((V - (50.)) / 200.))))))
        bb_Xr1 = (6. / (1. + (E(((V - (-30.)) / 11.5)))))
        bb_Xr2 = (1.12 / (1. + (E(((V - (60.)) / 20.)))))
        bb_Xs = (1. / (1. + (E(((V - (35.)) / 15.)))))
        cc_D = (1. / (1. + (E(((50. - (V)) / 20.)))))
        cc_F = ((180. / (1. + (E(((V + 30.) / 10.))))) + 20.)
        cc_F2 = (80. / (1. + (E(((V + 30.) / 10.)))))
        den = (pmf_INaCa / (1. + (self.ksat * (E((((self.n - (1.)) * V) * F_RT))))))
        vt[:, c["rec_iNaK"]] = (1. / ((1. + (0.1245 * (E(((-0.1 * V) * F_RT))))) + (0.0353 * (E(((-V) * F_RT))))))
        vt[:, c["rec_ipK"]] = (1. / (1. + (E(((25. - (V)) / 5.98)))))
        tau_R = ((9.5 * (E((((-(V + 40.)) * (V + 40.)) / 1800.)))) + 0.8)
        if self.cell_type == "ENDO":
            tau_S = ((1000. * (E((((-(V + 67.)) * (V + 67.)) / 1000.)))) + 8.)
        else:
            tau_S = (((85. * (E((((-(V + 45.)) * (V + 45.)) / 320.)))) + (5. / (1. + (E(((V - (20.)) / 5.)))))) + 3.)
        vt[:, c["INaCa_A"]] = ((den * self.Cao) * (E(((self.n * V) * F_RT))))
        vt[:, c["INaCa_B"]] = (((den * (E((((self.n - (1.)) * V) * F_RT)))) * Nao3) * 2.5)
        J_inf = H_inf
        tau_D = ((aa_D * bb_D) + cc_D)
        tau_F2 = ((aa_F2 + bb_F2) + cc_F2)
        tau_F_factor = ((aa_F + bb_F) + cc_F)
        tau_H = (1.0 / (aa_H + bb_H))
        tau_J = (1.0 / (aa_J + bb_J))
        tau_M = (aa_M * bb_M)
        tau_Xr1 = (aa_Xr1 * bb_Xr1)
        tau_Xr2 = (aa_Xr2 * bb_Xr2)
        tau_Xs = ((aa_Xs * bb_Xs) + 80.)
        tau_F = torch.where((V > 0.), (tau_F_factor * self.scl_tau_f), tau_F_factor)
        gates = [("D", D_inf, tau_D), ("F2", F2_inf, tau_F2), ("H", H_inf, tau_H), ("J", J_inf, tau_J),
                 ("M", M_inf, tau_M), ("R", R_inf, tau_R), ("S", S_inf, tau_S), ("Xr1", Xr1_inf, tau_Xr1),
                 ("Xr2", Xr2_inf, tau_Xr2), ("Xs", Xs_inf, tau_Xs), ("F", F_inf, tau_F)]
        for g, inf, tau in gates:       # :262-304 Rush-Larsen A = -inf*expm1(-dt/tau), B = exp(-dt/tau)
            vt[:, c[g + "_B"]] = E(((-dt) / tau))
            vt[:, c[g + "_A"]] = ((-inf) * torch.expm1(((-dt) / tau)))
        self.V_tab = vt

        VEk = lut_grid(*self.VEk_T, dtype)
        et = torch.zeros((VEk.shape[0], 1)).to(dtype)
        a_K1 = (0.1 / (1. + (E((0.06 * (VEk - (200.)))))))
        b_K1 = (((3. * (E((0.0002 * (VEk + 100.))))) + (E((0.1 * (VEk - (10.)))))) / (1. + (E((-0.5 * VEk)))))
        et[:, 0] = (a_K1 / (a_K1 + b_K1))
        self.VEk_tab = et

    def initialize(self, n):                                # :322-351
        self.construct_tables()
        f = lambda v: torch.full((n,), v, dtype=self.dtype)  # noqa: E731
        self.GCaL, self.GKr = f(self.GCaL_init), f(self.GKr_init)
        self.GKs, self.Gto = f(self.GKs_init), f(self.Gto_init)
        init = dict(CaSR=self.CaSR_init, CaSS=self.CaSS_init, Cai=self.Cai_init, D=self.d_init,
                    F=self.F_init, F2=self.F2_init, FCaSS=self.FCaSS_init, H=self.H_init, J=self.J_init,
                    Ki=self.Ki_init, M=self.M_init, Nai=self.Nai_init, R=self.R_init, R_=self.R__init,
                    S=self.S_init, Xr1=self.Xr1_init, Xr2=self.Xr2_init, Xs=self.Xs_init)
        self.s = {k: f(v) for k, v in init.items()}
        return f(self.V_init)

    def states(self):
        return self.s

    def differentiate(self, V):                             # :353-454
        s = self.s
        RTONF = ((self.Rconst * self.T) / self.Fconst)
        inverseVcF = (1. / (self.Vc * self.Fconst))
        inverseVcF2 = (1. / ((2. * self.Vc) * self.Fconst))
        inverseVssF2 = (1. / ((2. * self.Vss) * self.Fconst))
        pmf_INaK = (self.knak * (self.Ko / (self.Ko + self.KmK)))
        sqrt_Ko = (math.sqrt((self.Ko / 5.4)))
        F_RT = (1. / RTONF)
        invVcF_Cm = (inverseVcF * self.CAPACITANCE)
        c = {n: i for i, n in enumerate(TTP_V_COLS)}
        Vr = interpolate(V, self.V_tab, *self._tparams(self.V_T))
        Cr = interpolate(s["CaSS"], self.CaSS_tab, *self._tparams(self.CaSS_T))
        CaSR, CaSS, Cai, Ki, Nai = s["CaSR"], s["CaSS"], s["Cai"], s["Ki"], s["Nai"]

        Eca = ((0.5 * RTONF) * (torch.log((self.Cao / Cai))))
        Ek = (RTONF * (torch.log((self.Ko / Ki))))
        Eks = (RTONF * (torch.log(((self.Ko + (self.pKNa * self.Nao)) / (Ki + (self.pKNa * Nai))))))
        Ena = (RTONF * (torch.log((self.Nao / Nai))))
        IpCa = ((self.GpCa * Cai) / (self.KpCa + Cai))
        a1 = ((((self.GCaL * self.Fconst) * F_RT) * 4.) * torch.where((V == 15.), ((1. / 2.) * F_RT), ((V - (15.)) / (torch.expm1(((2. * (V - (15.))) * F_RT))))))
        ICaL_A = (a1 * Vr[:, c["a2"]])
        ICaL_B = (a1 * self.Cao)
        IKr = ((((self.GKr * sqrt_Ko) * s["Xr1"]) * s["Xr2"]) * (V - (Ek)))
        IKs = (((self.GKs * s["Xs"]) * s["Xs"]) * (V - (Eks)))
        INa = ((((((self.GNa * s["M"]) * s["M"]) * s["M"]) * s["H"]) * s["J"]) * (V - (Ena)))
        INaK = ((pmf_INaK * (Nai / (Nai + self.KmNa))) * Vr[:, c["rec_iNaK"]])
        IbCa = (self.GbCa * (V - (Eca)))
        IbNa = (self.GbNa * (V - (Ena)))
        IpK = ((self.GpK * Vr[:, c["rec_ipK"]]) * (V - (Ek)))
        Ito = (((self.Gto * s["R"]) * s["S"]) * (V - (Ek)))
        VEk = (V - (Ek))
        Er = interpolate(VEk, self.VEk_tab, *self._tparams(self.VEk_T))
        ICaL = ((((s["D"] * s["F"]) * s["F2"]) * s["FCaSS"]) * ((ICaL_A * CaSS) - (ICaL_B)))
        INaCa = ((((Vr[:, c["INaCa_A"]] * Nai) * Nai) * Nai) - ((Vr[:, c["INaCa_B"]] * Cai)))
        IK1 = ((self.GK1 * Er[:, 0]) * (V - (Ek)))
        Iion = (((((((((((IKr + IKs) + IK1) + Ito) + INa) + IbNa) + ICaL) + IbCa) + INaK) + INaCa) + IpCa) + IpK)

        Ileak = (self.Vleak * (CaSR - (Cai)))
        Iup = (self.Vmaxup / (1. + ((self.Kup * self.Kup) / (Cai * Cai))))
        Ixfer = (self.Vxfer * (CaSS - (Cai)))
        diff_Ki = ((-(((((IK1 + Ito) + IKr) + IKs) - ((2. * INaK))) + IpK)) * invVcF_Cm)
        diff_Nai = ((-(((INa + IbNa) + (3. * INaK)) + (3. * INaCa))) * invVcF_Cm)
        kCaSR = (self.maxsr - (((self.maxsr - (self.minsr)) / (1. + ((self.EC / CaSR) * (self.EC / CaSR))))))
        diff_Cai = (((Ixfer - (((((IbCa + IpCa) - ((2. * INaCa))) * inverseVcF2) * self.CAPACITANCE))) - (((Iup - (Ileak)) * (self.Vsr / self.Vc)))) / (1. + (((self.Bufc * self.Kbufc) / (self.Kbufc + Cai)) / (self.Kbufc + Cai))))
        diff_R_ = ((self.k4 * (1. - (s["R_"]))) - ((((self.k2_ * kCaSR) * CaSS) * s["R_"])))
        k1 = (self.k1_ / kCaSR)
        O = (((k1 * Cr[:, 0]) * s["R_"]) / (self.k3 + (k1 * Cr[:, 0])))
        Irel = ((self.Vrel * O) * (CaSR - (CaSS)))
        diff_CaSR = (((Iup - (Irel)) - (Ileak)) / (1. + (((self.Bufsr * self.Kbufsr) / (CaSR + self.Kbufsr)) / (CaSR + self.Kbufsr))))
        diff_CaSS = (((((-Ixfer) * (self.Vc / self.Vss)) + (Irel * (self.Vsr / self.Vss))) + (((-ICaL) * inverseVssF2) * self.CAPACITANCE)) / (1. + (((self.Bufss * self.Kbufss) / (CaSS + self.Kbufss)) / (CaSS + self.Kbufss))))
        dt = self.dt
        s["CaSR"] = CaSR + diff_CaSR * dt
        s["CaSS"] = CaSS + diff_CaSS * dt
        s["Cai"] = Cai + diff_Cai * dt
        s["Ki"] = Ki + diff_Ki * dt
        s["Nai"] = Nai + diff_Nai * dt
        s["R_"] = s["R_"] + diff_R_ * dt
        # Rush-Larsen gates (:414-450)
        s["D"] = Vr[:, c["D_A"]] + Vr[:, c["D_B"]] * s["D"]
        s["F"] = Vr[:, c["F_A"]] + Vr[:, c["F_B"]] * s["F"]
        s["F2"] = Vr[:, c["F2_A"]] + Vr[:, c["F2_B"]] * s["F2"]
        s["FCaSS"] = Cr[:, 1] + Cr[:, 2] * s["FCaSS"]
        for g in ("H", "J", "M", "R", "S", "Xr1", "Xr2", "Xs"):
            s[g] = Vr[:, c[g + "_A"]] + Vr[:, c[g + "_B"]] * s[g]
        return -Iion


# --------------------------------------------------------------------------
# CourtemancheRamirezNattel  (torchcor/ionic/CourtemancheRamirezNattel.py:5-444)
# --------------------------------------------------------------------------
CRN_STATES = ["Ca_rel", "Ca_up", "Cai", "Ki", "d", "f", "f_Ca", "h", "j", "m", "oa", "oi",
              "u", "ua", "ui", "v", "w", "xr", "xs"]
CRN_V_COLS = ["GKur", "INaK", "IbNa", "d_A", "d_B", "f_A", "f_B", "h_A", "h_B", "j_A", "j_B",
              "m_A", "m_B", "oa_A", "oa_B", "oi_A", "oi_B", "ua_A", "ua_B", "ui_A", "ui_B",
              "vrow_29", "vrow_31", "vrow_32", "vrow_36", "vrow_7", "w_A", "w_B", "xr_A", "xr_B",
              "xs_A", "xs_B"]                                                      # :104-137
CRN_CAI_COLS = ["carow_1", "carow_2", "carow_3", "conCa", "f_Ca_A"]                # :96-102
CRN_FN_COLS = ["u_A", "v_A", "v_B"]                                                # :139-143


class CourtemancheRamirezNattel:
    name = "CourtemancheRamirezNattel"

    def __init__(self, dt, dtype=torch.float32):
        P = dict(  # :9-94
            C_B1a=3.79138232501097e-05, C_B1b=0.0811764705882353, C_B1c=0.00705882352941176,
            C_B1d=0.00537112496043221, C_B1e=11.5, C_Fn1=9.648e-13, C_Fn2=2.5910306809e-13,
            C_dCa_rel=8., C_dCaup=0.0869565217391304, Ca_rel_init=1.49, Ca_up_init=1.49,
            Cai_init=1.02e-1, F=96.4867, K_Q10=3., K_up=0.00092, Ki_init=139.0, KmCa=1.38,
            KmCmdn=0.00238, KmCsqn=0.8, KmKo=1.5, KmNa=87.5, KmNa3=669921.875, KmNai=10.,
            KmTrpn=0.0005, Nai=11.2, R=8.3143, T=310., V_init=-81.2, Volcell=20100., Voli=13668.,
            Volrel=96.48, Volup=1109.52, d_init=1.37e-4, f_Ca_init=0.775, f_init=0.999, gamma=0.35,
            h_init=0.965, j_init=0.978, k_rel=30., k_sat=0.1, m_init=2.91e-3, maxCmdn=0.05,
            maxCsqn=10., maxTrpn=0.07, oa_init=3.04e-2, oi_init=0.999, tau_f_Ca=2., tau_tr=180.,
            tau_u=8., u_init=0., ua_init=4.96e-3, ui_init=0.999, v_init=1., w_init=0.999,
            xr_init=3.29e-5, xs_init=1.87e-2,
            ACh=0.000001, Cao=1.8, Cm=100., GACh=0., GCaL=0.1238, GK1=0.09, GKr=0.0294, GKs=0.129,
            GNa=7.8, GbCa=0.00113, GbNa=0.000674, Gto=0.1652, Ko=5.4, Nao=140., factorGKur=1.,
            factorGrel=1., factorGtr=1., factorGup=1., factorhGate=0., factormGate=0.,
            factoroaGate=0., factorxrGate=1., maxCaup=15., maxINaCa=1600., maxINaK=0.60,
            maxIpCa=0.275, maxIup=0.005)
        self.__dict__.update(P)
        self.dt = dt
        self.dtype = dtype
        self.Cai_T = (3e-4, 30.0, 3e-4)                      # :145-167
        self.V_T = (-200., 200., 0.1)
        self.fn_T = (-2e-11, 10.0e-11, 2e-15)
        self.f_Ca_rush_larsen_B = math.exp(((-self.dt) / self.tau_f_Ca))   # :199-200
        self.u_rush_larsen_B = math.exp(((-self.dt) / self.tau_u))

    _tparams = staticmethod(TenTusscherPanfilov._tparams)

    def construct_tables(self):                             # :212-328
        dt, dtype = self.dt, self.dtype
        E = torch.exp
        E_Na = ((self.R * self.T) / self.F) * (math.log((self.Nao / self.Nai)))
        f_Ca_rush_larsen_C = math.expm1(((-dt) / self.tau_f_Ca))
        sigma = ((math.exp((self.Nao / 67.3))) - 1.) / 7.
        u_rush_larsen_C = math.expm1(((-dt) / self.tau_u))

        Cai = lut_grid(*self.Cai_T, dtype)
        ct = torch.zeros((Cai.shape[0], 5)).to(dtype)
        ct[:, 3] = Cai / 1000
        con = ct[:, 3]
        ct[:, 0] = (self.factorGup * self.maxIup) / (1. + (self.K_up / con))
        ct[:, 1] = (((((((self.maxTrpn * self.KmTrpn) / (con + self.KmTrpn)) / (con + self.KmTrpn)) + (((self.maxCmdn * self.KmCmdn) / (con + self.KmCmdn)) / (con + self.KmCmdn))) + 1.) / self.C_B1c) / 1000.)
        ct[:, 2] = (((self.maxIpCa * con) / (0.0005 + con)) - (((((self.GbCa * self.R) * self.T) / 2.) / self.F) * (torch.log((self.Cao / con)))))
        f_Ca_inf = 1. / (1. + (con / 0.00035))
        ct[:, 4] = (-f_Ca_inf) * f_Ca_rush_larsen_C
        self.Cai_tab = ct

        V = lut_grid(*self.V_T, dtype)
        vt = torch.zeros((V.shape[0], 32)).to(dtype)
        c = {n: i for i, n in enumerate(CRN_V_COLS)}
        vt[:, c["GKur"]] = (0.005 + (0.05 / (1. + (E(((15. - V) / 13.))))))
        vt[:, c["IbNa"]] = (self.GbNa * (V - E_Na))
        a_h = torch.where(V >= -40., 0.0, (0.135 * (E((((V + 80.) - self.factorhGate) / -6.8)))))
        a_j = torch.where(V < -40., ((((-127140. * (E((0.2444 * V)))) - (3.474e-5 * (E((-0.04391 * V))))) * (V + 37.78)) / (1. + (E((0.311 * (V + 79.23)))))), 0.)
        a_m = torch.where(V == -47.13, 3.2, ((0.32 * (V + 47.13)) / (1. - (E((-0.1 * (V + 47.13)))))))
        aa_oa = (0.65 / ((E(((V + 10.) / -8.5))) + (E(((30. - V) / 59.0)))))
        aa_oi = (1. / (18.53 + (E(((V + 113.7) / 10.95)))))
        aa_ua = (0.65 / ((E(((V + 10.) / -8.5))) + (E(((V - 30.) / -59.0)))))
        aa_ui = (1. / (21. + (E(((V - 185.) / -28.)))))
        aa_xr = (self.factorxrGate * ((0.0003 * (V + 14.1)) / (1. - (E(((V + 14.1) / -5.))))))
        aa_xs = ((4.e-5 * (V - (19.9))) / (1. - (E(((19.9 - (V)) / 17.)))))
        b_h = torch.where((V >= -40.), ((1. / 0.13) / (1. + (E(((-(V + 10.66)) / 11.1))))), ((3.56 * (E((0.079 * V)))) + (3.1e5 * (E((0.35 * V))))))
        b_j = torch.where((V >= -40.), ((0.3 * (E((-2.535e-7 * V)))) / (1. + (E((-0.1 * (V + 32.)))))), ((0.1212 * (E((-0.01052 * V)))) / (1. + (E((-0.1378 * (V + 40.14)))))))
        b_m = (0.08 * (E(((-(V - self.factormGate)) / 11.))))
        bb_oa = (0.65 / (2.5 + (E(((V + 82.) / 17.)))))
        bb_oi = (1. / (35.56 + (E(((-(V + 1.26)) / 7.44)))))
        bb_ua = (0.65 / (2.5 + (E(((V + 82.) / 17.)))))
        bb_ui = (E(((V - 158.) / 16.)))
        bb_xr = ((1.0 / self.factorxrGate) * ((7.3898e-5 * (V - 3.3328)) / ((E(((V - 3.3328) / 5.1237))) - (1.))))
        bb_xs = ((3.5e-5 * (V - 19.9)) / ((E(((V - 19.9) / 9.))) - 1.))
        d_inf = (1. / (1. + (E(((-(V + 10.)) / 8.)))))
        f_NaK = (1. / ((1. + (0.1245 * (E(((((-0.1 * self.F) * V) / self.R) / self.T))))) + ((0.0365 * sigma) * (E(((((-self.F) * V) / self.R) / self.T))))))
        f_inf = (1. / (1. + (E(((V + 28.) / 6.9)))))
        oa_inf = (1. / (1. + (E(((-((V + 20.47) - self.factoroaGate)) / 17.54)))))
        oi_inf = (1. / (1. + (E(((V + 43.1) / 5.3)))))
        tau_d = torch.where(V == -10., (((1. / 6.24) / 0.035) / 2.), ((((1. - ((E(((-(V + 10.)) / 6.24))))) / 0.035) / (V + 10.)) / (1. + (E(((-(V + 10.)) / 6.24))))))
        tau_f = (9. / ((0.0197 * (E((((-0.0337 * 0.0337) * (V + 10.)) * (V + 10.))))) + 0.02))
        tau_w = (((6. * (1. - (E(((7.9 - V) / 5.))))) / (1. + (0.3 * (E(((7.9 - (V)) / 5.)))))) / (V - (7.9)))
        ua_inf = (1. / (1. + (E(((V + 30.3) / -9.6)))))
        ui_inf = (1. / (1. + (E(((V - 99.45) / 27.48)))))
        vt[:, c["vrow_29"]] = (self.GCaL * (V - 65.))
        vt[:, c["vrow_31"]] = ((((((((self.maxINaCa * (E(((((self.gamma * self.F) * V) / self.R) / self.T)))) * self.Nai) * self.Nai) * self.Nai) * self.Cao) / (self.KmNa3 + ((self.Nao * self.Nao) * self.Nao))) / (self.KmCa + self.Cao)) / (1. + (self.k_sat * (E((((((self.gamma - (1.)) * self.F) * V) / self.R) / self.T))))))
        vt[:, c["vrow_32"]] = ((((((((self.maxINaCa * (E((((((self.gamma - 1.) * self.F) * V) / self.R) / self.T)))) * self.Nao) * self.Nao) * self.Nao) / (self.KmNa3 + ((self.Nao * self.Nao) * self.Nao))) / (self.KmCa + self.Cao)) / (1. + (self.k_sat * (E((((((self.gamma - (1.)) * self.F) * V) / self.R) / self.T)))))) / 1000.)
        vt[:, c["vrow_36"]] = (V * self.GbCa)
        vt[:, c["vrow_7"]] = (self.GNa * (V - E_Na))
        w_inf = (1. - (1. / (1. + (E(((40. - V) / 17.))))))
        xr_inf = (1. / (1. + (E(((V + 14.1) / -6.5)))))
        xs_inf = (1. / (torch.sqrt((1. + (E(((V - 19.9) / -12.7)))))))
        vt[:, c["INaK"]] = ((((self.maxINaK * f_NaK) / (1. + (pow((self.KmNai / self.Nai), 1.5)))) * self.Ko) / (self.Ko + self.KmKo))
        for g, inf, tau in (("d", d_inf, tau_d), ("f", f_inf, tau_f)):
            vt[:, c[g + "_B"]] = (E(((-dt) / tau)))
            vt[:, c[g + "_A"]] = ((-inf) * torch.expm1(((-dt) / tau)))
        for g, a, b in (("h", a_h, b_h), ("j", a_j, b_j), ("m", a_m, b_m)):   # :278-283
            vt[:, c[g + "_A"]] = (((-a) / (a + b)) * (torch.expm1(((-dt) * (a + b)))))
            vt[:, c[g + "_B"]] = (E(((-dt) * (a + b))))
        tau_oa = ((1. / (aa_oa + bb_oa)) / self.K_Q10)
        tau_oi = ((1. / (aa_oi + bb_oi)) / self.K_Q10)
        tau_ua = ((1. / (aa_ua + bb_ua)) / self.K_Q10)
        tau_ui = ((1. / (aa_ui + bb_ui)) / self.K_Q10)
        tau_xr = (1. / (aa_xr + bb_xr))
        tau_xs = (0.5 / (aa_xs + bb_xs))
        for g, inf, tau in (("w", w_inf, tau_w), ("oa", oa_inf, tau_oa), ("oi", oi_inf, tau_oi),
                            ("ua", ua_inf, tau_ua), ("ui", ui_inf, tau_ui), ("xr", xr_inf, tau_xr),
                            ("xs", xs_inf, tau_xs)):
            vt[:, c[g + "_B"]] = (E(((-dt) / tau)))
            vt[:, c[g + "_A"]] = ((-inf) * torch.expm1(((-dt) / tau)))
        self.V_tab = vt

        fn = lut_grid(*self.fn_T, dtype)
        ft = torch.zeros((fn.shape[0], 3)).to(dtype)
        tau_v = (1.91 + (2.09 / (1. + (E(((3.4175e-13 - fn) / 13.67e-16))))))
        u_inf = (1. / (1. + (E(((3.4175e-13 - fn) / 13.67e-16)))))
        v_inf = (1. - (1. / (1. + (E(((6.835e-14 - fn) / 13.67e-16))))))
        ft[:, 0] = ((-u_inf) * u_rush_larsen_C)
        ft[:, 2] = (E(((-dt) / tau_v)))
        ft[:, 1] = ((-v_inf) * (torch.expm1(((-dt) / tau_v))))
        self.fn_tab = ft

    def initialize(self, n):                                # :330-355
        self.construct_tables()
        f = lambda v: torch.full((n,), v, dtype=self.dtype)  # noqa: E731
        self.s = {k: f(getattr(self, k + "_init")) for k in CRN_STATES}
        return f(self.V_init)

    def states(self):
        return self.s

    def differentiate(self, V):                             # :358-444
        s = self.s
        c = {n: i for i, n in enumerate(CRN_V_COLS)}
        Vr = interpolate(V, self.V_tab, *self._tparams(self.V_T))
        Cr = interpolate(s["Cai"], self.Cai_tab, *self._tparams(self.Cai_T))
        E = torch.exp
        E_K = (((self.R * self.T) / self.F) * (torch.log((self.Ko / s["Ki"]))))
        ICaL = (((Vr[:, c["vrow_29"]] * s["d"]) * s["f"]) * s["f_Ca"])
        IKACh = (((self.GACh * (10.0 / (1.0 + (9.13652 / (pow(self.ACh, 0.477811)))))) * (0.0517 + (0.4516 / (1.0 + (E(((V + 59.53) / 17.18))))))) * (V - E_K))
        INa = (((((Vr[:, c["vrow_7"]] * s["m"]) * s["m"]) * s["m"]) * s["h"]) * s["j"])
        INaCa = (Vr[:, c["vrow_31"]] - (s["Cai"] * Vr[:, c["vrow_32"]]))
        vrow_13 = (self.Gto * (V - E_K))
        vrow_18 = ((self.factorGKur * Vr[:, c["GKur"]]) * (V - E_K))
        vrow_21 = ((self.GKr * (V - E_K)) / (1. + (E(((V + 15.) / 22.4)))))
        vrow_24 = (self.GKs * (V - E_K))
        vrow_8 = ((self.GK1 * (V - E_K)) / (1. + (E((0.07 * (V + 80.))))))
        IK1 = vrow_8
        IKr = (vrow_21 * s["xr"])
        IKs = ((vrow_24 * s["xs"]) * s["xs"])
        IKur = ((((vrow_18 * s["ua"]) * s["ua"]) * s["ua"]) * s["ui"])
        IpCa = (Cr[:, 2] + Vr[:, c["vrow_36"]])
        Ito = ((((vrow_13 * s["oa"]) * s["oa"]) * s["oa"]) * s["oi"])
        Iion = INa + IK1 + Ito + IKur + IKr + IKs + ICaL + IpCa + INaCa + Vr[:, c["IbNa"]] + Vr[:, c["INaK"]] + IKACh

        Itr = ((self.factorGtr * (s["Ca_up"] - s["Ca_rel"])) / self.tau_tr)
        Irel = ((((((self.factorGrel * s["u"]) * s["u"]) * s["v"]) * self.k_rel) * s["w"]) * (s["Ca_rel"] - (Cr[:, 3])))
        dIups = (Cr[:, 0] - ((self.maxIup / self.maxCaup) * s["Ca_up"]))
        diff_Ca_rel = ((Itr - Irel) / (1. + ((self.C_dCa_rel / (s["Ca_rel"] + self.KmCsqn)) / (s["Ca_rel"] + self.KmCsqn))))
        diff_Ki = ((-((((((Ito + IKr) + IKur) + IKs) + IK1) + IKACh) - (2.0 * Vr[:, c["INaK"]]))) / (self.F * self.Voli))
        diff_Ca_up = (dIups - (Itr * self.C_dCaup))
        diff_Cai = ((((self.C_B1d * (((INaCa + INaCa) - IpCa) - ICaL)) - (self.C_B1e * dIups)) + Irel) / Cr[:, 1])
        dt = self.dt
        s["Ca_rel"] = s["Ca_rel"] + diff_Ca_rel * dt
        s["Ca_up"] = s["Ca_up"] + diff_Ca_up * dt
        s["Cai"] = s["Cai"] + diff_Cai * dt
        s["Ki"] = s["Ki"] + diff_Ki * dt

        fn = ((self.C_Fn1 * Irel) - (self.C_Fn2 * (ICaL - (0.4 * INaCa))))
        Fr = interpolate(fn, self.fn_tab, *self._tparams(self.fn_T))
        s["d"] = Vr[:, c["d_A"]] + Vr[:, c["d_B"]] * s["d"]
        s["f"] = Vr[:, c["f_A"]] + Vr[:, c["f_B"]] * s["f"]
        s["f_Ca"] = Cr[:, 4] + self.f_Ca_rush_larsen_B * s["f_Ca"]
        s["h"] = Vr[:, c["h_A"]] + Vr[:, c["h_B"]] * s["h"]
        s["j"] = Vr[:, c["j_A"]] + Vr[:, c["j_B"]] * s["j"]
        s["m"] = Vr[:, c["m_A"]] + Vr[:, c["m_B"]] * s["m"]
        s["oa"] = Vr[:, c["oa_A"]] + Vr[:, c["oa_B"]] * s["oa"]
        s["oi"] = Vr[:, c["oi_A"]] + Vr[:, c["oi_B"]] * s["oi"]
        s["u"] = Fr[:, 0] + self.u_rush_larsen_B * s["u"]
        s["ua"] = Vr[:, c["ua_A"]] + Vr[:, c["ua_B"]] * s["ua"]
        s["ui"] = Vr[:, c["ui_A"]] + Vr[:, c["ui_B"]] * s["ui"]
        s["v"] = Fr[:, 1] + Fr[:, 2] * s["v"]
        s["w"] = Vr[:, c["w_A"]] + Vr[:, c["w_B"]] * s["w"]
        s["xr"] = Vr[:, c["xr_A"]] + Vr[:, c["xr_B"]] * s["xr"]
        s["xs"] = Vr[:, c["xs_A"]] + Vr[:, c["xs_B"]] * s["xs"]
        return -Iion


IONIC = {"ModifiedMS2v": ModifiedMS2v, "MitchellSchaeffer": ModifiedMS2v,
         "TenTusscherPanfilov": TenTusscherPanfilov, "CourtemancheRamirezNattel": CourtemancheRamirezNattel}


# --------------------------------------------------------------------------
# the monodomain solve loop  (torchcor/simulator/monodomain.py:18-226)
# --------------------------------------------------------------------------
@dataclass
class Result:
    AT: torch.Tensor
    RT: torch.Tensor
    Vm: torch.Tensor            # (nsnap+1, N)
    n_total_iter: int
    iters: list = field(default_factory=list)
    system: System = None


class Monodomain:
    """CPU restatement of ``Monodomain`` (monodomain.py:18-226), minus NVML/IO."""

    Chi, Cm, theta = 140, 0.01, 0.5                         # :44-46

    def __init__(self, ionic_model, T, dt, dtype=None):
        self.ionic = ionic_model
        self.T, self.dt = T, dt
        self.nt = int(T / dt)                               # :25
        self.dtype = dtype if dtype is not None else torch.float32

    def load_arrays(self, nodes, elems, regions, fibres):   # :60-73 after parsing
        self.n_nodes = nodes.shape[0]
        self.nodes = torch.from_numpy(np.asarray(nodes)).to(dtype=self.dtype)
        self.elems = torch.from_numpy(np.asarray(elems)).to(dtype=torch.int)
        self.regions = torch.from_numpy(np.asarray(regions)).to(dtype=torch.int)
        self.fibres = torch.from_numpy(np.asarray(fibres)).to(dtype=self.dtype)
        self.stimuli = Stimuli(self.n_nodes, self.dtype)
        self.conductivity = Conductivity(self.regions, dtype=self.dtype)

    def load_mesh(self, path, unit_conversion=1000):
        self.load_arrays(*read_mesh(path, unit_conversion))

    def add_stimulus(self, vtx, start, duration, intensity, period=None, count=1):   # :75-78
        region = vtx if isinstance(vtx, torch.Tensor) else read_vtx(vtx)
        self.stimuli.add(region, start, duration, intensity, self.T if period is None else period, count)

    def add_conductivity(self, region_ids, il, it, el=None, et=None):
        self.conductivity.add(region_ids, il, it, el, et)

    def assemble(self):                                     # :83-106
        _, _, sm = self.conductivity.sigma(self.fibres)
        self.system = build_system(self.nodes, self.elems, sm, self.dt, self.dtype, self.Chi, self.Cm, self.theta)
        self.cg = PCG(self.system.PC, self.system.A, dtype=torch.float64)

    def phie_recovery(self, Vm, a_tol=1e-5, r_tol=1e-5, max_iter=100):   # :254-286
        """Extracellular potential of every Vm frame: K(sigma_i + sigma_e) phi = -K(sigma_i) V
        by Jacobi-PCG in float64 with the linear-extrapolation guess across frames, then
        phi -= mean(phi) in place on the returned tensor (which, for float64 frames, is the
        solver's own x, as in the reference)."""
        si, se, _ = self.conductivity.sigma(self.fibres)
        local = tri_surface_local_matrices if self.elems.shape[1] == 3 else tet_local_matrices
        n = self.nodes.shape[0]
        Me, Ke = local(self.nodes, self.elems, si + se, self.dtype)
        K_ie, _ = scatter_coo(self.elems, Me, Ke, n, self.dtype)
        Me, Ke = local(self.nodes, self.elems, si, self.dtype)
        K_i, _ = scatter_coo(self.elems, Me, Ke, n, self.dtype)
        cg = PCG(jacobi(K_ie), K_ie.to_sparse_csr(), dtype=torch.float64)
        cg.initialize(x=torch.zeros_like(Vm[0]), linear_guess=True)
        K_i = K_i.to_sparse_csr()
        out, iters = [], []
        for i in range(Vm.shape[0]):
            b = -K_i @ Vm[i, :]
            phi, it = cg.solve(b, a_tol=a_tol, r_tol=r_tol, max_iter=max_iter)
            phi -= phi.mean()
            out.append(phi)
            iters.append(it)
        return torch.stack(out, dim=0), iters

    def step(self, u, t, a_tol, r_tol, max_iter):           # :109-139
        du = self.ionic.differentiate(u) / 100
        b = u * self.Cm + self.dt * du
        Istim = self.stimuli.apply(t) / 100
        b += self.dt * Istim
        b = self.system.M @ b
        b -= (1 - self.theta) * self.dt * self.system.K @ u
        return self.cg.solve(b, a_tol=a_tol, r_tol=r_tol, max_iter=max_iter)

    def solve(self, a_tol, r_tol, max_iter, calculate_AT_RT=True, linear_guess=True,
              snapshot_interval=1, n_steps=None, on_step=None):   # :141-226
        self.assemble()
        u = self.ionic.initialize(self.n_nodes)
        u0 = u.clone()
        self.cg.initialize(x=u, linear_guess=linear_guess)
        per_frame = int(snapshot_interval / self.dt)
        AT = torch.ones_like(u0) * -1
        RT = torch.ones_like(u0) * -1
        t = 0
        total = 0
        iters = []
        snaps = [u0]
        nt = self.nt if n_steps is None else min(n_steps, self.nt)
        for n in range(1, nt + 1):
            t += self.dt
            u, it = self.step(u, t, a_tol, r_tol, max_iter)
            total += it
            iters.append(it)
            if calculate_AT_RT:
                AT[(u > 0) & (AT == -1)] = t
                RT[(AT > 0) & (RT == -1) & (u < -70)] = t
            if n % per_frame == 0:
                snaps.append(u.clone())
            if on_step is not None:
                on_step(n, t, u)
        return Result(AT=AT, RT=RT, Vm=torch.stack(snaps, 0), n_total_iter=total, iters=iters,
                      system=self.system)
