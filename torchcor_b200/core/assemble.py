"""P1 assembly on the device (the role of ``torchcor/core/assemble.py``).

``assemble_system`` builds, for one mesh, the CSR pattern and scatter map (host
C++), the element matrices (one thread per element), the deterministic
slot-ordered sums into CSR values, the monodomain system values and the
sliced-ELL copy the solver streams.  ``Matrices3D`` / ``Matrices3DSurface``
keep the reference's class names and return (K, M) as sparse CSR tensors.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from torchcor_b200 import _lib
from torchcor_b200._lib import check, ptr, stream_ptr

PAD = 128


def n_padded(n):
    return (n + PAD - 1) // PAD * PAD


@dataclass
class Pattern:
    """CSR pattern and scatter map: numpy arrays (host build) or device tensors."""
    n_nodes: int
    k: int
    rowptr: object
    col: object
    slot_ptr: object
    slot_src: object
    diag: object
    n_nonzero: int = None

    @property
    def nnz(self):
        return int(self.rowptr[-1]) if self.n_nonzero is None else self.n_nonzero

    def on(self, name, device):
        """One of the arrays as a device tensor."""
        a = getattr(self, name)
        return a if isinstance(a, torch.Tensor) else torch.from_numpy(a).to(device)

    def host(self, name):
        a = getattr(self, name)
        return a.cpu().numpy() if isinstance(a, torch.Tensor) else a


def build_pattern(elems, n_nodes: int) -> Pattern:
    """CSR pattern (equal to the reference's coalesce -> to_sparse_csr) and the
    contribution map in the reference's COO order: host C++ for a numpy array,
    the device build (same arrays, bit for bit) for a CUDA tensor, the host build
    for a CUDA tensor with a row beyond the device build's 1024 contributions."""
    if isinstance(elems, torch.Tensor):
        if not elems.is_cuda:
            elems = elems.numpy()
        else:
            try:
                return build_pattern_device(elems, n_nodes)
            except _lib.TcbError as e:
                if e.status != _lib.TCB_ERANGE:
                    raise
                # a row with more element contributions than the device sort takes
                elems = elems.cpu().numpy()
    lib = _lib.load()
    el = np.ascontiguousarray(elems, dtype=np.int32)
    E, k = el.shape
    nnz = C.c_int64()
    check(lib.tcb_pattern_size(ptr(el), E, k, n_nodes, C.byref(nnz)))
    rowptr = np.empty(n_nodes + 1, dtype=np.int32)
    col = np.empty(nnz.value, dtype=np.int32)
    slot_ptr = np.empty(nnz.value + 1, dtype=np.int32)
    slot_src = np.empty(k * k * E, dtype=np.int32)
    diag = np.empty(n_nodes, dtype=np.int32)
    check(lib.tcb_pattern_build(ptr(el), E, k, n_nodes, ptr(rowptr), ptr(col), ptr(slot_ptr), ptr(slot_src),
                                ptr(diag)))
    return Pattern(n_nodes, k, rowptr, col, slot_ptr, slot_src, diag)


def build_pattern_device(elems: torch.Tensor, n_nodes: int) -> Pattern:
    """``build_pattern`` on the GPU for device-resident elements."""
    lib = _lib.load()
    dev = elems.device
    el = elems.to(torch.int32).contiguous()
    E, k = el.shape
    work = torch.empty(2 * (n_nodes + 1), device=dev, dtype=torch.int64)
    keys = torch.empty(k * k * E, device=dev, dtype=torch.int64)     # uint64 keys
    iwork = torch.empty(2 * n_nodes + 1, device=dev, dtype=torch.int32)
    nnz = C.c_int64()
    s = stream_ptr()
    check(lib.tcb_pattern_device(ptr(el), E, k, n_nodes, ptr(work), ptr(keys), ptr(iwork), C.byref(nnz), s))
    i32 = dict(device=dev, dtype=torch.int32)
    rowptr, col = torch.empty(n_nodes + 1, **i32), torch.empty(nnz.value, **i32)
    slot_ptr, slot_src = torch.empty(nnz.value + 1, **i32), torch.empty(k * k * E, **i32)
    diag = torch.empty(n_nodes, **i32)
    check(lib.tcb_pattern_device_emit(ptr(work), ptr(keys), E, k, n_nodes, ptr(rowptr), ptr(col), ptr(slot_ptr),
                                      ptr(slot_src), ptr(diag), s))
    return Pattern(n_nodes, k, rowptr, col, slot_ptr, slot_src, diag, n_nonzero=nnz.value)


def _elems_on(elems, dev):
    if isinstance(elems, torch.Tensor):
        return elems.to(device=dev, dtype=torch.int32).contiguous()
    return torch.from_numpy(np.ascontiguousarray(elems, dtype=np.int32)).to(dev)


def local_matrices(nodes, elems, sl, st, fibres):
    """(ke (E,k,k), mw (E,)) on the device; mw = volume/20 or area/12."""
    lib = _lib.load()
    E, k = elems.shape
    ke = torch.empty((E, k, k), device=nodes.device, dtype=torch.float32)
    mw = torch.empty((E,), device=nodes.device, dtype=torch.float32)
    check(lib.tcb_assemble_local(k, ptr(nodes), ptr(elems), E, ptr(sl), ptr(st), ptr(fibres), ptr(ke), ptr(mw),
                                 stream_ptr()))
    return ke, mw


@dataclass
class System:
    """Device matrices of one monodomain system."""
    n: int
    n_pad: int
    nnz: int
    rowptr: torch.Tensor          # CSR pattern (int32)
    col: torch.Tensor
    m_val: torch.Tensor           # M
    k_val: torch.Tensor           # K / chi
    a_val: torch.Tensor           # Cm*M + theta*dt*K/chi
    krhs_val: torch.Tensor        # ((1-theta)*dt) * K/chi
    d_inv: torch.Tensor           # 1/diag(A), padded to n_pad
    n_slices: int
    slice_ptr: torch.Tensor       # sliced ELL (int64 offsets)
    sell_col: torch.Tensor
    sell_m: torch.Tensor
    sell_k: torch.Tensor
    sell_a: torch.Tensor
    sell_dcol: torch.Tensor = None   # int16 col - row, or None
    a_split: bool = False            # every A value == fp32(fp32(M*Cm) + K')

    def csr(self, values):
        return torch.sparse_csr_tensor(self.rowptr, self.col, values, size=(self.n, self.n))


def assemble_system(nodes, elems_np, sl, st, fibres, dt, chi=140, cm=0.01, theta=0.5, pattern=None) -> System:
    """Assemble M, K/chi, A and the Jacobi preconditioner (monodomain.py:83-106)."""
    lib = _lib.load()
    dev = nodes.device
    n = nodes.shape[0]
    n_pad = n_padded(n)
    pat = pattern if pattern is not None else build_pattern(elems_np, n)
    nnz = pat.nnz
    k = pat.k
    elems = _elems_on(elems_np, dev)
    ke, mw = local_matrices(nodes, elems, sl, st, fibres)
    slot_ptr = pat.on("slot_ptr", dev)
    slot_src = pat.on("slot_src", dev)
    k_val = torch.empty(nnz, device=dev, dtype=torch.float32)
    m_val = torch.empty(nnz, device=dev, dtype=torch.float32)
    s = stream_ptr()
    check(lib.tcb_assemble_gather(k, ptr(slot_ptr), ptr(slot_src), nnz, ptr(ke), ptr(mw), ptr(k_val), ptr(m_val), s))
    del ke, mw, slot_ptr, slot_src
    diag = pat.on("diag", dev)
    a_val = torch.empty(nnz, device=dev, dtype=torch.float32)
    krhs = torch.empty(nnz, device=dev, dtype=torch.float32)
    d_inv = torch.empty(n_pad, device=dev, dtype=torch.float32)
    a_split = torch.ones(1, device=dev, dtype=torch.int32)
    check(lib.tcb_assemble_system(nnz, n, n_pad, ptr(diag), ptr(k_val), ptr(m_val), float(chi), float(cm), float(dt),
                                  float(theta), ptr(a_val), ptr(krhs), ptr(d_inv), ptr(a_split), s))
    # sliced ELL
    n_slices = (n + _lib.TCB_SLICE - 1) // _lib.TCB_SLICE
    sp = np.empty(n_slices + 1, dtype=np.int64)
    n_entries = C.c_int64()
    rowptr_host = pat.host("rowptr")           # keep the host copy alive across the call
    check(lib.tcb_sell_layout(ptr(rowptr_host), n, ptr(sp), C.byref(n_entries)))
    rowptr = pat.on("rowptr", dev)
    col = pat.on("col", dev)
    slice_ptr = torch.from_numpy(sp).to(dev)
    ne = n_entries.value
    sell_col = torch.empty(ne, device=dev, dtype=torch.int32)
    sell = [torch.empty(ne, device=dev, dtype=torch.float32) for _ in range(3)]
    vin = (C.c_void_p * 3)(ptr(m_val), ptr(krhs), ptr(a_val))
    vout = (C.c_void_p * 3)(*[ptr(t) for t in sell])
    check(lib.tcb_sell_pack(n, ptr(rowptr), ptr(col), ptr(slice_ptr), n_slices, 3, vin, ptr(sell_col), vout, s))
    # int16 column offsets when the mesh ordering keeps every |col - row| < 32768
    dcol = torch.empty(ne, device=dev, dtype=torch.int16)
    mx = torch.zeros(1, device=dev, dtype=torch.int32)
    check(lib.tcb_sell_delta(n, ptr(slice_ptr), n_slices, ptr(sell_col), ptr(dcol), ptr(mx), s))
    if int(mx.item()) >= 32768:
        dcol = None
    return System(n=n, n_pad=n_pad, nnz=nnz, rowptr=rowptr, col=col, m_val=m_val, k_val=k_val, a_val=a_val,
                  krhs_val=krhs, d_inv=d_inv, n_slices=n_slices, slice_ptr=slice_ptr, sell_col=sell_col,
                  sell_m=sell[0], sell_k=sell[1], sell_a=sell[2], sell_dcol=dcol, a_split=bool(a_split.item()))


def assemble_phie(nodes, elems_np, sl_i, st_i, sl_e, st_e, fibres) -> System:
    """Matrices of the extracellular potential recovery (monodomain.py:254-286)
    in the solver's layout: M := K(sigma_i), K' := 0, A := K(sigma_i + sigma_e)
    (each sigma formed per element as st I + (sl - st) f f^T), 1/diag(A).
    A is produced by the monodomain system kernel with Cm = 0, chi = theta = dt = 1,
    which returns K(sigma_i + sigma_e) exactly and a zero K'."""
    lib = _lib.load()
    dev = nodes.device
    n = nodes.shape[0]
    n_pad = n_padded(n)
    pat = build_pattern(elems_np, n)
    nnz, k = pat.nnz, pat.k
    elems = _elems_on(elems_np, dev)
    slot_ptr = pat.on("slot_ptr", dev)
    slot_src = pat.on("slot_src", dev)
    s = stream_ptr()

    def stiffness(sl, st):
        ke, mw = local_matrices(nodes, elems, sl.contiguous(), st.contiguous(), fibres)
        kv = torch.empty(nnz, device=dev, dtype=torch.float32)
        mv = torch.empty(nnz, device=dev, dtype=torch.float32)
        check(lib.tcb_assemble_gather(k, ptr(slot_ptr), ptr(slot_src), nnz, ptr(ke), ptr(mw), ptr(kv), ptr(mv), s))
        return kv, mv

    kie, mass = stiffness(sl_i + sl_e, st_i + st_e)
    ki, _ = stiffness(sl_i, st_i)
    diag = pat.on("diag", dev)
    a_val = torch.empty(nnz, device=dev, dtype=torch.float32)
    zero = torch.empty(nnz, device=dev, dtype=torch.float32)
    d_inv = torch.empty(n_pad, device=dev, dtype=torch.float32)
    check(lib.tcb_assemble_system(nnz, n, n_pad, ptr(diag), ptr(kie), ptr(mass), 1.0, 0.0, 1.0, 1.0,
                                  ptr(a_val), ptr(zero), ptr(d_inv), None, s))
    n_slices = (n + _lib.TCB_SLICE - 1) // _lib.TCB_SLICE
    sp = np.empty(n_slices + 1, dtype=np.int64)
    n_entries = C.c_int64()
    rowptr_host = pat.host("rowptr")           # keep the host copy alive across the call
    check(lib.tcb_sell_layout(ptr(rowptr_host), n, ptr(sp), C.byref(n_entries)))
    rowptr = pat.on("rowptr", dev)
    col = pat.on("col", dev)
    slice_ptr = torch.from_numpy(sp).to(dev)
    ne = n_entries.value
    sell_col = torch.empty(ne, device=dev, dtype=torch.int32)
    sell = [torch.empty(ne, device=dev, dtype=torch.float32) for _ in range(3)]
    vin = (C.c_void_p * 3)(ptr(ki), ptr(zero), ptr(a_val))
    vout = (C.c_void_p * 3)(*[ptr(t) for t in sell])
    check(lib.tcb_sell_pack(n, ptr(rowptr), ptr(col), ptr(slice_ptr), n_slices, 3, vin, ptr(sell_col), vout, s))
    dcol = torch.empty(ne, device=dev, dtype=torch.int16)
    mx = torch.zeros(1, device=dev, dtype=torch.int32)
    check(lib.tcb_sell_delta(n, ptr(slice_ptr), n_slices, ptr(sell_col), ptr(dcol), ptr(mx), s))
    if int(mx.item()) >= 32768:
        dcol = None
    return System(n=n, n_pad=n_pad, nnz=nnz, rowptr=rowptr, col=col, m_val=ki, k_val=kie, a_val=a_val,
                  krhs_val=zero, d_inv=d_inv, n_slices=n_slices, slice_ptr=slice_ptr, sell_col=sell_col,
                  sell_m=sell[0], sell_k=sell[1], sell_a=sell[2], sell_dcol=dcol, a_split=False)


class _Matrices:
    k = 4

    def __init__(self, vertices, elems, device, dtype):
        self.vertices = vertices
        self.elems = elems
        self.device = device
        self.dtype = dtype

    def assemble_matrices(self, sigma_l, sigma_t, fibres):
        """(K, M) as sparse CSR tensors.  The reference takes the (E,3,3) tensor;
        here the per-element (sigma_l, sigma_t, fibre) it is formed from."""
        el = self.elems.cpu().numpy() if isinstance(self.elems, torch.Tensor) else np.asarray(self.elems)
        n = self.vertices.shape[0]
        pat = build_pattern(el, n)
        nodes = self.vertices.to(self.device, torch.float32).contiguous()
        elems = torch.from_numpy(np.ascontiguousarray(el, dtype=np.int32)).to(self.device)
        ke, mw = local_matrices(nodes, elems, sigma_l.to(self.device, torch.float32).contiguous(),
                                sigma_t.to(self.device, torch.float32).contiguous(),
                                fibres.to(self.device, torch.float32).contiguous())
        lib = _lib.load()
        dev = self.device
        k_val = torch.empty(pat.nnz, device=dev, dtype=torch.float32)
        m_val = torch.empty(pat.nnz, device=dev, dtype=torch.float32)
        sp = torch.from_numpy(pat.slot_ptr).to(dev)
        ss = torch.from_numpy(pat.slot_src).to(dev)
        check(lib.tcb_assemble_gather(el.shape[1], ptr(sp), ptr(ss), pat.nnz, ptr(ke), ptr(mw), ptr(k_val),
                                      ptr(m_val), stream_ptr()))
        rp = torch.from_numpy(pat.rowptr).to(dev)
        cl = torch.from_numpy(pat.col).to(dev)
        K = torch.sparse_csr_tensor(rp, cl, k_val, size=(n, n))
        M = torch.sparse_csr_tensor(rp, cl, m_val, size=(n, n))
        return K, M


class Matrices3D(_Matrices):
    """P1 tetrahedra (assemble.py:148-248)."""

    def __init__(self, vertices, tetrahedrons, device, dtype):
        super().__init__(vertices, tetrahedrons, device, dtype)


class Matrices3DSurface(_Matrices):
    """P1 triangles of a surface embedded in 3-D (assemble.py:99-145)."""
    k = 3

    def __init__(self, vertices, triangles, device, dtype):
        super().__init__(vertices, triangles, device, dtype)
