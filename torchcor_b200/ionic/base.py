"""Common machinery of the device ionic models.

A model keeps its Python-level parameters as plain attributes (settable as in
the reference, e.g. ``model.tau_in = 0.15`` before ``initialize``), its state
as one (n_states, n_pad) float32 tensor, structure-of-arrays, and its lookup
tables in one float32 tensor built on the device at ``initialize``.  State
variables read and write as attributes (``model.Cai``) through views of that
tensor, like the reference's per-state tensors.
"""
from __future__ import annotations

import numpy as np
import torch

from torchcor_b200 import _lib
from torchcor_b200._lib import check, ptr, stream_ptr
from torchcor_b200.device import get_device

PAD = 128


class DeviceIonicModel:
    model_id: int = 0
    name: str = ""
    _internal = {"_state", "_tables", "_n", "_n_pad", "_state_names", "_node_params", "_node_set", "_node_names",
                 "device", "dtype", "dt"}

    def __init__(self, dt, device=None, dtype=torch.float32):
        object.__setattr__(self, "_state", None)
        object.__setattr__(self, "_tables", None)
        object.__setattr__(self, "_n", 0)
        object.__setattr__(self, "_n_pad", 0)
        object.__setattr__(self, "_state_names", None)
        object.__setattr__(self, "_node_params", None)
        object.__setattr__(self, "_node_set", False)
        object.__setattr__(self, "_node_names", None)
        self.dt = dt
        self.device = torch.device(device) if device is not None else get_device()
        if dtype not in (None, torch.float32):
            raise NotImplementedError("torchcor_b200 ionic models run in float32 on the device")
        self.dtype = torch.float32

    # ------------------------------------------------------------ parameters
    def _param_value(self, name):
        return float(getattr(self, name))

    def param_array(self) -> np.ndarray:
        names = _lib.model_params(self.model_id)
        return np.array([self._param_value(n) for n in names], dtype=np.float64)

    def node_param_names(self):
        """Per-node parameters of the model (TTP: GCaL, GKr, GKs, Gto - the reference's
        per-node conductance tensors, TenTusscherPanfilov.py:327-330)."""
        if self._node_names is None:
            object.__setattr__(self, "_node_names", _lib.model_node_params(self.model_id))
        return self._node_names

    @property
    def node_params(self):
        """(n_params, n_pad) per-node parameters once a caller set any of them node by
        node after initialize(); None while they are the uniform *_init values."""
        return self._node_params if self._node_set else None

    def state_names(self):
        if self._state_names is None:
            object.__setattr__(self, "_state_names", _lib.model_states(self.model_id))
        return self._state_names

    # ------------------------------------------------------------ device state
    def initialize(self, n_nodes: int) -> torch.Tensor:
        """Build the tables, fill the state with the initial values and return V (n_nodes,)."""
        if self.dt is None:
            raise ValueError(f"{type(self).__name__}: dt is not set")
        lib = _lib.load()
        if self.device.type != "cuda":
            raise RuntimeError("torchcor_b200 ionic models need a CUDA device (no CPU fallback)")
        p = self.param_array()
        ns, nt = C_int64(), C_int64()
        check(lib.tcb_model_layout(self.model_id, ptr(p), ns.ref, nt.ref))
        n_pad = (n_nodes + PAD - 1) // PAD * PAD
        state = torch.empty((ns.value, n_pad), device=self.device, dtype=torch.float32)
        tables = torch.empty((max(nt.value, 1),), device=self.device, dtype=torch.float32)
        v = torch.empty((n_pad,), device=self.device, dtype=torch.float32)
        s = stream_ptr()
        with torch.cuda.device(self.device):
            check(lib.tcb_model_tables(self.model_id, ptr(p), ptr(tables), s))
            check(lib.tcb_model_init(self.model_id, ptr(p), ptr(state), n_pad, ptr(v), s))
        object.__setattr__(self, "_state", state)
        object.__setattr__(self, "_tables", tables)
        object.__setattr__(self, "_n", n_nodes)
        object.__setattr__(self, "_n_pad", n_pad)
        # initialize() fills the per-node parameters with the uniform values, as the reference does
        names = self.node_param_names()
        if names:
            rows = torch.empty((len(names), n_pad), device=self.device, dtype=torch.float32)
            for k, nm in enumerate(names):
                self.__dict__.pop(nm, None)
                rows[k].fill_(float(np.float32(getattr(self, nm + "_init"))))
            object.__setattr__(self, "_node_params", rows)
        object.__setattr__(self, "_node_set", False)
        return v[:n_nodes].clone()

    def differentiate(self, V: torch.Tensor) -> torch.Tensor:
        """dV = -Iion at V, advancing the internal state by dt (one call = one step)."""
        if self._state is None:
            raise RuntimeError("initialize() must be called before differentiate()")
        V = V.to(self.device, torch.float32).contiguous()
        if V.numel() != self._n:
            raise ValueError(f"V has {V.numel()} entries, the model was initialised for {self._n}")
        dv = torch.empty_like(V)
        with torch.cuda.device(self.device):
            check(_lib.load().tcb_model_differentiate(self.model_id, ptr(self.param_array()), ptr(self._tables),
                                                      ptr(self.node_params), ptr(self._state), self._n_pad, self._n,
                                                      ptr(V), ptr(dv), stream_ptr()))
        return dv

    @property
    def state(self):
        """(n_states, n_pad) state tensor (rows in ``state_names()`` order)."""
        return self._state

    @property
    def tables(self):
        return self._tables

    def __getattr__(self, name):
        # only called for attributes not found normally: the state variables and the
        # per-node parameters (before initialize(): the reference's 1-element tensors)
        if name.startswith("__"):
            raise AttributeError(name)
        st = object.__getattribute__(self, "_state")
        if st is not None and name in self.state_names():
            return st[self.state_names().index(name), : self._n]
        if name in self.node_param_names():
            rows = object.__getattribute__(self, "_node_params")
            if rows is not None:
                return rows[self.node_param_names().index(name), : self._n]
            return torch.tensor([float(getattr(self, name + "_init"))], dtype=torch.float32)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        rows = self.__dict__.get("_node_params")
        if rows is not None and name not in self._internal and name in self.node_param_names() and \
                isinstance(value, (torch.Tensor, np.ndarray, float, int)):
            # a per-node parameter set node by node (or to one value) after initialize()
            rows[self.node_param_names().index(name), : self._n] = torch.as_tensor(value, device=rows.device,
                                                                                    dtype=torch.float32)
            object.__setattr__(self, "_node_set", True)
            return
        st = self.__dict__.get("_state")
        if st is not None and name not in self._internal and name in self.state_names() and \
                isinstance(value, (torch.Tensor, np.ndarray)):
            st[self.state_names().index(name), : self._n] = torch.as_tensor(value, device=st.device,
                                                                              dtype=torch.float32)
            return
        object.__setattr__(self, name, value)


class C_int64:
    def __init__(self):
        import ctypes
        self._v = ctypes.c_int64()
        self.ref = ctypes.byref(self._v)

    @property
    def value(self):
        return self._v.value
