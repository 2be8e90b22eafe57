"""ctypes binding of ``libtcb200.so`` (declarations in ``include/tcb200.h``).

The library is loaded on first use.  There is no fallback: if it is missing
or cannot be loaded, every compute entry point raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libtcb200.so"

TCB_OK = 0
TCB_EINVAL = -1
TCB_ECUDA = -2
TCB_ETIMEOUT = -3
TCB_ENOMEM = -4
TCB_ERANGE = -5
TCB_SLICE = 32
TCB_MAX_STIMULI = 32
MODEL_MS, MODEL_TTP, MODEL_CRN = 1, 2, 3

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_f64 = C.c_double
_pi64 = C.POINTER(C.c_int64)


class tcb_mono(C.Structure):
    """Mirror of ``struct tcb_mono``."""
    _fields_ = [
        ("n_nodes", _i64), ("n_pad", _i64), ("n_slices", _i64), ("nt", _i64),
        ("model", _i32), ("n_states", _i32),
        ("slice_ptr", _vp), ("col", _vp), ("col_delta", _vp), ("m_val", _vp), ("k_val", _vp), ("a_val", _vp), ("d_inv", _vp),
        ("state", _vp), ("tables", _vp),
        ("x", _vp), ("bprime", _vp), ("r", _vp), ("p", _vp), ("ap", _vp), ("z", _vp), ("p2", _vp),
        ("at", _vp), ("rt", _vp),
        ("snapshots", _vp),
        ("stim_bits", _vp), ("step_t", _vp), ("step_stim", _vp), ("stim_amp", C.c_float * TCB_MAX_STIMULI),
        ("a_tol", _f64), ("r_tol", _f64),
        ("max_iter", _i32), ("linear_guess", _i32), ("at_rt", _i32), ("per_frame", _i32), ("a_split", _i32),
        ("cm", C.c_float), ("dt", C.c_float), ("snap_ring", _i32), ("ionic_variant", _i32), ("cg_per_sm", _i32),
        ("fused_step", _i32),
        ("step_iters", _vp), ("counter", _vp), ("scratch", _vp), ("barrier", _vp),
        ("params", _vp),
        ("node_params", _vp),
    ]


class tcb_batch_plan(C.Structure):
    """Mirror of ``struct tcb_batch_plan``."""
    _fields_ = [
        ("workspace", _vp),
        ("n_sims", _i32), ("cg_blocks", _i32), ("cg_smem", _i32), ("n_groups", _i32),
        ("group_model", _i32 * 3), ("group_shared", _i32 * 3), ("cg_variant", _i32), ("cg_stage_bytes", _i32),
        ("cg_stage_ok", _i32), ("cg_flags", _i32),
        ("group_tiles", _i64 * 3),
        ("total_slices", _i64), ("group_consts", (C.c_char * 1024) * 3),
        ("ionic_tiles_per_block", _i32), ("ionic_blocks_per_sm", _i32), ("ionic_staged", _i32),
        ("ionic_stage_ok", _i32),
    ]


# (name, restype, argtypes) of every entry point in include/tcb200.h
SIGNATURES = [
    ("tcb_version", C.c_int, []),
    ("tcb_status_string", C.c_char_p, [C.c_int]),
    ("tcb_last_error", C.c_int, [C.c_char_p, _i64]),
    ("tcb_pattern_size", C.c_int, [_vp, _i64, _i32, _i64, _pi64]),
    ("tcb_pattern_build", C.c_int, [_vp, _i64, _i32, _i64, _vp, _vp, _vp, _vp, _vp]),
    ("tcb_text_scratch", _i64, [_i64]),
    ("tcb_text_newlines", C.c_int, [_vp, _i64, _vp, _vp, _i64, _pi64, _vp]),
    ("tcb_text_parse", C.c_int, [_vp, _i64, _vp, _i64, _i64, _i64, _i32, _i32, _i32, _vp, _vp, _vp]),
    ("tcb_pattern_device", C.c_int, [_vp, _i64, _i32, _i64, _vp, _vp, _vp, _pi64, _vp]),
    ("tcb_pattern_device_emit", C.c_int, [_vp, _vp, _i64, _i32, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("tcb_sell_layout", C.c_int, [_vp, _i64, _vp, _pi64]),
    ("tcb_assemble_local", C.c_int, [_i32, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("tcb_assemble_gather", C.c_int, [_i32, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    ("tcb_assemble_system", C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _f64, _f64, _f64, _f64, _vp, _vp, _vp, _vp,
                                      _vp]),
    ("tcb_sell_delta", C.c_int, [_i64, _vp, _i64, _vp, _vp, _vp, _vp]),
    ("tcb_sell_pack", C.c_int, [_i64, _vp, _vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp]),
    ("tcb_model_params", C.c_char_p, [_i32]),
    ("tcb_model_states", C.c_char_p, [_i32]),
    ("tcb_model_layout", C.c_int, [_i32, _vp, _pi64, _pi64]),
    ("tcb_model_table_info", C.c_int, [_i32, _i32, _pi64, C.POINTER(_i32), C.POINTER(_i32), _pi64]),
    ("tcb_ionic_variant", C.c_int, [_i32, _i32, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32),
                                    C.POINTER(_i32), C.POINTER(_i32)]),
    ("tcb_model_tables", C.c_int, [_i32, _vp, _vp, _vp]),
    ("tcb_model_init", C.c_int, [_i32, _vp, _vp, _i64, _vp, _vp]),
    ("tcb_model_node_params", C.c_char_p, [_i32]),
    ("tcb_model_differentiate", C.c_int, [_i32, _vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp, _vp]),
    ("tcb_mono_scratch_doubles", _i64, []),
    ("tcb_mono_run", C.c_int, [C.POINTER(tcb_mono), _i64, _i64, _vp]),
    ("tcb_mono_cg_run", C.c_int, [C.POINTER(tcb_mono), _i64, _i64, _vp]),
    ("tcb_mono_profile", C.c_int, [C.POINTER(tcb_mono), _i64, _i64, _vp, C.POINTER(_f64), C.POINTER(_f64)]),
    ("tcb_mono_cg_kernel", C.c_int, [C.POINTER(tcb_mono)]),
    ("tcb_mono_run_noalloc", C.c_int, [C.POINTER(tcb_mono), _i64, _i64, _vp]),
    ("tcb_mono_finish", C.c_int, [C.POINTER(tcb_mono), _vp]),
    ("tcb_mono_check", C.c_int, [C.POINTER(tcb_mono), _vp]),
    ("tcb_batch_workspace_bytes", _i64, [_i32]),
    ("tcb_batch_prepare", C.c_int, [C.POINTER(tcb_mono), _i32, _vp, _i64, C.POINTER(tcb_batch_plan)]),
    ("tcb_batch_set_cg", C.c_int, [C.POINTER(tcb_batch_plan), _i32]),
    ("tcb_batch_set_ionic", C.c_int, [C.POINTER(tcb_batch_plan), _i32, _i32, _i32]),
    ("tcb_batch_run", C.c_int, [C.POINTER(tcb_batch_plan), _i64, _vp]),
    ("tcb_batch_check", C.c_int, [C.POINTER(tcb_batch_plan), _vp]),
]

_lock = threading.Lock()
_lib = None


class TcbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"libtcb200: {message} (status {status})")
        self.status = status


def load():
    """Load and declare ``libtcb200.so`` (raises RuntimeError if unavailable)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m torchcor_b200.build` "
                               "(torchcor_b200 has no CPU fallback)")
        lib = C.CDLL(os.fspath(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status):
    if status != TCB_OK:
        lib = load()
        buf = C.create_string_buffer(1024)
        lib.tcb_last_error(buf, len(buf))
        raise TcbError(status, buf.value.decode(errors="replace") or lib.tcb_status_string(status).decode())
    return status


def ptr(t):
    """Device/host address of a C-contiguous tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        if not t.flags["C_CONTIGUOUS"]:
            raise ValueError("array passed to libtcb200 must be C-contiguous")
        return t.ctypes.data
    if not t.is_contiguous():
        raise ValueError("tensor passed to libtcb200 must be contiguous")
    return t.data_ptr()


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def model_params(model):
    return load().tcb_model_params(model).decode().split(",")


def table_layout(model):
    """[(rows, ncol, stride, offset)] of the model's lookup tables."""
    lib = load()
    out = []
    for i in range(3):
        r, c, st, off = C.c_int64(), C.c_int32(), C.c_int32(), C.c_int64()
        if lib.tcb_model_table_info(model, i, C.byref(r), C.byref(c), C.byref(st), C.byref(off)) != TCB_OK:
            break
        out.append((r.value, c.value, st.value, off.value))
    return out


def model_states(model):
    return load().tcb_model_states(model).decode().split(",")


def model_node_params(model):
    """Names of the model's per-node parameters (rows of tcb_mono.node_params)."""
    s = load().tcb_model_node_params(model).decode()
    return s.split(",") if s else []


def ionic_variants(model):
    """[(nodes_per_thread, blocks_per_sm, fast_math, staged)] of the model's ionic
    kernel instances (instance k + 1 in ``tcb_mono.ionic_variant``); entry 0 is the default."""
    lib = load()
    cnt, v, b, f, st = (C.c_int32() for _ in range(5))
    check(lib.tcb_ionic_variant(model, 0, C.byref(cnt), C.byref(v), C.byref(b), C.byref(f), C.byref(st)))
    out = []
    for k in range(1, cnt.value + 1):
        check(lib.tcb_ionic_variant(model, k, C.byref(cnt), C.byref(v), C.byref(b), C.byref(f), C.byref(st)))
        out.append((v.value, b.value, f.value, st.value))
    return out
