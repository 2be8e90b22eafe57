"""The C ABI of libtcb200.so and the host-side logic that needs no GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest
import torch

from tests.golden import cases as CS
from tests.helpers import golden

HEADER = Path(__file__).resolve().parent.parent / "include" / "tcb200.h"


def declared_functions():
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tcb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n


def test_python_signatures_cover_header(lib):
    from torchcor_b200 import _lib
    assert sorted(n for n, _, _ in _lib.SIGNATURES) == declared_functions()


def test_status_strings(lib):
    assert lib.tcb_version() >= 1
    assert lib.tcb_status_string(0) == b"ok"
    assert lib.tcb_status_string(-3) == b"device wait timed out"


def test_struct_layout_matches_header(lib):
    from torchcor_b200 import _lib
    # the ctypes mirror must be as large as the C struct the library reads
    src = HEADER.read_text()
    body = src[src.index("typedef struct tcb_mono"):src.index("} tcb_mono;")]
    fields = re.findall(r"\b([a-z_]+)\s*(?:\[[A-Z_]+\])?\s*[;,]", body)
    names = [f for f, *_ in _lib.tcb_mono._fields_]
    for f in names:
        assert f in body, f
    assert C.sizeof(_lib.tcb_mono) % 8 == 0


@pytest.mark.parametrize("model,cls", [(1, "ModifiedMS2v"), (2, "TenTusscherPanfilov"),
                                       (3, "CourtemancheRamirezNattel")])
def test_model_parameter_names_resolve(lib, model, cls):
    from torchcor_b200 import _lib, ionic
    m = getattr(ionic, cls)(*(("ENDO", 0.01) if model == 2 else (0.01,)), device="cpu")
    p = m.param_array()
    assert len(p) == len(_lib.model_params(model))
    assert np.isfinite(p).all()
    ns = C.c_int64()
    nt = C.c_int64()
    assert lib.tcb_model_layout(model, p.ctypes.data, C.byref(ns), C.byref(nt)) == 0
    assert ns.value == len(_lib.model_states(model))


def test_table_sizes_match_reference_arange(lib):
    from torchcor_b200 import ionic
    ns, nt = C.c_int64(), C.c_int64()
    m = ionic.TenTusscherPanfilov("ENDO", 0.01, device="cpu")
    lib.tcb_model_layout(2, m.param_array().ctypes.data, C.byref(ns), C.byref(nt))
    rows = lambda a, b, r: torch.arange(a, b, r).shape[0]  # noqa: E731
    from torchcor_b200 import _lib
    lay = _lib.table_layout(2)
    assert [(r, c) for r, c, _, _ in lay] == [(rows(-800., 800., 0.05), 27), (rows(0.00001, 10.0, 0.00001), 3),
                                             (rows(-800., 800., 0.05), 1)]
    assert [st for _, _, st, _ in lay] == [28, 4, 1]
    assert nt.value == sum(r * st for r, _, st, _ in lay)
    m = ionic.CourtemancheRamirezNattel(0.02, device="cpu")
    lib.tcb_model_layout(3, m.param_array().ctypes.data, C.byref(ns), C.byref(nt))
    lay = _lib.table_layout(3)
    assert [(r, c) for r, c, _, _ in lay] == [(rows(-200., 200., 0.1), 32), (rows(3e-4, 30.0, 3e-4), 5),
                                             (rows(-2e-11, 10.0e-11, 2e-15), 3)]
    assert nt.value == sum(r * st for r, _, st, _ in lay)


@pytest.mark.parametrize("name", ["cube6_ms_f32", "cfg1_ms_f32", "cube8_ttp_f32", "ico3_crn_f32",
                                  "cube4_ms_period_f32"])
def test_pattern_bit_exact(lib, name):
    from torchcor_b200.core.assemble import build_pattern
    case = CS.case(name)
    g = golden(name)
    nodes, elems, _, _ = CS.mesh_arrays(case)
    p = build_pattern(elems, len(nodes))
    assert np.array_equal(p.rowptr, g["crow"])
    assert np.array_equal(p.col, g["col"])
    assert np.array_equal(p.col[p.diag], np.arange(len(nodes)))
    # every element contribution is listed exactly once, in reference COO order per slot
    k = elems.shape[1]
    assert p.slot_ptr[-1] == k * k * len(elems)
    assert np.array_equal(np.sort(p.slot_src), np.arange(k * k * len(elems)))
    E = len(elems)
    src = p.slot_src.astype(np.int64)
    order = ((src % (k * k)) * E + src // (k * k))
    seg = np.repeat(np.arange(p.nnz), np.diff(p.slot_ptr))
    same = seg[1:] == seg[:-1]
    assert (order[1:][same] > order[:-1][same]).all()
    # the listed element entry really lands in that slot
    e, ab = src // (k * k), src % (k * k)
    rows = elems[e, ab // k]
    cols = elems[e, ab % k]
    slot_row = np.repeat(np.arange(len(nodes)), np.diff(p.rowptr))[seg]
    assert np.array_equal(rows, slot_row) and np.array_equal(cols, p.col[seg])


def test_pattern_cube_formula(lib):
    from torchcor_b200 import meshgen
    from torchcor_b200.core.assemble import build_pattern
    for n in (3, 7, 12):
        nodes, elems = meshgen.cube(n, 1.0)
        p = build_pattern(elems, len(nodes))
        assert p.nnz == (n + 1) ** 3 + 2 * (3 * n * (n + 1) ** 2 + 3 * n ** 2 * (n + 1) + n ** 3)


def test_pattern_rejects_bad_input(lib):
    from torchcor_b200._lib import TcbError
    from torchcor_b200.core.assemble import build_pattern
    with pytest.raises(TcbError):
        build_pattern(np.array([[0, 1, 2, 9]]), 4)        # node index out of range
    with pytest.raises(TcbError):
        build_pattern(np.array([[0, 1, 2, 3]]), 6)        # nodes 4, 5 belong to no element


def test_sell_layout(lib):
    rowptr = np.array([0, 3, 5, 9] + [9 + 2 * i for i in range(1, 40)], dtype=np.int32)
    n = len(rowptr) - 1
    sp = np.empty((n + 31) // 32 + 1, dtype=np.int64)
    ne = C.c_int64()
    assert lib.tcb_sell_layout(rowptr.ctypes.data, n, sp.ctypes.data, C.byref(ne)) == 0
    lens = np.diff(rowptr)
    for s in range(len(sp) - 1):
        assert sp[s + 1] - sp[s] == 32 * lens[32 * s: 32 * s + 32].max()
    assert ne.value == sp[-1]


def test_stimulus_schedule_matches_oracle():
    from oracle import port as P
    from torchcor_b200.core.stimulation import Stimuli
    dt, T = 0.01, 12.0
    nt = int(T / dt)
    specs = [(0.0, 1.0, 100, 4.0, 2), (5.0, 1.0, 50, T, 1), (0.3, 0.01, 10, 0.7, 5)]
    ours = Stimuli(10, "cpu", torch.float32)
    ref = P.Stimuli(10, torch.float32)
    for k, (a, d, I, per, cnt) in enumerate(specs):
        ours.add(None, a, d, I, per, cnt, region=[k])
        ref.add(torch.tensor([k]), a, d, I, per, cnt)
    t32, mask = ours.schedule(nt, dt)
    t = 0
    for n in range(1, nt + 1):
        t += dt
        want = sum(1 << k for k, s in enumerate(ref.items) if ref.active(s, t))
        assert mask[n] == want, n
        assert t32[n] == np.float32(t)
        dense = ref.apply(t)
        bits = ours.membership_bits() & mask[n]
        amp = ours.amplitudes()
        got = np.array([sum(amp[k] for k in range(3) if (b >> k) & 1) for b in bits], dtype=np.float32)
        np.testing.assert_array_equal(got, dense.numpy())


def test_mesh_reader_matches_oracle(tmp_path):
    from oracle import port as P
    from torchcor_b200.core.mesh import MeshReader
    for name in ("cube6_ms_f32", "ico3_crn_f32"):
        case = CS.case(name)
        CS.write_case_mesh(case, tmp_path / name)
        a = MeshReader(tmp_path / name).read(1000)
        b = P.read_mesh(tmp_path / name, 1000)
        for x, y in zip(a, b):
            assert x.shape == y.shape and np.array_equal(x, y)


def test_mesh_reader_count_mismatch(tmp_path):
    from torchcor_b200.core.mesh import MeshReader
    d = tmp_path / "bad"
    d.mkdir()
    (d / "m.pts").write_text("3\n0 0 0\n1 0 0\n")
    (d / "m.elem").write_text("1\nTr 0 1 2 1\n")
    (d / "m.lon").write_text("1\n1 0 0\n")
    with pytest.raises(ValueError):
        MeshReader(d).read()


def test_conductivity_matches_oracle():
    from oracle import port as P
    from torchcor_b200.core.conductivity import Conductivity
    reg = torch.tensor([1, 2, 2, 3, 1], dtype=torch.int32)
    fib = torch.nn.functional.normalize(torch.rand(5, 3, dtype=torch.float64), dim=1).float()
    for args in ([([1, 3], 0.5, 0.2), ([2], 0.9, 0.3)], [([1, 2, 3], 0.17, 0.019, 0.62, 0.2)]):
        a, b = Conductivity(reg, torch.float32), P.Conductivity(reg, torch.float32)
        for x in args:
            a.add(*x)
            b.add(*x)
        for u, v in zip(a.calculate_sigma(fib), b.sigma(fib)):
            assert (u is None and v is None) or torch.equal(u, v)


def test_monodomain_requires_cuda():
    from torchcor_b200.ionic import ModifiedMS2v
    from torchcor_b200.simulator import Monodomain
    with pytest.raises(RuntimeError):
        Monodomain(ModifiedMS2v(0.01, device="cpu"), T=1.0, dt=0.01, device="cpu")


def test_rcm_order_is_a_bandwidth_reducing_permutation():
    from torchcor_b200 import meshgen
    from torchcor_b200.simulator.monodomain import rcm_order
    nodes, tris = meshgen.icosphere_fast(4, 25.0)
    p = rcm_order(tris, len(nodes))
    assert np.array_equal(np.sort(p), np.arange(len(nodes)))
    inv = np.empty_like(p)
    inv[p] = np.arange(len(p))
    bw = lambda e: max(np.abs(e[:, i] - e[:, j]).max() for i in range(3) for j in range(3))  # noqa: E731
    assert bw(inv[tris]) * 10 < bw(tris)


def test_pattern_from_cpu_tensor_equals_numpy(lib):
    """build_pattern takes a CPU tensor like a numpy array (host build)."""
    from torchcor_b200 import meshgen
    from torchcor_b200.core.assemble import build_pattern
    nodes, elems = meshgen.cube(5, 1.0)
    h = build_pattern(elems, len(nodes))
    t = build_pattern(torch.from_numpy(np.ascontiguousarray(elems, dtype=np.int32)), len(nodes))
    assert t.nnz == h.nnz
    for name in ("rowptr", "col", "slot_ptr", "slot_src", "diag"):
        assert np.array_equal(t.host(name), h.host(name)), name


def test_solve_loop_graph_replay_accounting():
    """The solve loop's step runner: one plain step before the graph is recorded,
    then whole G-step replays and the rest as plain launches; the graph is recorded
    once per prepared run; G = 0 or a stretch shorter than G runs plain launches."""
    from torchcor_b200.simulator import Monodomain

    class Fake:
        def __init__(self):
            self._sim, self.log = {}, []

        def run_steps(self, n):
            if n:
                self.log.append(("plain", n))
            return n

        def capture_steps(self, g):
            self.log.append(("capture", g))

            def replay():
                self.log.append(("replay", g))
            replay.n_steps = g
            return replay

    f = Fake()
    Monodomain._advance(f, 1000, 7)
    assert f.log[:2] == [("plain", 1), ("capture", 7)]
    assert f.log.count(("replay", 7)) == 142 and f.log[-1] == ("plain", 5)
    assert sum(k for op, k in f.log if op != "capture") == 1000
    f.log.clear()
    Monodomain._advance(f, 100, 7)
    assert ("capture", 7) not in f.log and f.log.count(("replay", 7)) == 14 and f.log[-1] == ("plain", 2)
    f.log.clear()
    Monodomain._advance(f, 5, 7)
    assert f.log == [("plain", 5)]
    g = Fake()
    Monodomain._advance(g, 50, 0)
    assert g.log == [("plain", 50)]


def test_misaligned_tables_rejected_before_any_launch(lib):
    """The ionic kernels read table column pairs as 8-byte vectors: a table pointer
    that is not 16-byte aligned is refused on the host (no device access happens,
    so fake addresses are enough here)."""
    from torchcor_b200 import _lib
    model = _lib.MODEL_TTP
    params = np.zeros(len(_lib.model_params(model)), dtype=np.float64)
    fake = 1 << 20
    st = lib.tcb_model_differentiate(model, _lib.ptr(params), fake + 4, None, fake, 1, 1, fake, fake, None)
    assert st == _lib.TCB_EINVAL
    assert lib.tcb_model_tables(model, _lib.ptr(params), fake + 8, None) == _lib.TCB_EINVAL


def test_misaligned_barrier_words_rejected_before_any_launch(lib):
    """The CG kernels' grid barrier keeps its count and generation in one 64-bit
    word: barrier words that are not 8-byte aligned are refused on the host, before
    any device access (fake addresses are enough)."""
    import ctypes
    from torchcor_b200 import _lib
    m = _lib.tcb_mono()
    fake = 1 << 20
    for name, typ in m._fields_:
        if typ in (ctypes.c_void_p,) or (isinstance(typ, type) and issubclass(typ, ctypes._Pointer)):
            ctypes.memmove(ctypes.addressof(m) + getattr(type(m), name).offset,
                           ctypes.byref(ctypes.c_void_p(fake)), ctypes.sizeof(ctypes.c_void_p))
    m.n_nodes, m.n_pad, m.n_slices, m.nt, m.model = 100, 128, 4, 10, _lib.MODEL_MS
    m.max_iter, m.cm, m.dt = 10, 0.01, 0.01
    m.node_params = None
    ctypes.memmove(ctypes.addressof(m) + type(m).barrier.offset, ctypes.byref(ctypes.c_void_p(fake + 4)),
                   ctypes.sizeof(ctypes.c_void_p))
    assert lib.tcb_mono_run(ctypes.byref(m), 1, 2, None) == _lib.TCB_EINVAL
    buf = ctypes.create_string_buffer(256)
    lib.tcb_last_error(buf, 256)
    assert b"barrier" in buf.value


def test_mitchell_schaeffer_constructor_forms(lib):
    """MitchellSchaeffer(device, dtype) (the reference's form, dt from the simulator)
    and MitchellSchaeffer(dt, device=..., dtype=...) give ModifiedMS2v's parameters."""
    from torchcor_b200 import ionic
    ref_form = ionic.MitchellSchaeffer(torch.device("cpu"), torch.float32)
    assert ref_form.dt is None and ref_form.device == torch.device("cpu") and ref_form.dtype == torch.float32
    str_form = ionic.MitchellSchaeffer("cpu")
    assert str_form.dt is None and str_form.device == torch.device("cpu")
    with_dt = ionic.MitchellSchaeffer(0.02, device="cpu", dtype=torch.float32)
    assert with_dt.dt == 0.02
    base = ionic.ModifiedMS2v(0.02, device="cpu")
    ref_form.dt = 0.02
    assert np.array_equal(ref_form.param_array(), base.param_array())
    assert np.array_equal(with_dt.param_array(), base.param_array())
    assert ref_form.name == "MitchellSchaeffer" and isinstance(ref_form, ionic.ModifiedMS2v)
    with pytest.raises(NotImplementedError):
        ionic.MitchellSchaeffer(torch.device("cpu"), torch.float64)
