"""Mesh ingest on the device: the same arrays, bit for bit, as the host reader
(np.loadtxt's doubles) and the host pattern builder."""
import numpy as np
import pytest
import torch

from tests.golden import cases as C
from tests.helpers import case_mesh_dir

pytestmark = pytest.mark.gpu


def _formats(rng, n):
    """Random doubles written in the ways mesh files write them."""
    vals = np.concatenate([rng.uniform(-3e4, 3e4, n), rng.normal(0, 1, n), rng.uniform(-1, 1, n) * 1e-7,
                           np.round(rng.uniform(-1e4, 1e4, n), 3), rng.integers(-10**6, 10**6, n).astype(float)])
    fmts = ["%.17g", "%.6f", "%.10e", "%.3f", "%g", "%.15g", "%.16e", "%.1f"]
    out = []
    for k, v in enumerate(vals):
        out.append(fmts[k % len(fmts)] % v)
    out += ["0", "-0.0", "+5", "1e-5", "123456789012345678", "0.0000000001234567890123456", "1E+3", "7.",
            "6.123233995736766036e-17", "-1.2345678901234567e-30", "9007199254740993", "1e-40"]
    return out


def test_device_parser_is_correctly_rounded(lib, cuda, tmp_path):
    from torchcor_b200.core.ingest import TextTable
    words = _formats(np.random.default_rng(3), 4000)
    words = words[: len(words) // 3 * 3]
    p = tmp_path / "t.pts"
    with open(p, "w") as f:
        f.write(f"{len(words) // 3}\n")
        for i in range(0, len(words), 3):
            f.write(" ".join(words[i:i + 3]) + ("\r\n" if i % 7 == 0 else "\n"))
    t = TextTable(p, cuda)
    got = t.parse(1, len(words) // 3, 0, 3, False)
    assert got is not None
    want = np.array([float(w) for w in words]).reshape(-1, 3)
    assert np.array_equal(got.cpu().numpy().view(np.int64), want.view(np.int64))


def test_device_parser_flags_what_it_cannot_read_exactly(lib, cuda, tmp_path):
    from torchcor_b200.core.ingest import TextTable
    p = tmp_path / "t.pts"
    p.write_text("2\n1.0 2.0 3.0\n1.2345678901234567890123 2 3\n")   # 23 significant digits
    assert TextTable(p, cuda).parse(1, 2, 0, 3, False) is None
    p.write_text("1\n1 2\n")                                           # too few fields
    assert TextTable(p, cuda).parse(1, 1, 0, 3, False) is None


@pytest.mark.parametrize("name", ["cube6_ms_f32", "ico3_crn_f32", "cube8_ttp_f32", "cfg1_ms_f32"])
def test_device_mesh_equals_host_mesh(lib, cuda, tmp_path, name):
    from torchcor_b200.core.ingest import read_mesh_device
    from torchcor_b200.core.mesh import MeshReader
    d = case_mesh_dir(C.case(name), tmp_path)
    nodes, elems, regions, fibres, on_host = read_mesh_device(d, cuda, 1000)
    assert on_host == []
    hn, he, hr, hf = MeshReader(d).read(1000)
    assert np.array_equal(nodes.cpu().numpy().view(np.int64), hn.view(np.int64))
    assert np.array_equal(elems.cpu().numpy(), he) and np.array_equal(regions.cpu().numpy(), hr)
    assert np.array_equal(fibres.cpu().numpy().view(np.int64), hf.view(np.int64))


@pytest.mark.parametrize("mesh", ["cube", "ico"])
def test_device_pattern_equals_host_pattern(lib, cuda, mesh):
    from torchcor_b200 import meshgen
    from torchcor_b200.core.assemble import build_pattern
    if mesh == "cube":
        nodes, el = meshgen.cube(30, 0.25)
    else:
        nodes, el = meshgen.icosphere_fast(6, 25.0)
    h = build_pattern(el, len(nodes))
    g = build_pattern(torch.from_numpy(el.astype(np.int32)).to(cuda), len(nodes))
    assert g.nnz == h.nnz
    for name in ("rowptr", "col", "slot_ptr", "slot_src", "diag"):
        assert np.array_equal(g.host(name), h.host(name)), name


def test_pattern_row_beyond_device_cap_uses_host_build(lib, cuda):
    """A fan of 400 triangles around node 0 puts 1,200 element contributions in row 0,
    more than one device sort takes: the build falls back to the host and still
    equals it."""
    from torchcor_b200.core.assemble import build_pattern
    m = 400
    el = np.array([(0, 1 + i, 1 + (i + 1) % m) for i in range(m)], dtype=np.int32)
    h = build_pattern(el, m + 1)
    g = build_pattern(torch.from_numpy(el).to(cuda), m + 1)
    assert g.nnz == h.nnz == (1 + m) + 4 * m      # hub row, rim rows (self, hub, two neighbours)
    for name in ("rowptr", "col", "slot_ptr", "slot_src", "diag"):
        assert np.array_equal(g.host(name), h.host(name)), name
