"""Autotuner cache and keys (CPU); the timed choice on a GPU is in test_gpu_batch.py."""
import ctypes as C
import json

from torchcor_b200 import tune


def test_cache_roundtrip(tmp_path):
    c = tune.TuneCache(tmp_path / "sub" / "tune.json")
    assert c.get("k") is None
    c.put("k", {"cg_variant": 2})
    c.put("k2", {"cg_variant": 1})
    assert c.get("k") == {"cg_variant": 2}
    assert json.loads((tmp_path / "sub" / "tune.json").read_text())["k2"] == {"cg_variant": 1}


def test_cache_survives_garbage(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    c = tune.TuneCache(p)
    assert c.get("x") is None
    c.put("x", {"cg_variant": 1})
    assert c.get("x") == {"cg_variant": 1}


def test_cache_path_env(tmp_path, monkeypatch):
    monkeypatch.setenv("TCB_TUNE_CACHE", str(tmp_path / "t.json"))
    assert tune.cache_path() == tmp_path / "t.json"


def test_batch_signature_buckets():
    a = tune.batch_signature([5000, 70000], ["TenTusscherPanfilov", "ModifiedMS2v"])
    b = tune.batch_signature([6000, 69000], ["ModifiedMS2v", "TenTusscherPanfilov"])
    assert a == b   # same log2 buckets and model set, order-free
    assert tune.batch_signature([5000] * 64, ["ModifiedMS2v"]) != tune.batch_signature([5000] * 2, ["ModifiedMS2v"])


def test_ionic_variant_table(lib):
    from torchcor_b200 import _lib
    for model in (_lib.MODEL_MS, _lib.MODEL_TTP, _lib.MODEL_CRN):
        shapes = _lib.ionic_variants(model)
        assert len(shapes) >= 3
        assert all(v in (1, 2, 4) and b >= 1 and f in (0, 1) and st in (0, 1) for v, b, f, st in shapes)
        assert any(v == 1 and st == 0 for v, _, _, st in shapes)   # the fallback for unaligned arrays
    cnt, v, b, f, st = (C.c_int32() for _ in range(5))
    args = (C.byref(cnt), C.byref(v), C.byref(b), C.byref(f), C.byref(st))
    assert lib.tcb_ionic_variant(_lib.MODEL_TTP, 99, *args) == _lib.TCB_ERANGE
    assert lib.tcb_ionic_variant(7, 0, *args) == _lib.TCB_EINVAL


class _FakeSim:
    def __init__(self, n, name):
        self._sim = {"struct": type("S", (), {"n_nodes": n})()}
        self.ionic_model = type("M", (), {"name": name})()


class _FakeBatch:
    """What tune_batch's cache-hit path touches of a MonodomainBatch."""

    def __init__(self, stage_ok):
        self.device = "cuda:0"
        self.sims = [_FakeSim(5000, "TenTusscherPanfilov"), _FakeSim(7000, "TenTusscherPanfilov")]
        self.stage_ok = stage_ok
        self.cg = self.ionic = None

    def cg_variants(self):
        return (2, 1, 3)

    def set_cg(self, v):
        self.cg = v

    def set_ionic(self, tiles_per_block=None, blocks_per_sm=None, staged=None):
        self.ionic = (tiles_per_block, blocks_per_sm, staged)

    def ionic_stage_ok(self):
        return self.stage_ok


def test_batch_cache_hit_applies_the_recorded_launch(tmp_path, monkeypatch):
    monkeypatch.setattr(tune, "device_key", lambda d: "dev")
    cache = tune.TuneCache(tmp_path / "t.json")
    b = _FakeBatch(True)
    key = tune.batch_key(b.device, [5000, 7000], ["TenTusscherPanfilov"] * 2)
    cache.put(key, {"cg_variant": 3, "ionic_tiles_per_block": 0, "ionic_blocks_per_sm": 6, "ionic_staged": 1})
    assert tune.tune_batch(b, cache=cache) == (3, None)
    assert b.cg == 3 and b.ionic == (0, 6, 1)
    b2 = _FakeBatch(False)                  # these arrays do not allow the staged form
    tune.tune_batch(b2, cache=cache)
    assert b2.cg == 3 and b2.ionic == (0, 0, 0)
    cache.put(key, {"cg_variant": 2})        # an entry without the ionic launch: the defaults
    b3 = _FakeBatch(True)
    tune.tune_batch(b3, cache=cache)
    assert b3.cg == 2 and b3.ionic == (0, 0, 0)
