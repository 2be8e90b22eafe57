"""Autotuner cache and keys (CPU); the timed choice on a GPU is in test_gpu_batch.py."""
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
