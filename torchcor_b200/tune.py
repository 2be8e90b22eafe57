"""Autotuning of launch choices, with the choices cached on disk.

The one runtime choice that depends on the hardware and on the shape of the
work is the batched CG kernel variant: 2 = streaming, sized for 2 blocks per SM
(64 registers a thread, twice the warps to hide memory latency); 1 = streaming,
1 block per SM (128 registers, no spills); 3 = 1 block per SM with the sliced-ELL
streams staged in shared memory by bulk asynchronous copies (only where every
ELL array is 16-byte aligned).  ``tune_batch`` times each candidate on the batch's own
steps -- real steps that advance every simulation, so nothing is wasted -- and
keeps the fastest; the choice is stored under a key made of the device and a
coarse signature of the batch (log2 buckets of total nodes and of the number of
simulations, and the set of ionic models), so later batches of the same shape
on the same kind of GPU reuse it without timing.

Cache file: ``$TCB_TUNE_CACHE`` if set, else ``~/.cache/torchcor_b200/tune.json``.
"""
from __future__ import annotations

import json
import math
import os
import tempfile
import threading
from pathlib import Path

import torch

CG_VARIANTS = (2, 1, 3)   # batched CG kernel variants, default first


def cache_path() -> Path:
    p = os.environ.get("TCB_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "torchcor_b200" / "tune.json"


class TuneCache:
    """A small JSON key -> choice store (whole-file rewrite, atomic rename)."""

    _lock = threading.Lock()

    def __init__(self, path=None):
        self.path = Path(path) if path is not None else cache_path()

    def load(self) -> dict:
        try:
            return json.loads(self.path.read_text())
        except (OSError, ValueError):
            return {}

    def get(self, key):
        return self.load().get(key)

    def put(self, key, value):
        with self._lock:
            data = self.load()
            data[key] = value
            self.path.parent.mkdir(parents=True, exist_ok=True)
            fd, tmp = tempfile.mkstemp(dir=self.path.parent, prefix=".tune.", suffix=".json")
            with os.fdopen(fd, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)


def device_key(device) -> str:
    props = torch.cuda.get_device_properties(device)
    return f"{props.name}/sm{props.major}{props.minor}x{props.multi_processor_count}"


def batch_signature(n_nodes, models) -> str:
    """Coarse shape of a batch: log2 buckets of total nodes and simulation count, model set."""
    total = int(sum(n_nodes))
    return (f"nodes2^{int(math.log2(max(total, 1)))}/sims2^{int(math.log2(max(len(n_nodes), 1)))}/"
            f"{'+'.join(sorted(set(models)))}")


def batch_key(device, n_nodes, models) -> str:
    return f"batch_cg|{device_key(device)}|{batch_signature(n_nodes, models)}"


def tune_batch(batch, steps=10, cache=None, force=False):
    """Pick the batched CG variant for ``batch`` (a prepared ``MonodomainBatch``).

    Uses the cached choice when there is one (unless ``force``); otherwise runs
    ``steps`` real batch steps with each candidate after one untimed step, keeps
    the fastest and records it.  Needs ``(steps + 1) * len(candidates)`` steps
    left in every simulation; with fewer it keeps the default and records
    nothing.  Returns ``(variant, timings_ms_per_step or None)``."""
    cache = cache if cache is not None else TuneCache()
    sims = batch.sims
    if not sims:
        return None, None
    key = batch_key(batch.device, [s._sim["struct"].n_nodes for s in sims], [s.ionic_model.name for s in sims])
    hit = None if force else cache.get(key)
    if hit is not None:
        if int(hit["cg_variant"]) in batch.cg_variants():
            batch.set_cg(int(hit["cg_variant"]))
            return int(hit["cg_variant"]), None
    candidates = batch.cg_variants()
    need = (steps + 1) * len(candidates)
    if min(s.nt + 1 - s._sim["next_step"] for s in sims) < need:
        return batch.cg_config[0], None
    stream = torch.cuda.current_stream(batch.device)
    times = {}
    for v in candidates:
        batch.set_cg(v)
        batch.step(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.step(steps)
        e1.record(stream)
        e1.synchronize()
        batch.check()
        times[v] = e0.elapsed_time(e1) / steps
    best = min(times, key=times.get)
    batch.set_cg(best)
    cache.put(key, {"cg_variant": best, "ms_per_step": {str(k): v for k, v in times.items()}})
    return best, times
