"""Autotuning of launch choices, with the choices cached on disk.

Single simulations (``tune_single``): the instance of the ionic kernel (1, 2
or 4 consecutive nodes per thread, each compiled for a register budget of some
blocks per SM and a division policy; ``_lib.ionic_variants``), the blocks per SM
of the CG kernel that keeps rows in shared memory (1 or 2, where the rows fit),
and whether a step runs as two launches or as the fused one.  Each
candidate is timed with CUDA events on a scratch copy of the simulation's
mutable device buffers, from the simulation's current step, so the simulation
itself is untouched; the key is the device, the model and log2 buckets of the
node count and of the non-zeros per row.

Batches (``tune_batch``): the batched CG kernel variant: 2 = streaming, sized for 2 blocks per SM
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


BATCH_IONIC_TPB = (0, 1, 2, 4, 8, 16)   # batched ionic tiles per block (0: sized from the groups)
BATCH_IONIC_BPS = (0, 4, 6, 8, 12)      # its register budget in blocks per SM (0: the default)
BATCH_IONIC_STAGED_BPS = (4, 6, 8)      # register budgets of the staged form


def tune_batch(batch, steps=10, cache=None, force=False):
    """Pick the batched CG variant, then the batched ionic launch (tiles per block,
    then register budget of the unstaged form; the staged form at each of its
    budgets; the fastest of them), for ``batch`` (a prepared ``MonodomainBatch``).

    Uses the cached choice when there is one (unless ``force``); otherwise runs
    ``steps`` real batch steps with each candidate after one untimed step, keeps
    the fastest of each and records them.  Needs ``(steps + 1) x`` (number of
    candidates) steps left in every simulation; with fewer it keeps the defaults
    and records nothing.  Returns ``(variant, timings_ms_per_step or None)``."""
    cache = cache if cache is not None else TuneCache()
    sims = batch.sims
    if not sims:
        return None, None
    key = batch_key(batch.device, [s._sim["struct"].n_nodes for s in sims], [s.ionic_model.name for s in sims])
    hit = None if force else cache.get(key)
    if hit is not None:
        if int(hit["cg_variant"]) in batch.cg_variants():
            batch.set_cg(int(hit["cg_variant"]))
            launch = (int(hit.get("ionic_tiles_per_block", 0)), int(hit.get("ionic_blocks_per_sm", 0)),
                      int(hit.get("ionic_staged", 0)))
            if launch[2] and not batch.ionic_stage_ok():
                launch = (0, 0, 0)        # these arrays do not allow the staged form: defaults
            batch.set_ionic(*launch)
            return int(hit["cg_variant"]), None
    candidates = batch.cg_variants()
    staged_ok = batch.ionic_stage_ok()
    need = (steps + 1) * (len(candidates) + len(BATCH_IONIC_TPB) + len(BATCH_IONIC_BPS) +
                          (len(BATCH_IONIC_STAGED_BPS) if staged_ok else 0))
    if min(s.nt + 1 - s._sim["next_step"] for s in sims) < need:
        return batch.cg_config[0], None
    stream = torch.cuda.current_stream(batch.device)

    def timed():
        batch.step(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.step(steps)
        e1.record(stream)
        e1.synchronize()
        batch.check()
        return e0.elapsed_time(e1) / steps

    times = {}
    for v in candidates:
        batch.set_cg(v)
        times[v] = timed()
    best = min(times, key=times.get)
    batch.set_cg(best)
    tpb_times = {}
    for t in BATCH_IONIC_TPB:
        batch.set_ionic(tiles_per_block=t, blocks_per_sm=0, staged=0)
        tpb_times[t] = timed()
    tpb = min(tpb_times, key=tpb_times.get)
    bps_times = {}
    for b in BATCH_IONIC_BPS:
        batch.set_ionic(tiles_per_block=tpb, blocks_per_sm=b, staged=0)
        bps_times[b] = timed()
    bps = min(bps_times, key=bps_times.get)
    staged_times = {}
    if staged_ok:
        for b in BATCH_IONIC_STAGED_BPS:
            batch.set_ionic(tiles_per_block=0, blocks_per_sm=b, staged=1)
            staged_times[b] = timed()
    staged = bool(staged_times) and min(staged_times.values()) < bps_times[bps]
    if staged:
        sb = min(staged_times, key=staged_times.get)
        batch.set_ionic(tiles_per_block=0, blocks_per_sm=sb, staged=1)
        entry_tpb, entry_bps = 0, sb
    else:
        batch.set_ionic(tiles_per_block=tpb, blocks_per_sm=bps, staged=0)
        entry_tpb, entry_bps = tpb, bps
    cache.put(key, {"cg_variant": best, "ms_per_step": {str(k): v for k, v in times.items()},
                    "ionic_tiles_per_block": entry_tpb, "ionic_blocks_per_sm": entry_bps,
                    "ionic_staged": int(staged),
                    "ionic_ms_per_step": {str(k): v for k, v in tpb_times.items()},
                    "ionic_budget_ms_per_step": {str(k): v for k, v in bps_times.items()},
                    "ionic_staged_ms_per_step": {str(k): v for k, v in staged_times.items()}})
    return best, times


# ---------------------------------------------------------------- single simulations
def single_key(device, n_nodes, nnz, model_name) -> str:
    return (f"mono|{device_key(device)}|nodes2^{int(math.log2(max(n_nodes, 1)))}/"
            f"nnz_per_row2^{int(math.log2(max(nnz / max(n_nodes, 1), 1.0)))}/{model_name}")


class ScratchSim:
    """Copies of a prepared simulation's mutable device buffers and a tcb_mono
    pointing at them (snapshots off): trial launches leave the simulation as it was."""

    def __init__(self, sim):
        import ctypes as C
        from torchcor_b200 import _lib
        d = sim._sim
        src = d["struct"]
        self.orig = {"state": sim.ionic_model.state, "x": d["x"], "bp": d["bp"], "r": d["r"], "p": d["p"],
                     "ap": d["ap"], "z": d["z"], "p2": d["p2"], "at_rt": d["at_rt"], "step_iters": d["step_iters"],
                     "counter": d["counter"], "scratch": d["scratch"], "barrier": d["barrier"]}
        self.buf = {k: v.clone() for k, v in self.orig.items()}
        m = _lib.tcb_mono()
        C.memmove(C.byref(m), C.byref(src), C.sizeof(m))
        b = self.buf
        m.state, m.x, m.bprime, m.r, m.p, m.ap, m.z, m.p2 = (_lib.ptr(b[k]) for k in
                                                            ("state", "x", "bp", "r", "p", "ap", "z", "p2"))
        m.at, m.rt = _lib.ptr(b["at_rt"][0]), _lib.ptr(b["at_rt"][1])
        m.snapshots, m.snap_ring = None, 0
        m.step_iters, m.counter = _lib.ptr(b["step_iters"]), _lib.ptr(b["counter"])
        m.scratch, m.barrier = _lib.ptr(b["scratch"]), _lib.ptr(b["barrier"])
        self.struct = m

    def reset(self):
        for k, v in self.orig.items():
            self.buf[k].copy_(v)


def time_steps(scratch, first, steps, stream):
    """(ionic ms, CG ms) per step over ``steps`` steps from ``first`` on the scratch copy,
    after one untimed step (the first launch of an instance loads it)."""
    import ctypes as C
    from torchcor_b200 import _lib
    lib = _lib.load()
    scratch.reset()
    m = scratch.struct
    _lib.check(lib.tcb_mono_run(C.byref(m), first, first + 1, stream.cuda_stream))
    mi, mc = C.c_double(0.0), C.c_double(0.0)
    _lib.check(lib.tcb_mono_profile(C.byref(m), first + 1, first + 1 + steps, stream.cuda_stream, C.byref(mi),
                                    C.byref(mc)))
    _lib.check(lib.tcb_mono_check(C.byref(m), stream.cuda_stream))
    return mi.value / steps, mc.value / steps


def tune_single(sim, steps=5, cache=None, force=False):
    """Choose the ionic kernel instance and the CG blocks per SM for a prepared
    ``Monodomain`` (after ``prepare`` or ``_setup``) and set them in its tcb_mono.

    Uses the cached choice when there is one (unless ``force``); otherwise times
    every candidate for ``steps`` steps on a scratch copy and records the fastest.
    Needs ``steps + 1`` steps left; with fewer it keeps the defaults.  Returns the
    choice ``{"ionic_variant": k, "cg_per_sm": c, ...}`` (with timings when measured)."""
    import ctypes as C
    from torchcor_b200 import _lib
    cache = cache if cache is not None else TuneCache()
    d = sim._sim
    m = d["struct"]
    model = sim.ionic_model
    key = single_key(sim.device, int(m.n_nodes), int(sim.system.nnz), model.name)
    hit = None if force else cache.get(key)
    shapes = _lib.ionic_variants(model.model_id)
    if hit is not None and 0 <= int(hit.get("ionic_variant", 0)) <= len(shapes):
        m.ionic_variant, m.cg_per_sm = int(hit["ionic_variant"]), int(hit.get("cg_per_sm", 0))
        m.fused_step = int(hit.get("fused_step", 0))
        return dict(hit, cached=True)
    first = d["next_step"]
    if sim.nt + 1 - first < steps + 1:
        return {"ionic_variant": int(m.ionic_variant), "cg_per_sm": int(m.cg_per_sm),
                "fused_step": int(m.fused_step), "measured": False}
    stream = torch.cuda.current_stream(sim.device)
    scratch = ScratchSim(sim)
    t_ion = {}
    for k in range(1, len(shapes) + 1):
        scratch.struct.ionic_variant, scratch.struct.cg_per_sm = k, 0
        t_ion[k] = time_steps(scratch, first, steps, stream)[0]
    best_ion = min(t_ion, key=t_ion.get)
    # the step as two launches (ionic + CG) or as one (fused), for each CG blocks per SM
    t_step = {}
    lib = _lib.load()
    for c in (2, 1):
        for fused in (0, 1):
            st = scratch.struct
            st.ionic_variant, st.cg_per_sm, st.fused_step = best_ion, c, fused
            if lib.tcb_mono_cg_kernel(C.byref(st)) != (2 if fused else 1):   # not resident / not fusable
                continue
            ti, tc = time_steps(scratch, first, steps, stream)
            t_step[(c, fused)] = ti + tc
    best_cg, best_fused = min(t_step, key=t_step.get) if t_step else (0, 0)
    del scratch
    m.ionic_variant, m.cg_per_sm, m.fused_step = best_ion, best_cg, best_fused
    choice = {"ionic_variant": best_ion, "cg_per_sm": best_cg, "fused_step": best_fused,
              "ionic_shape": list(shapes[best_ion - 1]), "ionic_ms": {str(k): v for k, v in t_ion.items()},
              "step_ms": {f"cg{c}_fused{f}": v for (c, f), v in t_step.items()}}
    cache.put(key, choice)
    return dict(choice, measured=True)
