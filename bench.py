#!/usr/bin/env python
"""Benchmark of the monodomain time step (node-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tcb|reference]

Default run (one JSON line):

* headline, ``ttp_cube``: ten Tusscher-Panfilov ENDO on a 100^3-cell tetrahedral
  cube (1,030,301 nodes, 6 M tets), see torchcor_b200/workloads.py.  A step is
  one monodomain time step: ionic update + stimulus + LAT/RT, right-hand side,
  Jacobi-PCG to atol = rtol = 1e-5.  After W warm-up steps the run continues
  untimed to step 400, a per-kernel profile window (steps 401..600, CUDA events
  around every launch, for the roofline) follows, and the K timed steps start at
  step 601 -- after the second stimulus (t = 5 ms), while the fronts travel and
  CG iterates.  K steps timed with CUDA events on the launch stream (replays of
  100-step CUDA graphs), barrier + synchronize on both sides, max over ranks;
  each rank runs an independent replica ("replicas only").  Beside it: the same
  workload's whole T = 100 ms run timed on the device (``full_run``), ``e2e`` (one
  ``Monodomain.solve`` through the public API from host arrays), the roofline of
  the dominant kernel, the CPU baseline, and clocks sampled over all of it.
* ``batch``: 64 cubes of 16..64 nodes per edge, Mitchell-Schaeffer/TTP 50/50,
  stepped together (``MonodomainBatch``) against the same simulations one after
  the other on the single-simulation path, plus a full batched run from host
  arrays (``batch.e2e``).
* ``serving``: a Poisson stream of requests (``--requests``, default 128) served
  with continuous batching: p50/p99 latency, throughput, GPU-busy fraction.

``--impl reference``: rank 0 times the reference's own time step on the host
cores (TorchCor installed under baseline/_ref, torch CPU with every host
thread; the oracle, its CPU restatement, where it is not installed) on the same
workload: assembly untimed, then a bounded number of steps.  The default line
also times the reference's step on the GPU (``reference_gpu``: context, not the
target).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from torchcor_b200 import replicas  # noqa: E402

METRIC = "node-steps/s"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms from the
    first ``mark`` to ``stop``; ``summary`` covers the samples taken inside the
    marked (GPU-busy) segments only.  ``mark(name)`` opens a segment,
    ``mark(None)`` closes the current one."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.samples = []            # (host time, line)
        self.segments = []           # [name, t_open, t_close or None]
        self.thread = None

    def _read(self):
        for line in self.proc.stdout:
            if line.strip():
                self.samples.append((time.perf_counter(), line))

    def mark(self, name):
        now = time.perf_counter()
        if self.segments and self.segments[-1][2] is None:
            self.segments[-1][2] = now
        if name is None:
            return
        if self.proc is None:
            try:
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._read, daemon=True)
                self.thread.start()
            except OSError:
                self.proc = False
        self.segments.append([name, now, None])

    def stop(self):
        self.mark(None)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self, names=None):
        sm, mx, reasons, per = [], None, set(), {}
        for t, line in self.samples:
            seg = next((g for g in self.segments if g[1] <= t <= (g[2] if g[2] is not None else float("inf"))),
                       None)
            if seg is None or (names is not None and seg[0] not in names):
                continue
            f = [x.strip() for x in line.split(",")]
            try:
                v = float(f[1])
                mx = float(f[2])
            except (ValueError, IndexError):
                continue
            sm.append(v)
            per.setdefault(seg[0], []).append(v)
            for nm, r in zip(self.NAMES, f[5:9]):
                if r.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "segments": {k: {"samples": len(v), "sm_mhz": float(np.median(v))}
                                                 for k, v in per.items()}}


def dist_setup(impl):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and impl == "tcb":
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    return world, rank, local


def make_sim(wl, device, T=None):
    from torchcor_b200.ionic import CourtemancheRamirezNattel, ModifiedMS2v, TenTusscherPanfilov
    from torchcor_b200.simulator import Monodomain
    if wl.model == "ttp":
        im = TenTusscherPanfilov(wl.cell_type, wl.dt, device=device)
    elif wl.model == "crn":
        im = CourtemancheRamirezNattel(wl.dt, device=device)
    else:
        im = ModifiedMS2v(wl.dt, device=device)
    sim = Monodomain(im, T=wl.T if T is None else T, dt=wl.dt, device=device)
    sim.load_arrays(wl.nodes_mm, wl.elems, wl.regions, wl.fibres)
    for c in wl.conductivity:
        sim.add_conductivity(**c)
    for s in wl.stimuli:
        sim.add_stimulus(None, s["start"], s["duration"], s["intensity"], period=wl.T, region=s["region"])
    return sim


def oracle_sim(wl):
    from oracle import port as P
    if wl.model == "ttp":
        im = P.TenTusscherPanfilov(wl.cell_type, wl.dt)
    elif wl.model == "crn":
        im = P.CourtemancheRamirezNattel(wl.dt)
    else:
        im = P.ModifiedMS2v(wl.dt)
    sim = P.Monodomain(im, wl.T, wl.dt)
    sim.load_arrays(wl.nodes_mm, wl.elems, wl.regions, wl.fibres)
    for c in wl.conductivity:
        sim.add_conductivity(**c)
    for s in wl.stimuli:
        sim.add_stimulus(torch.from_numpy(np.asarray(s["region"])), s["start"], s["duration"], s["intensity"], wl.T)
    return sim


def time_oracle(wl, budget_s, min_steps=2, max_steps=None, warmup=0):
    """Oracle on the workload: assembly (timed separately), ``warmup`` untimed
    steps, then steps until ``budget_s`` seconds of stepping (at least ``min_steps``)."""
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    sim = oracle_sim(wl)
    t0 = time.perf_counter()
    sim.assemble()
    t_asm = time.perf_counter() - t0
    u = sim.ionic.initialize(sim.n_nodes)
    sim.cg.initialize(u, linear_guess=True)
    t = 0.0
    warmup = min(warmup, wl.nt - 1)
    for _ in range(warmup):
        t += wl.dt
        u, _ = sim.step(u, t, 1e-5, 1e-5, 100)
    n = 0
    el = 0.0
    while (el < budget_s or n < min_steps) and (max_steps is None or n < max_steps) and n + warmup < wl.nt:
        t += wl.dt
        t1 = time.perf_counter()
        u, _ = sim.step(u, t, 1e-5, 1e-5, 100)
        el += time.perf_counter() - t1
        n += 1
    return dict(value=wl.n_nodes * n / el, steps=n, seconds=el, assemble_s=t_asm, cores=cores, warmup=warmup)


REF_DIR = ROOT / "baseline" / "_ref"


def import_reference():
    """The reference package installed under baseline/_ref (``pip install --target``),
    imported with empty stand-ins for its post-processing imports (pyvista,
    matplotlib, the ECG module), which the time step never calls; None if absent."""
    if not (REF_DIR / "torchcor").is_dir():
        return None
    import types
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    for name in ["pyvista", "matplotlib", "matplotlib.pyplot", "matplotlib.animation"]:
        sys.modules.setdefault(name, types.ModuleType(name))
    ecg = types.ModuleType("torchcor.signalanalysis.signalanalysis.ecg_QS")
    ecg.Ecg = None
    sys.modules.setdefault("torchcor.signalanalysis.signalanalysis.ecg_QS", ecg)
    if not torch.cuda.is_available():
        torch.cuda.current_device = lambda: 0      # Monodomain.__init__ asks NVML for the GPU
    import torchcor.core as core
    import torchcor.ionic as ionic
    import torchcor.simulator.monodomain as md
    if not torch.cuda.is_available():
        class _U:
            gpu = 0
            used = 0
        md.nvmlInit = lambda: None
        md.nvmlDeviceGetHandleByIndex = lambda i: None
        md.nvmlDeviceGetUtilizationRates = lambda h: _U()
        md.nvmlDeviceGetMemoryInfo = lambda h: _U()
    return md, ionic, core


class ReferenceRun:
    """The reference's own monodomain time step (Monodomain.step with its ionic
    class, Stimuli, Preconditioner and ConjugateGradient; monodomain.py:109-139) on
    a workload, on the CPU or a GPU.  The mesh arrays are set as load_mesh sets
    them (monodomain.py:60-73) and the stimuli are read from .vtx files by the
    reference; the matrices come from the oracle's restatement of the assembly
    (bit-identical to Matrices3D.assemble_matrices at every size the tests pin),
    because the reference assembles through Python lists (minutes at 6 M tets)
    and assembly is not part of the timed step."""

    def __init__(self, wl, system=None):
        self.wl = wl
        self.mods = import_reference()
        if self.mods is None:
            raise RuntimeError("reference not installed under baseline/_ref")
        if system is None:
            from oracle import port as P
            osim = oracle_sim(wl)
            _, _, sm = osim.conductivity.sigma(osim.fibres)
            t0 = time.perf_counter()
            system = P.build_system(osim.nodes, osim.elems, sm, wl.dt, torch.float32)
            self.assemble_s = time.perf_counter() - t0
        self.system = system

    def build(self, device):
        md, ionic, core = self.mods
        wl = self.wl
        if wl.model == "ttp":
            im = ionic.TenTusscherPanfilov(wl.cell_type, wl.dt, device=device, dtype=torch.float32)
        elif wl.model == "crn":
            im = ionic.CourtemancheRamirezNattel(wl.dt, device=device, dtype=torch.float32)
        else:
            im = ionic.ModifiedMS2v(wl.dt, device=device, dtype=torch.float32)
        sim = md.Monodomain(im, T=wl.T, dt=wl.dt, device=device, dtype=torch.float32)
        sim.n_nodes = wl.n_nodes
        sim.nodes = torch.from_numpy(wl.nodes_mm).to(dtype=torch.float32, device=device)
        sim.elems = torch.from_numpy(np.ascontiguousarray(wl.elems)).to(dtype=torch.int, device=device)
        sim.regions = torch.from_numpy(np.ascontiguousarray(wl.regions)).to(dtype=torch.int, device=device)
        sim.fibres = torch.from_numpy(wl.fibres).to(dtype=torch.float32, device=device)
        sim.stimuli = core.Stimuli(sim.n_nodes, device, torch.float32)
        sim.conductivity = core.Conductivity(sim.regions, dtype=torch.float32)
        for c in wl.conductivity:
            sim.add_conductivity(**c)
        with tempfile.TemporaryDirectory() as d:
            for k, st in enumerate(wl.stimuli):
                f = Path(d) / f"s{k}.vtx"
                idx = np.asarray(st["region"], dtype=np.int64)
                f.write_text(f"{len(idx)}\nintra\n" + "\n".join(str(int(i)) for i in idx) + "\n")
                sim.add_stimulus(str(f), st["start"], st["duration"], st["intensity"], period=wl.T)
        S = self.system
        sim.K = S.K.to(device)
        sim.M = S.M.to(device)
        A = S.A_coo.to(device)
        sim.pcd = core.Preconditioner()
        sim.pcd.create_Jocobi(A)
        sim.A = A.to_sparse_csr()
        sim.cg = core.ConjugateGradient(sim.pcd, sim.A, dtype=torch.float64)
        u = sim.ionic_model.initialize(sim.n_nodes)
        sim.cg.initialize(x=u, linear_guess=True)
        return sim, u

    def time(self, device, warmup, budget_s, min_steps=3, max_steps=None, first_step=1):
        """Steps first_step.. : `warmup` untimed, then until `budget_s` seconds of
        stepping (at least min_steps, at most max_steps).  Returns node-steps/s etc."""
        sim, u = self.build(device)
        wl = self.wl
        t = 0.0
        cuda = torch.device(device).type == "cuda"
        n_done = 0
        while n_done < first_step - 1 + warmup and n_done < wl.nt - 1:
            t += wl.dt
            u, _, _, _ = sim.step(u, t, 1e-5, 1e-5, 100)
            n_done += 1
        if cuda:
            torch.cuda.synchronize(device)
        n, el, iters = 0, 0.0, 0
        while (el < budget_s or n < min_steps) and (max_steps is None or n < max_steps) and n_done < wl.nt:
            t += wl.dt
            t1 = time.perf_counter()
            u, it, _, _ = sim.step(u, t, 1e-5, 1e-5, 100)
            if cuda:
                torch.cuda.synchronize(device)
            el += time.perf_counter() - t1
            n += 1
            n_done += 1
            iters += int(it)
        return dict(value=wl.n_nodes * n / el, steps=n, seconds=el, first=n_done - n + 1,
                    cg_iterations_per_step=iters / max(n, 1))


def reference_arm(a, wl, world, rank):
    if rank != 0:
        return
    # warm-up steps are run untimed inside the same session; the timed sample is
    # bounded to keep the whole run within a few minutes
    budget = float(os.environ.get("TCB_REFERENCE_BUDGET_S", "60"))
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    if import_reference() is not None:
        ref = ReferenceRun(wl)
        r = ref.time("cpu", a.warmup, budget, min_steps=min(a.steps, 3), max_steps=a.steps)
        kind = "reference"
        sample = (f"the reference's Monodomain.step (TorchCor 0.1.8 from baseline/_ref, torch CPU, {cores} threads) "
                  f"on the full workload: {a.warmup} warm-up steps untimed, then {r['steps']} timed steps "
                  f"({r['seconds']:.1f} s); matrices from the oracle's assembly ({ref.assemble_s:.1f} s, untimed)")
        r["warmup"] = a.warmup
    else:
        r = time_oracle(wl, budget_s=budget, min_steps=min(a.steps, 3), max_steps=a.steps, warmup=a.warmup)
        kind = "port"
        sample = (f"oracle (CPU restatement of the reference path, torch CPU, {r['cores']} threads) on the full "
                  f"workload: assembly {r['assemble_s']:.1f} s and {r['warmup']} warm-up steps untimed, then "
                  f"{r['steps']} timed steps ({r['seconds']:.1f} s)")
    v = r["value"]
    line = {"metric": METRIC, "value": v, "unit": METRIC, "n_gpus": world, "steps": r["steps"], "warmup": r["warmup"],
            "ms_per_step": 1000 * r["seconds"] / r["steps"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": wl.name, "nodes": wl.n_nodes, "elements": int(len(wl.elems)), "dt_ms": wl.dt,
                       "T_ms": wl.T, "parallelism": "replicas only"},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# the timed window starts after the second stimulus of the headline workload (t = 5 ms)
FIRST_TIMED_STEP = 601


def tcb_arm(a, wl, world, rank, local, clk):
    from torchcor_b200 import _lib
    from torchcor_b200.workloads import algorithmic_bytes
    import ctypes as C
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pre = max(a.warmup, FIRST_TIMED_STEP - 1 - a.profile_steps)     # untimed steps before the profile window
    need = pre + a.profile_steps + a.steps
    T_run = max(wl.T, (need + 1) * wl.dt)
    sim = make_sim(wl, dev, T=T_run)
    sim.assemble()
    sys_ = sim.system
    sim._setup(1e-5, 1e-5, 100, True, True, 1.0, keep_snapshots=False)
    stream = torch.cuda.current_stream(dev)
    sim.run_steps(a.warmup)
    tuned = sim.autotune()                        # launch shapes for this device and shape (cached)
    sim.run_steps(pre - a.warmup)
    torch.cuda.synchronize(dev)
    lib = _lib.load()
    st = sim._sim["struct"]
    _lib.check(lib.tcb_mono_check(C.byref(st), stream.cuda_stream))
    kind = lib.tcb_mono_cg_kernel(C.byref(st))
    fused = kind == 2
    cg_name = {2: "cg_resident_kernel (fused step)", 1: "cg_resident_kernel", 0: "cg_kernel"}[kind]
    # per-kernel event times for the roofline: steps pre+1 .. pre+profile_steps,
    # each kernel bracketed by events on the launch stream (the same steps every run,
    # so an ncu capture of them measures the same launches)
    msi, msc = C.c_double(0.0), C.c_double(0.0)
    s0 = sim._sim["next_step"]
    torch.cuda.nvtx.range_push("profile_window")      # what the ncu captures in profiles/ select
    _lib.check(lib.tcb_mono_profile(C.byref(st), s0, s0 + a.profile_steps, stream.cuda_stream,
                                    C.byref(msi), C.byref(msc)))
    torch.cuda.nvtx.range_pop()
    sim._sim["next_step"] = s0 + a.profile_steps
    p_iters = sim._sim["step_iters"][s0: s0 + a.profile_steps].sum().item()
    kp = p_iters / a.profile_steps + 1.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the timed steps replay CUDA graphs of G steps (Monodomain.capture_steps), the
    # remainder runs as plain launches
    G = a.graph_steps if 0 < a.graph_steps <= a.steps else 0
    replay = sim.capture_steps(G) if G else None
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    t_first = sim._sim["next_step"]
    clk.mark("headline")
    e0.record(stream)
    done = 0
    if replay:
        for _ in range(a.steps // G):
            replay()
        done = (a.steps // G) * G
    if a.steps > done:
        sim.run_steps(a.steps - done)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    del replay
    ms = replicas.reduce_max(e0.elapsed_time(e1))     # slowest rank (replicas only)
    _lib.check(lib.tcb_mono_check(C.byref(st), stream.cuda_stream))
    iters = sim._sim["step_iters"][t_first: t_first + a.steps].sum().item()
    k_loop = iters / a.steps + 1.0                    # CG loop passes per step (n_iter + 1)
    b_ion, b_rhs, b_iter = algorithmic_bytes(sys_.n, sys_.nnz, sim.ionic_model.state.shape[0])
    t_ion = msi.value / a.profile_steps * 1e-3
    t_cg = msc.value / a.profile_steps * 1e-3
    peak, peak_kind = peaks()
    cg_bytes = b_rhs + kp * b_iter + (b_ion if fused else 0)
    gbs_cg = cg_bytes / t_cg / 1e9
    gbs_ion = b_ion / t_ion / 1e9 if t_ion > 0 else None
    step_bytes = b_ion + b_rhs + k_loop * b_iter
    value = world * wl.n_nodes * a.steps / (ms / 1e3)
    dominant = (cg_name, gbs_cg, cg_bytes) if t_cg >= t_ion else ("mono_ionic_kernel", gbs_ion, b_ion)
    kernels = {cg_name: {"ms_per_launch": 1e3 * t_cg, "bytes": cg_bytes, "GB/s": gbs_cg, "cg_loop_passes": kp}}
    if not fused:
        kernels["mono_ionic_kernel"] = {"ms_per_launch": 1e3 * t_ion, "bytes": b_ion, "GB/s": gbs_ion}
    # DRAM traffic per launch of the dominant kernel over the same profile steps,
    # from an ncu capture (profiles/traffic.json; the capture command is stored there)
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        rec = json.loads(tf.read_text()).get(wl.name, {}).get(dominant[0])
        traffic = rec.get("bytes_per_launch") if isinstance(rec, dict) else None
    del sim
    torch.cuda.empty_cache()

    # the whole run of the workload (T = 100 ms, every step), timed on the device
    full = None
    if not a.no_full_run:
        simf = make_sim(wl, dev)
        simf.assemble()
        simf._setup(1e-5, 1e-5, 100, True, True, 1.0, keep_snapshots=False)
        simf.autotune()
        torch.cuda.synchronize(dev)
        clk.mark("full_run")
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        simf._advance(wl.nt, 100)
        f1.record(stream)
        torch.cuda.synchronize(dev)
        fms = replicas.reduce_max(f0.elapsed_time(f1))
        f_iters = simf._sim["step_iters"][1: wl.nt + 1].sum().item()
        full = {"value": world * wl.n_nodes * wl.nt / (fms / 1e3), "unit": METRIC, "steps": wl.nt,
                "ms_per_step": fms / wl.nt, "cg_iterations_per_step": f_iters / wl.nt,
                "what": "every step 1..nt of the workload on the device (CUDA events; replays of 100-step "
                        "graphs after one plain step), no set-up or download"}
        del simf
        torch.cuda.empty_cache()

    # e2e: one full solve of the workload through the public API from host arrays
    e2e = None
    if not a.no_e2e:
        if world > 1:
            torch.distributed.barrier()
        clk.mark("e2e")
        with tempfile.TemporaryDirectory() as d:
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            sim2 = make_sim(wl, dev)
            sim2.solve(1e-5, 1e-5, 100, calculate_AT_RT=True, linear_guess=True, snapshot_interval=1.0,
                       verbose=False, result_path=d)
            torch.cuda.synchronize(dev)
            wall = time.perf_counter() - t0
            e_iters = int(sim2.n_total_iter)
            h2d = (wl.nodes_mm.size * 4 + wl.elems.size * 4 + wl.regions.size * 4 + wl.fibres.size * 4 +
                   wl.n_nodes * 4 + (wl.nt + 1) * 8)
            d2h = 2 * wl.n_nodes * 4 + (wl.nt // int(1.0 / wl.dt) + 1) * wl.n_nodes * 4 + (wl.nt + 1) * 4
            del sim2
        wall = replicas.reduce_max(wall)
        e2e = {"value": world * wl.n_nodes * wl.nt / wall, "unit": METRIC,
               "h2d_bytes_per_step": int(h2d // wl.nt), "d2h_bytes_per_step": int(d2h // wl.nt),
               "cg_iterations_per_step": e_iters / wl.nt,
               "what": f"one Monodomain.solve of the workload (T={wl.T} ms, {wl.nt} steps) from host arrays: "
                       f"mesh upload, assembly, all steps, AT/RT/Vm download and save; wall {wall:.2f} s"}

    cpu = ref_gpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        clk.mark(None)
        budget = float(os.environ.get("TCB_CPU_BASELINE_S", "15"))
        cores = os.cpu_count() or 1
        torch.set_num_threads(cores)
        if import_reference() is not None:
            ref = ReferenceRun(wl)
            r = ref.time("cpu", 3, budget)
            cpu = {"value": r["value"], "unit": METRIC, "cores": cores, "kind": "reference",
                   "sample": f"the reference's Monodomain.step (TorchCor 0.1.8, torch CPU, {cores} threads) on the "
                             f"full workload: steps {r['first']}..{r['first'] + r['steps'] - 1} timed "
                             f"({r['seconds']:.1f} s) after 3 untimed; matrices from the oracle's assembly "
                             f"({ref.assemble_s:.1f} s, untimed)"}
            if not a.no_reference_gpu:
                # context, not the target: the reference's own PyTorch step on this GPU
                clk.mark("reference_gpu")
                rg = ref.time(dev, 5, 10.0, min_steps=50, max_steps=a.reference_gpu_steps,
                              first_step=FIRST_TIMED_STEP)
                clk.mark(None)
                ref_gpu = {"value": rg["value"], "unit": METRIC, "ms_per_step": 1e3 * rg["seconds"] / rg["steps"],
                           "steps": [rg["first"], rg["first"] + rg["steps"] - 1],
                           "cg_iterations_per_step": rg["cg_iterations_per_step"],
                           "what": "the reference's Monodomain.step (TorchCor 0.1.8: ATen and cuSPARSE kernels, "
                                   "host-synchronised CG) on this GPU, same workload, wall clock per step with a "
                                   "synchronize; matrices from the oracle's assembly"}
                del ref
                torch.cuda.empty_cache()
        else:
            r = time_oracle(wl, budget_s=budget, min_steps=3, warmup=3)
            cpu = {"value": r["value"], "unit": METRIC, "cores": r["cores"], "kind": "port",
                   "sample": f"oracle on the full workload, {r['steps']} steps after an untimed "
                             f"{r['assemble_s']:.1f} s assembly and {r['warmup']} untimed warm-up steps "
                             f"({r['seconds']:.1f} s of stepping)"}
    clk.mark(None)
    shape = tuned.get("ionic_shape") or list(_lib.ionic_variants(st.model)[max(tuned["ionic_variant"], 1) - 1])
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl.name, "nodes": wl.n_nodes, "elements": int(len(wl.elems)), "nnz": sys_.nnz,
                   "dt_ms": wl.dt, "T_ms": wl.T, "parallelism": "replicas only" if world > 1 else "single",
                   "cg_tol": 1e-5, "timed_steps": [t_first, t_first + a.steps - 1],
                   "untimed_steps_before": t_first - 1, "cg_iterations_per_step": iters / a.steps,
                   "cuda_graph_steps": G, "l2": "inputs larger than L2 (per-step working set > 300 MB)",
                   "simulated_ms_per_s": world * wl.dt * a.steps / (ms / 1e3),
                   "tuned": {"ionic_variant": int(tuned["ionic_variant"]),
                             "ionic_nodes_per_thread": int(shape[0]), "ionic_blocks_per_sm": int(shape[1]),
                             "ionic_fast_math": int(shape[2]),
                             "ionic_staged": int(shape[3]) if len(shape) > 3 else 0,
                             "cg_blocks_per_sm": int(tuned["cg_per_sm"]),
                             "fused_step": int(tuned.get("fused_step", 0)),
                             "source": "cache" if tuned.get("cached") else "measured"}},
        "gpu_launches": (1 if fused else 2) * a.steps,
        "roofline": {"bound": "hbm", "kernel": dominant[0], "achieved": dominant[1], "peak": peak,
                     "unit": "GB/s", "frac": dominant[1] / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} HBM copy bandwidth",
                     "profile_steps": [s0, s0 + a.profile_steps - 1],
                     "kernels": kernels,
                     "step": {"bytes": step_bytes, "GB/s": step_bytes / (ms / a.steps * 1e-3) / 1e9}},
        "full_run": full,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "reference_gpu": ref_gpu,
    }


def batch_arm(a, world, rank, local, clk, steps=None):
    """Batched mix (64 cubes, MS/TTP) vs the same simulations one at a time on the
    single-simulation path, and a full batched run from host arrays.  Returns the
    line (``--workload batch_cubes``) or the ``batch`` object of the default line."""
    from torchcor_b200.simulator import MonodomainBatch
    from torchcor_b200.workloads import algorithmic_bytes, batch_cubes
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    wls = batch_cubes()
    total = sum(w.n_nodes for w in wls)
    K = steps or a.steps
    stream = torch.cuda.current_stream(dev)
    batch = MonodomainBatch(dev)
    if a.cg_variant:
        batch.set_cg(a.cg_variant)
    t0 = time.perf_counter()
    for w in wls:
        batch.add(make_sim(w, dev), 1e-5, 1e-5, 100, snapshot_interval=w.T)
    batch.step(a.warmup)
    torch.cuda.synchronize(dev)
    setup_s = time.perf_counter() - t0
    batch.check()
    tuned = None
    if not a.cg_variant:
        from torchcor_b200.tune import tune_batch
        tuned = tune_batch(batch, steps=10)[1]
        torch.cuda.synchronize(dev)
    if a.batch_ionic != "auto":   # force the batched ionic form (its default budget and tiles)
        batch.set_ionic(0, 0, staged=a.batch_ionic == "staged")
    cg_cfg = batch.cg_config
    ionic_tpb, ionic_bps, ionic_staged = batch.ionic_tiles_per_block, batch.ionic_blocks_per_sm, batch.ionic_staged
    # the timed steps replay CUDA graphs of G steps, the remainder runs as plain launches
    G = a.batch_graph_steps if 0 < a.batch_graph_steps <= K else 0
    replay = batch.capture(G) if G else None
    if replay:
        replay()
    torch.cuda.synchronize(dev)
    first = batch.sims[0]._sim["next_step"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    clk.mark("batch")
    torch.cuda.nvtx.range_push("batch_timed")         # what the ncu captures in profiles/ select
    e0.record(stream)
    done = 0
    if replay:
        for _ in range(K // G):
            replay()
        done = (K // G) * G
    if K > done:
        batch.step(K - done)
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize(dev)
    clk.mark(None)
    ms = replicas.reduce_max(e0.elapsed_time(e1))     # slowest rank (each rank runs the batch)
    batch.check()
    # CG passes of the timed steps: the batch kernel runs max_i(it_i + 1) passes a
    # step; a node needs only its own simulation's it_i + 1
    its = torch.stack([s._sim["step_iters"][first:first + K].long() for s in batch.sims])
    sizes = torch.tensor([s._sim["struct"].n_nodes for s in batch.sims], device=its.device, dtype=torch.float64)
    passes_max = float((its.max(0).values + 1).double().mean().item())
    passes_node = float(((its + 1).double() * sizes[:, None]).sum().item() / (sizes.sum().item() * K))
    # algorithmic bytes of the timed steps (each simulation's B_ion + B_rhs + (it+1) B_iter)
    step_bytes = 0.0
    for k, s_ in enumerate(batch.sims):
        bi, br, bt = algorithmic_bytes(s_.system.n, s_.system.nnz, s_.ionic_model.state.shape[0])
        step_bytes += bi + br + float((its[k] + 1).double().mean().item()) * bt
    peak, peak_kind = peaks()
    value = world * total * K / (ms / 1e3)
    del batch, replay
    torch.cuda.empty_cache()
    # the plain single-simulation path on the same simulations over the same steps,
    # one after the other
    plain_ms = 0.0
    if not a.no_plain:
        for w in wls:
            sim = make_sim(w, dev)
            sim.prepare(1e-5, 1e-5, 100, snapshot_interval=w.T)
            sim.autotune()
            sim.run_steps(first - 1)
            torch.cuda.synchronize(dev)
            clk.mark("batch_plain")
            e0.record(stream)
            sim.run_steps(K)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            clk.mark(None)
            plain_ms += e0.elapsed_time(e1)
            del sim
    plain_ms = replicas.reduce_max(plain_ms)
    plain = world * total * K / (plain_ms / 1e3) if plain_ms else None
    # e2e: every simulation built from host arrays, batched, run to its end, results on the host
    e2e = None
    if not a.no_e2e:
        torch.cuda.synchronize(dev)
        clk.mark("batch_e2e")
        t0 = time.perf_counter()
        b2 = MonodomainBatch(dev)
        if a.cg_variant:
            b2.set_cg(a.cg_variant)
        sims = [b2.add(make_sim(w, dev), 1e-5, 1e-5, 100, snapshot_interval=w.T) for w in wls]
        b2.autotune()
        b2.run()
        at = [s.activation_time.cpu() for s in sims]
        torch.cuda.synchronize(dev)
        wall = replicas.reduce_max(time.perf_counter() - t0)
        clk.mark(None)
        nt = wls[0].nt
        h2d = sum(w.nodes_mm.size * 4 + w.elems.size * 4 + w.regions.size * 4 + w.fibres.size * 4 + w.n_nodes * 4
                  for w in wls)
        d2h = sum(2 * w.n_nodes * 4 + w.n_nodes * 4 for w in wls)
        e2e = {"value": world * total * nt / wall, "unit": METRIC, "h2d_bytes_per_step": int(h2d // nt),
               "d2h_bytes_per_step": int(d2h // nt), "activated_nodes": int(sum(int((x > 0).sum()) for x in at)),
               "what": f"the {len(wls)} simulations built from host arrays, batched (MonodomainBatch.run), "
                       f"every one run to T = {wls[0].T} ms ({nt} steps), AT/RT/Vm downloaded; wall {wall:.2f} s"}
        del b2, sims
        torch.cuda.empty_cache()
    out = {"metric": METRIC, "value": value, "unit": METRIC, "steps": K, "ms_per_step": ms / K,
           "timed_steps": [first, first + K - 1], "cuda_graph_steps": G,
           "config": {"workload": f"batch of {len(wls)} tet cubes (16..64 nodes per edge, h 0.25 mm), "
                                  f"Mitchell-Schaeffer/TTP ENDO 50/50, dt 0.01 ms",
                      "simulations": len(wls), "nodes": total, "cg_variant": cg_cfg[0], "cg_blocks": cg_cfg[1],
                      "ionic_tiles_per_block": ionic_tpb, "ionic_blocks_per_sm": ionic_bps,
                      "ionic_staged": ionic_staged,
                      "autotune_ms_per_step": tuned, "cg_iterations_per_step":
                          float(its.sum().item()) / K / len(wls),
                      "cg_passes_per_step": passes_max, "cg_passes_per_node_step": passes_node,
                      "setup_s": setup_s},
           "gpu_launches": 2 * K,
           "roofline": {"bound": "hbm", "kernel": "whole batch step (one ionic launch + one batched CG launch)",
                        "achieved": step_bytes / (ms / K * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": step_bytes / (ms / K * 1e-3) / 1e9 / peak, "traffic": None,
                        "peak_source": f"{peak_kind} HBM copy bandwidth", "bytes_per_step": step_bytes},
           "plain_single_path": {"value": plain, "unit": METRIC,
                                 "what": "each simulation alone through Monodomain (tuned launch shapes, same "
                                         "steps), summed device time"},
           "speedup_vs_plain": (value / plain) if plain else None,
           "e2e": e2e}
    return out


def serving_arm(a, world, rank, local, clk):
    """Request stream served on one GPU per rank (independent replicas): throughput
    and p50/p99 request latency."""
    from torchcor_b200 import serving
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    reqs = serving.generate_requests(count=a.requests, seed=2025 + rank, capacity=a.capacity, load=a.load)
    server = serving.Server(dev)
    if world > 1:
        torch.distributed.barrier()
    clk.mark("serving")
    summ = server.run(reqs)
    clk.mark(None)
    # each rank serves its own stream: whole-job rate = all ranks' node-steps / slowest wall
    total_ns = replicas.reduce_sum(summ["node_steps"])
    wall = replicas.reduce_max(summ["wall_s"])
    return {"metric": METRIC, "value": total_ns / wall, "unit": METRIC,
            "config": {"workload": f"serving: {a.requests} requests, Poisson arrivals offered at {a.load} x "
                                   f"{a.capacity:.3g} node-steps/s, N lognormal(median 50k) in [10k, 500k], "
                                   f"cube/icosphere 50/50, MS/TTP/CRN, T U(50,300) ms, dt 0.01 ms",
                       "parallelism": "replicas only"},
            "serving": summ}


def standalone_line(obj, a, world):
    """A batch or serving object as a line of its own (--workload batch_cubes|serving)."""
    line = {"metric": METRIC, "value": obj["value"], "unit": METRIC, "n_gpus": world, "steps": obj.get("steps"),
            "warmup": a.warmup, "ms_per_step": obj.get("ms_per_step"), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    line.update({k: v for k, v in obj.items() if k not in line})
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="tcb", choices=["tcb", "reference"])
    ap.add_argument("--workload", default="ttp_cube", choices=["ttp_cube", "ms_cube", "batch_cubes", "serving"])
    ap.add_argument("--requests", type=int, default=128, help="serving: requests in the stream")
    ap.add_argument("--load", type=float, default=0.9, help="serving: offered load / capacity")
    ap.add_argument("--capacity", type=float, default=4.5e9,
                    help="serving: node-steps/s the arrival rate assumes (the server's measured saturation "
                         "for this mix on a B200)")
    ap.add_argument("--graph-steps", type=int, default=100,
                    help="steps per captured CUDA graph in the timed region (0 = plain launches)")
    ap.add_argument("--batch-graph-steps", type=int, default=50)
    ap.add_argument("--batch-steps", type=int, default=200, help="timed batch steps in the default line")
    ap.add_argument("--no-plain", action="store_true", help="batch: skip the one-at-a-time comparison")
    ap.add_argument("--batch-ionic", default="auto", choices=["auto", "unstaged", "staged"],
                    help="batch: batched ionic form (auto = the tuner's choice)")
    ap.add_argument("--cg-variant", type=int, default=0, choices=[0, 1, 2, 3],
                    help="batch: batched CG variant (1/2 streaming, 3 staged); 0 = autotuned")
    ap.add_argument("--profile-steps", type=int, default=200)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-full-run", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own PyTorch step on the GPU")
    ap.add_argument("--reference-gpu-steps", type=int, default=300)
    ap.add_argument("--no-batch", action="store_true", help="default line without the batch object")
    ap.add_argument("--no-serving", action="store_true", help="default line without the serving object")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be at least 3")
    from torchcor_b200.workloads import WORKLOADS
    world, rank, local = dist_setup(a.impl)
    if a.impl == "reference":
        if a.workload in WORKLOADS:
            reference_arm(a, WORKLOADS[a.workload](), world, rank)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the single-simulation "
                              "workloads (ttp_cube, ms_cube); the reference has no batched or served path"}))
        return
    clk = ClockSampler(local)
    try:
        if a.workload == "serving":
            line = standalone_line(serving_arm(a, world, rank, local, clk), a, world)
        elif a.workload == "batch_cubes":
            line = standalone_line(batch_arm(a, world, rank, local, clk), a, world)
        else:
            line = tcb_arm(a, WORKLOADS[a.workload](), world, rank, local, clk)
            if a.workload == "ttp_cube" and not a.no_batch:
                line["batch"] = batch_arm(a, world, rank, local, clk, steps=a.batch_steps)
            if a.workload == "ttp_cube" and not a.no_serving:
                line["serving"] = serving_arm(a, world, rank, local, clk)
    finally:
        clk.stop()
    line["clocks"] = clk.summary()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
