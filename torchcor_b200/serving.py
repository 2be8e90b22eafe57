"""Serving loop: many monodomain requests arriving over time, stepped together.

A request is one simulation (mesh, ionic model, end time).  The server keeps a
``MonodomainBatch`` of the admitted requests and runs it in rounds of a few
hundred steps; between rounds it

* retires every simulation that has run all its steps (final AT/RT update,
  results copied to the host, device memory released) and records the
  request's completion time;
* admits arrived requests, oldest first, while their estimated device
  footprint fits the memory budget and the batch has room, building each one
  (mesh, conductivities, stimuli, assembly, device state) and adding it to the
  batch.

Simulations that join or leave do not disturb the others: every simulation keeps
its own step counter, tolerances and iteration count on the device, so a
request's results are those of the same simulation run alone (up to the float64
reduction order inside CG).

Latency of a request = completion time - arrival time (wall clock, including
queueing, set-up, stepping and the copy of its results to the host).

``generate_requests`` draws the serving workload: Poisson arrivals; node count
lognormal (median 50,000, sigma 0.8) clipped to [10,000, 500,000]; half cubes of
n = round(N^(1/3)) - 1 elements per edge (0.25 mm spacing, -x face stimulated
for 1 ms at intensity 100, il/it = 0.5/0.2), half icospheres of radius 25 mm of
the level whose node count is nearest N (so up to 655,362 nodes at level 8;
cap z > 24.5 mm stimulated for 2 ms at
intensity 50, seeded random tangent fibres, il/it = 0.4/0.1); ionic model uniform
over Mitchell-Schaeffer, ten Tusscher-Panfilov ENDO and Courtemanche; end time
uniform in [50, 300] ms; dt 0.01 ms.  The arrival rate is set so the offered
work is ``load`` times a stated device capacity in node-steps/s.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from torchcor_b200 import meshgen

MODELS = ("ms", "ttp", "crn")
ICO_LEVEL_NODES = {lv: 10 * 4 ** lv + 2 for lv in range(3, 9)}


@dataclass
class Request:
    rid: int
    arrival_s: float
    mesh: str           # "cube" | "ico"
    size: int           # cube: elements per edge; ico: subdivision level
    model: str          # "ms" | "ttp" | "crn"
    T: float
    dt: float = 0.01
    seed: int = 0
    a_tol: float = 1e-5
    r_tol: float = 1e-5
    max_iter: int = 100
    # filled in by the server
    admitted_s: float = None
    done_s: float = None
    n_total_iter: int = None
    result: dict = field(default=None, repr=False)

    @property
    def n_nodes(self):
        return (self.size + 1) ** 3 if self.mesh == "cube" else ICO_LEVEL_NODES[self.size]

    @property
    def nt(self):
        return int(self.T / self.dt)

    @property
    def latency_s(self):
        return None if self.done_s is None else self.done_s - self.arrival_s


def generate_requests(count=512, seed=2025, median=50_000, sigma=0.8, lo=10_000, hi=500_000,
                      capacity=5e9, load=0.9, T_range=(50.0, 300.0), dt=0.01):
    """The seeded request stream described in the module docstring."""
    rng = np.random.default_rng(seed)
    N = np.clip(rng.lognormal(math.log(median), sigma, size=count), lo, hi)
    kinds = rng.integers(0, 2, size=count)
    models = rng.integers(0, 3, size=count)
    Ts = rng.uniform(T_range[0], T_range[1], size=count)
    reqs = []
    for k in range(count):
        if kinds[k] == 0:
            mesh, size = "cube", max(2, int(round(N[k] ** (1.0 / 3.0))) - 1)
        else:
            mesh = "ico"
            size = min(ICO_LEVEL_NODES, key=lambda lv: abs(ICO_LEVEL_NODES[lv] - N[k]))
        reqs.append(Request(k, 0.0, mesh, size, MODELS[models[k]], float(Ts[k]), dt, seed=seed * 1000 + k))
    work = np.array([r.n_nodes * r.nt for r in reqs], dtype=np.float64)
    rate = load * capacity / work.mean()                  # requests per second
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.cumsum(gaps) - gaps[0]
    for r, a in zip(reqs, t):
        r.arrival_s = float(a)
    return reqs


def build_sim(req: Request, device, reorder=None):
    """The ``Monodomain`` of a request (mesh, conductivities, stimuli; not yet assembled).
    Icosphere nodes are renumbered by reverse Cuthill-McKee unless ``reorder=False``
    (their subdivision numbering scatters neighbours across the whole index range);
    the structured cubes keep their numbering."""
    from torchcor_b200.ionic import CourtemancheRamirezNattel, ModifiedMS2v, TenTusscherPanfilov
    from torchcor_b200.simulator import Monodomain
    if req.model == "ttp":
        im = TenTusscherPanfilov("ENDO", req.dt, device=device)
    elif req.model == "crn":
        im = CourtemancheRamirezNattel(req.dt, device=device)
    else:
        im = ModifiedMS2v(req.dt, device=device)
    if reorder is None:
        reorder = req.mesh == "ico"
    sim = Monodomain(im, T=req.T, dt=req.dt, device=device, reorder=reorder)
    if req.mesh == "cube":
        nodes_um, elems = meshgen.cube(req.size, 0.25)
        fib = meshgen.fibres_constant(len(elems))
        sim.load_arrays(nodes_um / 1000.0, elems, np.ones(len(elems), dtype=np.int64), fib)
        sim.add_conductivity([1], il=0.5, it=0.2)
        sim.add_stimulus(None, 0.0, 1.0, 100, region=meshgen.cube_face(req.size, 0, 0))
    else:
        nodes_um, tris = meshgen.icosphere_fast(req.size, 25.0)
        fib = meshgen.fibres_random_tangent(nodes_um, tris, req.seed)
        sim.load_arrays(nodes_um / 1000.0, tris, np.ones(len(tris), dtype=np.int64), fib)
        sim.add_conductivity([1], il=0.4, it=0.1)
        sim.add_stimulus(None, 0.0, 2.0, 50, region=np.nonzero(nodes_um[:, 2] > 24_500.0)[0])
    return sim


# lookup-table bytes per model (float32 tables, padded rows)
_TABLE_BYTES = {"ms": 0, "ttp": 17 << 20, "crn": 4 << 20}
_STATES = {"ms": 1, "ttp": 19, "crn": 19}


def footprint_bytes(req: Request) -> int:
    """Device bytes a request holds while it runs, with a 10 % margin: the CSR copy
    (int32 columns, float32 M, K/chi, A, K' - 20 B per non-zero) and the sliced-ELL
    solver copy (int32 and int16 columns, float32 M, K', A - 18 B per stored entry,
    slices padded to their widest row), 13 per-node vectors (solution ring, CG
    vectors, 1/diag, AT/RT, stimulus bits) and the ionic state, the mesh arrays the
    simulation keeps (coordinates, elements, regions, fibres), the per-step
    schedule and the lookup tables.  Checked against the memory a built request
    holds by the GPU tests."""
    n = req.n_nodes
    if req.mesh == "cube":
        n_elems, k, nnz_row = 6 * req.size ** 3, 4, 15
    else:
        n_elems, k, nnz_row = 20 * 4 ** req.size, 3, 7
    nnz = n * nnz_row
    matrices = 20 * nnz + 4 * (n + 1) + 18 * nnz * 1.1
    vectors = n * (13 * 4 + 4 * _STATES[req.model])
    mesh = 12 * n + (4 * k + 16) * n_elems
    return int(1.1 * (matrices + vectors + mesh) + 12 * (req.nt + 1) + _TABLE_BYTES[req.model])


class Server:
    """Runs a request stream on one GPU (see the module docstring)."""

    def __init__(self, device=None, memory_budget=None, max_sims=256, round_steps=200, autotune=True):
        from torchcor_b200.simulator import MonodomainBatch
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget = int(0.8 * free)
        self.memory_budget = memory_budget
        self.round_steps = round_steps
        self.batch = MonodomainBatch(self.device, max_sims)
        self.autotune = autotune
        self.in_use = 0
        self.active = {}      # id(sim) -> (request, bytes)
        self.node_steps = 0
        self.busy_s = 0.0

    def _build(self, req, now_fn):
        """Mesh, assembly and device state of a request (on the current stream)."""
        req.admitted_s = now_fn()
        sim = build_sim(req, self.device)
        sim.prepare(req.a_tol, req.r_tol, req.max_iter, snapshot_interval=req.T)
        return sim

    def _join(self, req, sim):
        self.batch.add(sim, req.a_tol, req.r_tol, req.max_iter, snapshot_interval=req.T)
        self.active[id(sim)] = (req, footprint_bytes(req))

    def _retire(self, sim, now_fn):
        req, nbytes = self.active.pop(id(sim))
        self.batch.remove(sim)
        req.result = {"AT": sim.activation_time.cpu(), "RT": sim.repolarization_time.cpu(),
                      "Vm": sim.current_solution().cpu()}
        req.n_total_iter = sim.n_total_iter
        req.done_s = now_fn()
        self.in_use -= nbytes
        self.node_steps += req.n_nodes * req.nt
        sim._sim = None

    def _fits(self, req):
        return (len(self.active) + self._staged < self.batch.max_sims and
                (not self.active and not self._staged or self.in_use + footprint_bytes(req) <= self.memory_budget))

    def run(self, requests, realtime=True):
        """Serve ``requests`` until all are done; returns the summary dict.  With
        ``realtime=False`` every request counts as arrived at time 0.

        Each round launches up to ``round_steps`` batch steps (ending when the
        first active simulation finishes), builds the requests that arrived
        meanwhile on a side stream while the round runs, then retires finished
        simulations and adds the new ones."""
        reqs = sorted(requests, key=lambda r: r.arrival_s)
        if not realtime:
            for r in reqs:
                r.arrival_s = 0.0
        pending = deque(reqs)
        main = torch.cuda.current_stream(self.device)
        side = torch.cuda.Stream(self.device)
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0   # noqa: E731
        tuned_key = None      # shape of the batch the launch was last chosen for
        self._staged = 0
        # where the loop's time goes: host seconds building, waiting for the round,
        # retiring and joining; device seconds of the batch steps (CUDA events)
        spent = {"build_s": 0.0, "wait_s": 0.0, "retire_s": 0.0, "join_s": 0.0}
        step_events = []
        while pending or self.active:
            if not self.active:
                if pending[0].arrival_s > now():
                    time.sleep(max(0.0, min(0.05, pending[0].arrival_s - now())))
                    continue
                req = pending.popleft()
                self.in_use += footprint_bytes(req)
                self._join(req, self._build(req, now))
                continue
            if self.autotune and len(self.active) >= 2:
                # the batch's shape (node and simulation counts in log2 buckets, model
                # set) changes as requests join and leave: choose its launch again
                # (from the cache when this shape was seen before; the timed steps
                # are real steps of the batch)
                from torchcor_b200.tune import batch_key
                key = batch_key(self.device, [s._sim["struct"].n_nodes for s in self.batch.sims],
                                [s.ionic_model.name for s in self.batch.sims])
                if key != tuned_key:
                    self.batch.autotune(steps=5)
                    tuned_key = key
            k = min(self.round_steps, min(s.nt + 1 - s._sim["next_step"] for s in self.batch.sims))
            t1 = time.perf_counter()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(main)
            self.batch.step(max(1, k))
            e1.record(main)
            step_events.append((e0, e1))
            # build arrived requests on the side stream while the round runs (a
            # builder thread was measured slower: its kernels and its hold on the
            # interpreter slowed the batch steps more than the overlap gained)
            staged = []
            tb = time.perf_counter()
            with torch.cuda.stream(side):
                while pending and pending[0].arrival_s <= now() and self._fits(pending[0]):
                    req = pending.popleft()
                    self.in_use += footprint_bytes(req)
                    self._staged += 1
                    staged.append((req, self._build(req, now)))
            tw = time.perf_counter()
            side.synchronize()
            main.synchronize()
            tr = time.perf_counter()
            self.busy_s += tr - t1
            spent["build_s"] += tw - tb
            spent["wait_s"] += tr - tw
            self.batch.check()
            for s in self.batch.finished():
                self._retire(s, now)
            tj = time.perf_counter()
            for req, sim in staged:
                self._join(req, sim)
            self._staged = 0
            spent["retire_s"] += tj - tr
            spent["join_s"] += time.perf_counter() - tj
        wall = now()
        torch.cuda.synchronize(self.device)
        spent["steps_device_s"] = sum(a.elapsed_time(b) for a, b in step_events) / 1e3
        spent["rounds"] = len(step_events)
        lat = np.array([r.latency_s for r in reqs])
        sim_ms = sum(r.T for r in reqs)
        return {"requests": len(reqs), "wall_s": wall, "node_steps": self.node_steps,
                "node_steps_per_s": self.node_steps / wall, "simulated_ms_per_s": sim_ms / wall,
                "requests_per_s": len(reqs) / wall,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "latency_mean_s": float(lat.mean()), "gpu_busy_frac": self.busy_s / wall,
                "steps_device_frac": spent["steps_device_s"] / wall, "loop": spent}
