"""``Monodomain`` with the interface of ``torchcor/simulator/monodomain.py:18-226``.

The time loop runs on the device: per step one ionic kernel (activation and
repolarisation update of the previous step, snapshot, ionic model, stimulus,
right-hand side) and one persistent cooperative kernel (mass/stiffness
products, extrapolated guess, Jacobi-PCG with the stopping test on the
device).  The host only launches; the step index, CG iteration counts and the
membrane-potential ring live in device memory, so a solve needs no host
synchronisation until it finishes.
"""
from __future__ import annotations

import ctypes as C
import time
from pathlib import Path

import numpy as np
import torch

from torchcor_b200 import _lib
from torchcor_b200._lib import check, ptr, stream_ptr
from torchcor_b200.core.assemble import assemble_phie, assemble_system
from torchcor_b200.core.conductivity import Conductivity
from torchcor_b200.core.mesh import MeshReader
from torchcor_b200.core.stimulation import Stimuli
from torchcor_b200.device import get_device
from torchcor_b200.simulator.resultio import FrameWriter


def rcm_order(elems, n_nodes):
    """Reverse Cuthill-McKee order (internal index -> node id) of the node graph
    whose edges join the nodes of each element."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    el = np.asarray(elems, dtype=np.int64)
    k = el.shape[1]
    rows = np.concatenate([el[:, i] for i in range(k) for j in range(k) if i != j])
    cols = np.concatenate([el[:, j] for i in range(k) for j in range(k) if i != j])
    g = sp.csr_matrix((np.ones(len(rows), dtype=np.int8), (rows, cols)), shape=(n_nodes, n_nodes))
    return np.asarray(reverse_cuthill_mckee(g, symmetric_mode=True), dtype=np.int64)


class Monodomain:
    def __init__(self, ionic_model, T, dt, device=None, dtype=None, reorder=False):
        self.device = torch.device(device) if device is not None else get_device()
        if self.device.type != "cuda":
            raise RuntimeError("torchcor_b200.Monodomain needs a CUDA device (no CPU fallback)")
        if dtype not in (None, torch.float32):
            raise NotImplementedError("torchcor_b200 runs the monodomain step in float32 "
                                      "(float64 inner products inside CG)")
        self.dtype = torch.float32
        self.T = T
        self.dt = dt
        self.nt = int(T / dt)                                  # monodomain.py:25
        self.ionic_model = ionic_model
        if getattr(ionic_model, "dt", None) is None:
            ionic_model.dt = dt
        self.Chi, self.Cm, self.theta = 140, 0.01, 0.5          # :44-46
        self.n_nodes = None
        self.nodes = self.elems = self.regions = self.fibres = None
        self.stimuli = None
        self.conductivity = None
        self.system = None
        self.K = self.M = self.A = None
        self.mesh_path = None
        self.result_path = None
        self._sim = None
        # reorder=True: nodes are renumbered by reverse Cuthill-McKee for memory
        # locality (torchcor/core/reorder.py:7-48 offers the same ordering); every
        # per-node input and output of this class stays in the caller's numbering,
        # only the exported M/K/A are in the internal one (node_order maps it)
        self.reorder = bool(reorder)
        self.node_order = None          # internal index -> caller's node id
        self._perm_t = self._inv_t = None

    # ------------------------------------------------------------------ input
    def load_mesh(self, path="Data/ventricle/Case_1", unit_conversion=1000, device_ingest=True):
        """Read the openCARP mesh in ``path`` (monodomain.py:60-73).  With
        ``device_ingest`` (default) the files are parsed and the CSR pattern is built
        on the GPU (same arrays as the host reader and pattern builder); files the
        device parser cannot read exactly go through the host reader, listed in
        ``self.ingest_host_files``."""
        self.mesh_path = Path(path)
        if device_ingest and not self.reorder:
            from torchcor_b200.core.ingest import read_mesh_device
            nodes, elems, regions, fibres, on_host = read_mesh_device(path, self.device, unit_conversion)
            self.ingest_host_files = on_host
            self.load_device_arrays(nodes, elems, regions, fibres)
            return
        nodes, elems, regions, fibres = MeshReader(path).read(unit_conversion=unit_conversion)
        self.ingest_host_files = None
        self.load_arrays(nodes, elems, regions, fibres)

    def load_device_arrays(self, nodes, elems, regions, fibres):
        """Mesh already on the device (tensors): nodes (N,3) in mm, elems (E,3|4),
        per-element regions and fibres.  The pattern of the assembly is then built
        on the device too."""
        dev = self.device
        self.n_nodes = int(nodes.shape[0])
        self.nodes = nodes.to(device=dev, dtype=torch.float32).contiguous()
        self.elems = elems.to(device=dev, dtype=torch.int32).contiguous()
        self._elems_np = self.elems                    # device elements: device pattern build
        self.regions = regions.to(device=dev, dtype=torch.int).contiguous()
        self.fibres = fibres.to(device=dev, dtype=torch.float32).contiguous()
        self.stimuli = Stimuli(self.n_nodes, dev, self.dtype)
        self.conductivity = Conductivity(self.regions, dtype=self.dtype)

    def load_arrays(self, nodes, elems, regions, fibres):
        """Mesh already in memory: nodes (N,3) in mm, elems (E,3|4), per-element regions and fibres."""
        self.n_nodes = int(nodes.shape[0])
        if self.reorder:
            elems = np.ascontiguousarray(elems, dtype=np.int32)
            perm = rcm_order(elems, self.n_nodes)
            inv = np.empty_like(perm)
            inv[perm] = np.arange(self.n_nodes, dtype=perm.dtype)
            nodes = np.asarray(nodes)[perm]
            elems = inv[elems].astype(np.int32)
            self.node_order = perm
            self._perm_t = torch.from_numpy(perm).to(self.device)
            self._inv_t = torch.from_numpy(inv).to(self.device)
        self.nodes = self._upload(nodes, torch.float32)
        self.elems = self._upload(elems, torch.int32)
        # the assembly pattern is built where the elements are (the device build on a GPU)
        self._elems_np = self.elems if self.elems.is_cuda else self.elems.numpy()
        self.regions = self._upload(regions, torch.int)
        self.fibres = self._upload(fibres, torch.float32)
        self.stimuli = Stimuli(self.n_nodes, self.device, self.dtype)
        self.conductivity = Conductivity(self.regions, dtype=self.dtype)

    def _upload(self, a, dtype):
        """Host array -> contiguous tensor of ``dtype`` on the device: the caller's
        bytes are copied as they are and converted there (a mesh reader's int64
        elements and float64 fibres would otherwise be converted on one host core)."""
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.to(self.device).to(dtype).contiguous()

    def _to_caller(self, t):
        """Per-node tensor (last axis) from the internal numbering to the caller's."""
        if t is None or self._inv_t is None:
            return t
        return t[..., self._inv_t if t.device == self._inv_t.device else self._inv_t.cpu()]

    def _to_internal(self, t):
        return t if t is None or self._perm_t is None else t[..., self._perm_t]

    def add_stimulus(self, vtx_filepath, start, duration, intensity, period=None, count=1, region=None):
        if period is None:
            period = self.T
        self.stimuli.add(vtx_filepath, start, duration, intensity, period, count, region=region)

    def add_conductivity(self, region_ids, il, it, el=None, et=None):
        self.conductivity.add(region_ids, il, it, el, et)

    # --------------------------------------------------------------- assembly
    def assemble(self):
        c = self.conductivity
        self.system = assemble_system(self.nodes, self._elems_np, c.sigma_l.contiguous(), c.sigma_t.contiguous(),
                                      self.fibres.contiguous(), self.dt, self.Chi, self.Cm, self.theta)
        s = self.system
        self.M = s.csr(s.m_val)
        self.K = s.csr(s.k_val)
        self.A = s.csr(s.a_val)
        return s

    # -------------------------------------------------------------- time loop
    def _setup(self, a_tol, r_tol, max_iter, calculate_AT_RT, linear_guess, snapshot_interval, keep_snapshots,
               snapshot_ring=0):
        s = self.system
        dev = self.device
        im = self.ionic_model
        u0 = im.initialize(self.n_nodes)
        n, n_pad, nt = s.n, s.n_pad, self.nt
        f32 = dict(device=dev, dtype=torch.float32)
        x = torch.zeros((3, n_pad), **f32)
        x[0, :n] = u0
        x[2, :n] = u0                                          # x_prev = x at initialise (solver.py:26)
        per_frame = int(snapshot_interval / self.dt)           # :150
        if per_frame == 0:
            raise ZeroDivisionError("snapshot_interval is shorter than dt")
        n_snap = nt // per_frame + 1
        ring = int(snapshot_ring) if keep_snapshots and snapshot_ring else 0
        snaps = torch.empty((ring if ring else n_snap, n), **f32) if keep_snapshots else None
        host_snaps = None
        if ring:
            # frames stream to pinned host memory; frame 0 is the initial state
            host_snaps = torch.empty((n_snap, n), dtype=torch.float32, pin_memory=True)
            host_snaps[0].copy_(u0)
        elif snaps is not None:
            snaps[0] = u0
        t32, mask = self.stimuli.schedule(nt, self.dt)
        # per-node arrays are n_pad long (the ionic kernels may read groups of nodes as
        # one vector access); AT/RT are exposed as their first n entries
        at_rt = torch.full((2, n_pad), -1.0, **f32)
        bits = np.zeros(n_pad, dtype=np.uint32)
        bits[:n] = self._stim_bits()
        sim = dict(
            x=x, bp=torch.zeros(n_pad, **f32), r=torch.zeros(n_pad, **f32), p=torch.zeros(n_pad, **f32),
            ap=torch.zeros(n_pad, **f32), z=torch.zeros(n_pad, **f32), p2=torch.zeros(n_pad, **f32),
            at_rt=at_rt, at=at_rt[0, :n], rt=at_rt[1, :n],
            snaps=snaps, u0=u0, ring=ring, host_snaps=host_snaps,
            stim_bits=torch.from_numpy(bits.view(np.int32)).to(dev),
            step_t=torch.from_numpy(t32).to(dev), step_stim=torch.from_numpy(mask.view(np.int32)).to(dev),
            step_iters=torch.zeros(nt + 1, device=dev, dtype=torch.int32),
            counter=torch.tensor([1, 0, 0, 0], device=dev, dtype=torch.int32),
            scratch=torch.zeros(int(_lib.load().tcb_mono_scratch_doubles()), device=dev, dtype=torch.float64),
            barrier=torch.zeros(4, device=dev, dtype=torch.int32),
            params=im.param_array(), per_frame=per_frame, next_step=1,
        )
        m = _lib.tcb_mono()
        m.n_nodes, m.n_pad, m.n_slices, m.nt = n, n_pad, s.n_slices, nt
        m.model, m.n_states = im.model_id, im.state.shape[0]
        m.slice_ptr, m.col, m.col_delta = ptr(s.slice_ptr), ptr(s.sell_col), ptr(s.sell_dcol)
        m.m_val, m.k_val, m.a_val, m.d_inv = ptr(s.sell_m), ptr(s.sell_k), ptr(s.sell_a), ptr(s.d_inv)
        m.state, m.tables = ptr(im.state), ptr(im.tables)
        m.x, m.bprime, m.r, m.p, m.ap, m.z, m.p2 = (ptr(sim[k]) for k in ("x", "bp", "r", "p", "ap", "z", "p2"))
        m.at, m.rt, m.snapshots = ptr(sim["at"]), ptr(sim["rt"]), ptr(snaps)
        m.stim_bits, m.step_t, m.step_stim = ptr(sim["stim_bits"]), ptr(sim["step_t"]), ptr(sim["step_stim"])
        amp = self.stimuli.amplitudes()
        for k in range(_lib.TCB_MAX_STIMULI):
            m.stim_amp[k] = float(amp[k])
        m.a_tol, m.r_tol, m.max_iter = float(a_tol), float(r_tol), int(max_iter)
        m.linear_guess, m.at_rt, m.per_frame = int(bool(linear_guess)), int(bool(calculate_AT_RT)), per_frame
        m.cm, m.dt = float(self.Cm), float(self.dt)
        m.snap_ring = ring
        m.a_split = int(s.a_split)
        m.step_iters, m.counter = ptr(sim["step_iters"]), ptr(sim["counter"])
        m.scratch, m.barrier = ptr(sim["scratch"]), ptr(sim["barrier"])
        m.params = sim["params"].ctypes.data
        m.node_params = ptr(im.node_params)
        sim["struct"] = m
        self._sim = sim
        return sim

    def _sync_node_params(self):
        """Point the device view at the model's per-node parameters once a caller has
        set them node by node (e.g. TTP conductances after initialize(), as the
        reference allows between steps)."""
        rows = self.ionic_model.node_params
        m = self._sim["struct"]
        want = ptr(rows) if rows is not None else None
        if (m.node_params or None) != want:
            m.node_params = want

    def run_steps(self, n_steps, stream=None):
        """Advance the prepared simulation by ``n_steps`` steps (asynchronous)."""
        self._sync_node_params()
        sim = self._sim
        a = sim["next_step"]
        b = min(a + n_steps, self.nt + 1)
        if b > a:
            check(_lib.load().tcb_mono_run(C.byref(sim["struct"]), a, b, stream_ptr(stream)))
        sim["next_step"] = b
        return b - a

    def _advance(self, n, graph_steps):
        """Run ``n`` steps: whole ``graph_steps``-step stretches replay one CUDA graph
        (recorded on first use, after a plain launch has configured the kernels), the
        rest run as plain launches."""
        sim = self._sim
        G = int(graph_steps or 0)
        if G > 1 and n >= G:
            rep = sim.get("graph")
            if rep is None or rep.n_steps != G:
                n -= self.run_steps(1)
                rep = sim["graph"] = self.capture_steps(G)
            while n >= G:
                rep()
                n -= G
        self.run_steps(n)

    def capture_steps(self, n_steps):
        """Record ``n_steps`` steps of the prepared simulation in a CUDA graph;
        returns a callable replaying them (with the step bookkeeping)."""
        self._sync_node_params()
        sim = self._sim
        lib = _lib.load()
        # the first launch on a device configures kernel attributes: keep it outside capture
        graph = torch.cuda.CUDAGraph()
        # thread-local capture: a thread writing result files may use CUDA meanwhile
        with torch.cuda.graph(graph, capture_error_mode="thread_local"):
            check(lib.tcb_mono_run(C.byref(sim["struct"]), 1, 1 + n_steps, stream_ptr()))

        def replay():
            if sim["next_step"] + n_steps > self.nt + 1:
                raise RuntimeError("not enough steps left for a full replay")
            graph.replay()
            sim["next_step"] += n_steps
        replay.graph = graph
        replay.n_steps = n_steps
        return replay

    def _stim_bits(self):
        bits = self.stimuli.membership_bits()          # caller's numbering
        return bits if self.node_order is None else np.ascontiguousarray(bits[self.node_order])

    def current_solution(self):
        """Membrane potential after the last step run (caller's node numbering)."""
        sim = self._sim
        return self._to_caller(sim["x"][(sim["next_step"] + 2) % 3, : self.n_nodes])

    def step(self, u, t, a_tol, r_tol, max_iter, verbose=False):
        """One step of the prepared simulation (monodomain.py:109-139).  ``u`` must be
        the previous solution and ``t`` the time of this step; returns
        (u, n_iter, ionic_time, electric_time)."""
        if self._sim is None:
            if self.system is None:
                self.assemble()
            self._setup(a_tol, r_tol, max_iter, True, True, 1, False)
        sim = self._sim
        n = sim["next_step"]
        if n > self.nt:
            raise RuntimeError("all time steps of this simulation have been run")
        sim["x"][(n + 2) % 3, : self.n_nodes] = self._to_internal(torch.as_tensor(u, device=self.device))
        sim["step_t"][n] = float(t)
        m = 0
        for k, s in enumerate(self.stimuli.stimulus_list):
            if self.stimuli.is_active(s, t):
                m |= 1 << k
        sim["step_stim"][n] = np.int32(np.uint32(m).view(np.int32))
        st = sim["struct"]
        st.a_tol, st.r_tol, st.max_iter = float(a_tol), float(r_tol), int(max_iter)
        t0 = time.time()
        self.run_steps(1)
        check(_lib.load().tcb_mono_check(C.byref(st), stream_ptr()))
        el = time.time() - t0
        return self.current_solution().clone(), int(sim["step_iters"][n].item()), 0.0, el

    # -------------------------------------------------- streamed snapshot output
    def _snapshot_stream_init(self):
        sim = self._sim
        sim["copy_stream"] = torch.cuda.Stream(self.device)
        sim["copied"] = [None] * sim["ring"]     # event per ring row: its last copy to the host is done
        sim["next_frame"] = 1                    # next frame to copy out (frame 0 is the initial state)

    def _frames_written(self):
        """Frames whose snapshot rows the steps launched so far have written (the
        ionic kernel of step f*per_frame + 1 writes frame f)."""
        sim = self._sim
        return (sim["next_step"] - 2) // sim["per_frame"] if sim["next_step"] >= 2 else 0

    def _before_steps(self, first_step, n_steps):
        """Make the compute stream wait until the ring rows that steps
        [first_step, first_step + n_steps) will overwrite have been copied out."""
        sim = self._sim
        pf, R = sim["per_frame"], sim["ring"]
        cur = torch.cuda.current_stream(self.device)
        f0 = max(1, (first_step - 1 + pf - 1) // pf)
        f1 = (first_step + n_steps - 2) // pf
        for f in range(max(f0, f1 - R + 1), f1 + 1):
            ev = sim["copied"][f % R]
            if ev is not None:
                cur.wait_event(ev)

    def _drain_snapshots(self, final=False):
        """Queue the copies of every frame written so far (on the copy stream, after
        the compute stream's work); with ``final`` also the last step's frame, which
        the finish kernel writes, and wait for all copies."""
        sim = self._sim
        pf, R = sim["per_frame"], sim["ring"]
        last = self.nt // pf if final else self._frames_written()
        if sim["next_frame"] > last:
            if final:
                sim["copy_stream"].synchronize()
            return
        cur = torch.cuda.current_stream(self.device)
        done = torch.cuda.Event()
        done.record(cur)
        cs = sim["copy_stream"]
        cs.wait_event(done)
        with torch.cuda.stream(cs):
            for f in range(sim["next_frame"], last + 1):
                sim["host_snaps"][f].copy_(sim["snaps"][f % R], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cs)
                sim["copied"][f % R] = ev
        sim["next_frame"] = last + 1
        if final:
            cs.synchronize()

    def finish(self, result_path=None, calculate_AT_RT=True):
        """AT/RT update and snapshot of the last step, error check, result files
        (the tail of monodomain.py:141-226).  Returns the total CG iterations."""
        sim = self._sim
        st = sim["struct"]
        lib = _lib.load()
        if sim.get("ring") and self.nt % sim["per_frame"] == 0:
            self._drain_snapshots()
            ev = sim["copied"][(self.nt // sim["per_frame"]) % sim["ring"]]
            if ev is not None:
                torch.cuda.current_stream(self.device).wait_event(ev)
        check(lib.tcb_mono_finish(C.byref(st), stream_ptr()))
        writer = sim.pop("vm_writer", None)
        if writer is not None:
            done = torch.cuda.Event()
            done.record(torch.cuda.current_stream(self.device))
            try:
                check(lib.tcb_mono_check(C.byref(st), stream_ptr()))
            except BaseException:
                writer.abort()
                raise
            writer.finish(done)       # Vm.pt is complete
        else:
            check(lib.tcb_mono_check(C.byref(st), stream_ptr()))
        self.n_total_iter = int(sim["step_iters"].sum().item())
        self.activation_time = self._to_caller(sim["at"])
        self.repolarization_time = self._to_caller(sim["rt"])
        if sim.get("ring"):
            self._drain_snapshots(final=True)
            self.solutions = self._to_caller(sim["host_snaps"])
        else:
            self.solutions = self._to_caller(sim["snaps"])
        if result_path is not None:
            rp = Path(result_path)
            rp.mkdir(parents=True, exist_ok=True)
            if calculate_AT_RT:
                torch.save(self.activation_time.cpu(), rp / "ATs.pt")
                torch.save(self.repolarization_time.cpu(), rp / "RTs.pt")
            if self.solutions is not None and writer is None:
                torch.save(self.solutions.cpu(), rp / "Vm.pt")
        return self.n_total_iter

    def phie_recovery(self, a_tol=1e-5, r_tol=1e-5, max_iter=100, Vm=None, verbose=False):
        """Extracellular potential of every Vm frame (monodomain.py:254-286):
        K(sigma_i + sigma_e) phi_e = -K(sigma_i) Vm, Jacobi-PCG with the linear
        extrapolation guess from the previous frames' solutions, then phi_e minus its
        mean.  ``Vm`` defaults to the snapshots of the last solve, else
        ``result_path/Vm.pt``; the result is returned, kept as ``self.phi_e`` and saved
        as ``result_path/Phi_e.pt`` when the solve had a result path.  Needs
        intracellular and extracellular conductivities (``add_conductivity(..., el, et)``).
        The solves run on the device (``tcb_mono_cg_run``); printing per frame, as the
        reference does, only with ``verbose=True``."""
        c = self.conductivity
        if c.sigma_il is None or c.sigma_el is None:
            raise ValueError("phie_recovery needs intracellular and extracellular conductivities "
                             "(add_conductivity(..., el=..., et=...))")
        if Vm is None:
            if getattr(self, "solutions", None) is not None:
                Vm = self.solutions
            elif self.result_path is not None and (self.result_path / "Vm.pt").exists():
                Vm = torch.load(self.result_path / "Vm.pt")
            else:
                raise ValueError("no Vm frames: solve with snapshot_interval < T first, or pass Vm")
        dev = self.device
        Vm = self._to_internal(Vm.to(device=dev, dtype=torch.float32)).contiguous()
        F, n = Vm.shape
        s = assemble_phie(self.nodes, self._elems_np, c.sigma_il.contiguous(), c.sigma_it.contiguous(),
                          c.sigma_el.contiguous(), c.sigma_et.contiguous(), self.fibres.contiguous())
        f32 = dict(device=dev, dtype=torch.float32)
        n_pad = s.n_pad
        buf = dict(x=torch.zeros((3, n_pad), **f32), bp=torch.zeros(n_pad, **f32), r=torch.zeros(n_pad, **f32),
                   p=torch.zeros(n_pad, **f32), ap=torch.zeros(n_pad, **f32), z=torch.zeros(n_pad, **f32),
                   p2=torch.zeros(n_pad, **f32), placeholder=torch.zeros(n_pad, **f32),
                   flags=torch.zeros(F + 2, device=dev, dtype=torch.int32),
                   step_t=torch.zeros(F + 2, **f32),
                   step_iters=torch.zeros(F + 1, device=dev, dtype=torch.int32),
                   counter=torch.tensor([1, 0, 0, 0], device=dev, dtype=torch.int32),
                   scratch=torch.zeros(int(_lib.load().tcb_mono_scratch_doubles()), device=dev,
                                       dtype=torch.float64),
                   barrier=torch.zeros(4, device=dev, dtype=torch.int32),
                   params=np.zeros(16, dtype=np.float64))
        m = _lib.tcb_mono()
        m.n_nodes, m.n_pad, m.n_slices, m.nt = n, n_pad, s.n_slices, F
        m.model, m.n_states = _lib.MODEL_MS, 1          # the ionic fields are placeholders: no ionic kernel runs
        m.slice_ptr, m.col, m.col_delta = ptr(s.slice_ptr), ptr(s.sell_col), ptr(s.sell_dcol)
        m.m_val, m.k_val, m.a_val, m.d_inv = ptr(s.sell_m), ptr(s.sell_k), ptr(s.sell_a), ptr(s.d_inv)
        m.state, m.tables = ptr(buf["placeholder"]), None
        m.x, m.bprime, m.r, m.p, m.ap, m.z, m.p2 = (ptr(buf[k]) for k in ("x", "bp", "r", "p", "ap", "z", "p2"))
        m.at = m.rt = ptr(buf["placeholder"])
        m.snapshots = None
        m.stim_bits, m.step_t, m.step_stim = ptr(buf["flags"]), ptr(buf["step_t"]), ptr(buf["flags"])
        m.a_tol, m.r_tol, m.max_iter = float(a_tol), float(r_tol), int(max_iter)
        m.linear_guess, m.at_rt, m.per_frame = 1, 0, 0
        m.cm, m.dt = 0.0, 1.0
        m.a_split = 0
        m.step_iters, m.counter = ptr(buf["step_iters"]), ptr(buf["counter"])
        m.scratch, m.barrier = ptr(buf["scratch"]), ptr(buf["barrier"])
        m.params = buf["params"].ctypes.data
        lib = _lib.load()
        out = torch.empty((F, n), **f32)
        for k in range(F):
            buf["bp"][:n] = -Vm[k]                       # b' := -Vm so that M b' = -K(sigma_i) Vm
            check(lib.tcb_mono_cg_run(C.byref(m), k + 1, k + 2, stream_ptr()))
            phi = out[k]
            phi.copy_(buf["x"][(k + 1) % 3, :n])         # the step's solution slot of the ring
            phi -= phi.mean()
            if verbose:
                print(phi.min().item(), phi.max().item(), int(buf["step_iters"][k + 1].item()), flush=True)
        check(lib.tcb_mono_check(C.byref(m), stream_ptr()))
        out = self._to_caller(out)
        self.phi_e = out
        self.phie_iters = buf["step_iters"][1:].cpu()
        if self.result_path is not None:
            torch.save(out.cpu(), self.result_path / "Phi_e.pt")
        return out

    def prepare(self, a_tol, r_tol, max_iter, calculate_AT_RT=True, linear_guess=True, snapshot_interval=1):
        """Assemble and set up the device state of a solve without running it
        (what ``solve`` does before its loop); used by ``MonodomainBatch``."""
        self.assemble()
        return self._setup(a_tol, r_tol, max_iter, calculate_AT_RT, linear_guess, snapshot_interval,
                           snapshot_interval < self.T)

    def set_launch(self, ionic_variant=None, cg_per_sm=None, fused_step=None):
        """Set the prepared simulation's launch shapes: ionic kernel instance (1..,
        0 = default), CG blocks per SM (0, 1, 2), fused step (0 or 1)."""
        m = self._sim["struct"]
        if ionic_variant is not None:
            m.ionic_variant = int(ionic_variant)
        if cg_per_sm is not None:
            m.cg_per_sm = int(cg_per_sm)
        if fused_step is not None:
            m.fused_step = int(fused_step)

    def autotune(self, steps=5, force=False):
        """Choose the launch shapes of the prepared simulation's kernels (ionic
        kernel instance, CG blocks per SM): the cached choice for this device and
        problem shape, else each candidate timed on a scratch copy of the
        simulation (``torchcor_b200.tune.tune_single``).  Returns the choice."""
        from torchcor_b200 import tune
        self.tuned = tune.tune_single(self, steps=steps, force=force)
        return self.tuned

    def solve(self, a_tol, r_tol, max_iter, calculate_AT_RT=True, linear_guess=True, snapshot_interval=1,
              verbose=True, result_path=None, snapshot_ring=None, graph_steps=100, autotune=True, launch=None,
              stream_results=True):
        """monodomain.py:141-226.  ``snapshot_ring=R`` keeps only R snapshot frames on
        the device and streams every frame, as soon as it is written, into a pinned host
        tensor on a separate stream (``solutions`` is then that host tensor); the
        default keeps every frame on the device, as the reference does.
        ``graph_steps=G`` runs every whole G-step stretch of the loop as the replay of
        one CUDA graph of the same kernels (recorded once per solve); the results are
        bit-identical to plain launches (``graph_steps=0``).  ``autotune`` picks the
        kernels' launch shapes first (``autotune()``; cached per device and shape);
        ``launch`` (a dict of ``ionic_variant``, ``cg_per_sm``, ``fused_step``) sets
        them explicitly instead.  ``stream_results`` (default) writes ``Vm.pt`` while
        the steps run: each frame goes from the device to its place in the file on a
        thread of its own as soon as it is written (the same file as ``torch.save``
        of the frames after the last step, which ``stream_results=False`` does)."""
        self.result_path = Path(result_path) if result_path is not None else None
        if self.result_path is not None:
            self.result_path.mkdir(parents=True, exist_ok=True)
        self.assemble()
        keep = snapshot_interval < self.T
        if snapshot_ring is not None and int(snapshot_ring) < 1:
            raise ValueError("snapshot_ring must be a positive number of frames")
        sim = self._setup(a_tol, r_tol, max_iter, calculate_AT_RT, linear_guess, snapshot_interval, keep,
                          snapshot_ring or 0)
        if launch:
            self.set_launch(**launch)
        elif autotune:
            self.autotune()
        t0 = time.time()
        ring = sim["ring"]
        writer = None
        if ring:
            self._snapshot_stream_init()
            chunk = max(1, sim["per_frame"])
        else:
            chunk = max(1, sim["per_frame"]) * (1 if verbose and snapshot_interval != self.T else 1000)
            if stream_results and keep and self.result_path is not None and self._inv_t is None:
                # Vm.pt is written while the steps run, frame by frame
                writer = sim["vm_writer"] = FrameWriter(self.result_path / "Vm.pt", sim["snaps"])
                chunk = max(1, sim["per_frame"])
        try:
            while sim["next_step"] <= self.nt:
                n = min(chunk, self.nt + 1 - sim["next_step"])
                if ring:
                    self._before_steps(sim["next_step"], n)
                self._advance(n, graph_steps)
                if ring:
                    self._drain_snapshots()
                if writer is not None:
                    ev = torch.cuda.Event()
                    ev.record(torch.cuda.current_stream(self.device))
                    writer.produced(self._frames_written() + 1, ev)
                if verbose and snapshot_interval != self.T:
                    torch.cuda.synchronize(self.device)
                    done = sim["next_step"] - 1
                    print(f"t: {round(done * self.dt, 1)}/{self.T}", "Time elapsed:", round(time.time() - t0, 2),
                          flush=True)
            n_total_iter = self.finish(self.result_path if keep or calculate_AT_RT else None, calculate_AT_RT)
        except BaseException:
            if sim.get("vm_writer") is not None:
                sim.pop("vm_writer").abort()
            raise
        elapsed = time.time() - t0
        if verbose:
            mem = torch.cuda.max_memory_allocated(self.device) / 1e9
            print(self.ionic_model.name, self.n_nodes, round(elapsed, 2), 0.0, round(elapsed, 2), n_total_iter,
                  "n/a", f"{round(mem, 2)}", flush=True)
            if calculate_AT_RT:
                at, rt = sim["at"].cpu(), sim["rt"].cpu()
                print("ATs: ", at.min().item(), at.max().item(), flush=True)
                print("RTs: ", rt.min().item(), rt.max().item(), flush=True)
        return n_total_iter
