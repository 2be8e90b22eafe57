"""Many monodomain simulations stepping together on one GPU.

``MonodomainBatch`` holds prepared ``Monodomain`` simulations of any sizes,
ionic models, time steps and end times.  Every batch step launches one ionic
kernel per model and one persistent CG kernel for all of them; each simulation
keeps its own step counter, stimulus schedule, tolerances and iteration count
(it stops iterating when it converges, the others go on), and simulations can
join or leave between steps.  Results are the same as running each one alone
(up to the float64 reduction order inside CG).
"""
from __future__ import annotations

import ctypes as C

import torch

from torchcor_b200 import _lib
from torchcor_b200._lib import check, stream_ptr

MAX_SIMS = 1024


class MonodomainBatch:
    def __init__(self, device=None, max_sims=MAX_SIMS):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        lib = _lib.load()
        self.max_sims = max_sims
        self._ws = torch.empty(int(lib.tcb_batch_workspace_bytes(max_sims)), dtype=torch.uint8, device=self.device)
        self._plan = _lib.tcb_batch_plan()
        self._structs = None
        self.sims = []
        self._dirty = True
        self._cg_variant = None
        self._ionic_tpb = 0
        self._ionic_bps = 0
        self._ionic_staged = 0

    def add(self, sim, a_tol=1e-5, r_tol=1e-5, max_iter=100, calculate_AT_RT=True, linear_guess=True,
            snapshot_interval=1):
        """Prepare ``sim`` (a ``Monodomain`` with mesh, conductivities and stimuli) and add it."""
        if len(self.sims) >= self.max_sims:
            raise RuntimeError(f"batch is full ({self.max_sims} simulations)")
        if sim._sim is None:
            sim.prepare(a_tol, r_tol, max_iter, calculate_AT_RT, linear_guess, snapshot_interval)
        self.sims.append(sim)
        self._dirty = True
        return sim

    def remove(self, sim, result_path=None):
        """Take ``sim`` out of the batch; if it has run all its steps, finish it."""
        self.sims.remove(sim)
        self._dirty = True
        if sim._sim["next_step"] > sim.nt:
            return sim.finish(result_path)
        return None

    def _prepare(self):
        n = len(self.sims)
        arr = (_lib.tcb_mono * n)()
        for i, s in enumerate(self.sims):
            s._sync_node_params()
            arr[i] = s._sim["struct"]
        self._structs = arr
        lib = _lib.load()
        check(lib.tcb_batch_prepare(arr, n, self._ws.data_ptr(), self._ws.numel(), C.byref(self._plan)))
        if self._cg_variant is not None:
            st = lib.tcb_batch_set_cg(C.byref(self._plan), int(self._cg_variant))
            if st != 0 and self._cg_variant == 3:   # staged variant not possible for these arrays
                self._cg_variant = None
            else:
                check(st)
        if self._ionic_staged and not self._plan.ionic_stage_ok:
            self._ionic_staged = 0       # the arrays of these simulations do not allow it
            if self._ionic_bps == 12:
                self._ionic_bps = 0
        if self._ionic_tpb or self._ionic_bps or self._ionic_staged:
            check(lib.tcb_batch_set_ionic(C.byref(self._plan), int(self._ionic_tpb), int(self._ionic_bps),
                                          int(self._ionic_staged)))
        self._dirty = False

    def set_cg(self, variant):
        """Use batched CG kernel variant 1 or 2 (streaming, sized for 1 or 2 blocks
        per SM) or 3 (ELL streams staged in shared memory by bulk copies)."""
        if variant not in (1, 2, 3):
            raise ValueError("variant must be 1, 2 or 3")
        self._cg_variant = variant
        if self.sims and not self._dirty:
            check(_lib.load().tcb_batch_set_cg(C.byref(self._plan), int(variant)))

    def set_ionic(self, tiles_per_block=None, blocks_per_sm=None, staged=None):
        """The batched ionic launch: tiles of 128 nodes each block walks, 0 (sized
        from the model groups, the default) or 1..64; the kernel instance's register
        budget, 0 (default: 8 blocks of 128 threads per SM with CRN simulations, else
        12; staged 6) or 4, 6, 8, 12 (not 12 staged); and the staged form (each
        block's next tile copied into shared memory by bulk copies while it computes
        one; hardware division for TTP and CRN, as the single-simulation default).
        ``None`` keeps the current value."""
        tpb = self._ionic_tpb if tiles_per_block is None else int(tiles_per_block)
        bps = self._ionic_bps if blocks_per_sm is None else int(blocks_per_sm)
        stg = self._ionic_staged if staged is None else int(bool(staged))
        if not 0 <= tpb <= 64:
            raise ValueError("tiles_per_block must be in 0..64")
        if bps not in ((0, 4, 6, 8) if stg else (0, 4, 6, 8, 12)):
            raise ValueError("blocks_per_sm must be 0, 4, 6, 8 or (unstaged) 12")
        self._ionic_tpb, self._ionic_bps, self._ionic_staged = tpb, bps, stg
        if self.sims and not self._dirty:
            check(_lib.load().tcb_batch_set_ionic(C.byref(self._plan), tpb, bps, stg))

    @property
    def ionic_staged(self):
        return self._ionic_staged

    def ionic_stage_ok(self):
        """True if the simulations' per-node arrays allow the staged ionic form."""
        if self._dirty and self.sims:
            self._prepare()
        return bool(self._plan.ionic_stage_ok)

    @property
    def ionic_tiles_per_block(self):
        return self._ionic_tpb

    @property
    def ionic_blocks_per_sm(self):
        return self._ionic_bps

    def cg_variants(self):
        """The CG variants this batch can use (3 needs 16-byte aligned ELL arrays)."""
        if self._dirty and self.sims:
            self._prepare()
        return (2, 1, 3) if self._plan.cg_stage_ok else (2, 1)

    def autotune(self, steps=10, cache=None, force=False):
        """Choose the batched CG variant for this batch's shape on this GPU
        (cached; on a miss it times real steps of the batch, see
        ``torchcor_b200.tune.tune_batch``).  Returns the chosen variant."""
        from torchcor_b200.tune import tune_batch
        if self._dirty and self.sims:
            self._prepare()
        return tune_batch(self, steps=steps, cache=cache, force=force)[0]

    @property
    def cg_config(self):
        """(CG variant, CG blocks) of the current plan."""
        if self._dirty and self.sims:
            self._prepare()
        return int(self._plan.cg_variant), int(self._plan.cg_blocks)

    def step(self, n_steps=1):
        """Advance every unfinished simulation by ``n_steps`` steps (asynchronous)."""
        if not self.sims:
            return
        if self._dirty:
            self._prepare()
        check(_lib.load().tcb_batch_run(C.byref(self._plan), int(n_steps), stream_ptr()))
        for s in self.sims:
            s._sim["next_step"] = min(s._sim["next_step"] + n_steps, s.nt + 1)

    def capture(self, n_steps):
        """Record ``n_steps`` batch steps in a CUDA graph; returns a callable that
        replays them (and advances the step bookkeeping).  The batch must not
        change while the graph is in use; every simulation must have at least
        ``n_steps`` steps left per replay (finished ones are skipped on the
        device, the bookkeeping stops at their last step)."""
        if self._dirty:
            self._prepare()
        graph = torch.cuda.CUDAGraph()
        plan = self._plan
        lib = _lib.load()
        with torch.cuda.graph(graph):
            check(lib.tcb_batch_run(C.byref(plan), int(n_steps), stream_ptr()))

        def replay():
            if self._dirty:
                raise RuntimeError("the batch changed after capture; capture again")
            graph.replay()
            for s in self.sims:
                s._sim["next_step"] = min(s._sim["next_step"] + n_steps, s.nt + 1)
        replay.graph = graph
        return replay

    def finished(self):
        return [s for s in self.sims if s._sim["next_step"] > s.nt]

    def remaining_steps(self):
        return max((s.nt + 1 - s._sim["next_step"] for s in self.sims), default=0)

    def check(self):
        if self.sims and not self._dirty:
            check(_lib.load().tcb_batch_check(C.byref(self._plan), stream_ptr()))

    def run(self, result_paths=None):
        """Step until every simulation has finished; finish and remove them all."""
        while self.sims:
            k = min(s.nt + 1 - s._sim["next_step"] for s in self.sims if s._sim["next_step"] <= s.nt) \
                if any(s._sim["next_step"] <= s.nt for s in self.sims) else 0
            if k > 0:
                self.step(k)
                self.check()
            for s in self.finished():
                self.remove(s, None if result_paths is None else result_paths.get(id(s)))
