"""Stimuli with the behaviour of ``torchcor/core/stimulation.py:6-63``.

A stimulus is a node set (``.vtx``), a window [start, start+duration] that
repeats every ``period`` up to ``count`` times, and an intensity.  On the
device, the simulator does not add dense vectors: it uploads one membership
bit per node and stimulus and a per-step mask of active stimuli, computed
here on the host with the reference's float64 arithmetic (``t`` accumulated
by ``t += dt``, inclusive window test).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from torchcor_b200.core.mesh import read_vtx
from torchcor_b200._lib import TCB_MAX_STIMULI


@dataclass
class StimConfig:
    vtx_filepath: str
    region: np.ndarray
    start: float
    duration: float
    intensity: float
    period: float
    count: float


class Stimuli:
    def __init__(self, n_nodes, device, dtype):
        self.stimulus_list: list[StimConfig] = []
        self.n_nodes = n_nodes
        self.device = device
        self.dtype = dtype

    def add(self, vtx_filepath, start, duration, intensity, period=None, count=1, region=None):
        if period is None:
            raise Exception("period is unspecified.")
        if len(self.stimulus_list) >= TCB_MAX_STIMULI:
            raise ValueError(f"at most {TCB_MAX_STIMULI} stimuli per simulation")
        if region is None:
            region = read_vtx(vtx_filepath)
        region = np.asarray(region, dtype=np.int64)
        if region.size and (region.min() < -self.n_nodes or region.max() >= self.n_nodes):
            raise IndexError("stimulus node index out of range")
        self.stimulus_list.append(StimConfig(str(vtx_filepath), region, start, duration, intensity, period, count))

    @staticmethod
    def is_active(s: StimConfig, t: float) -> bool:
        """Window test of stimulation.py:51-58 (float64, inclusive)."""
        p_t = t % s.period
        t_t = t / s.period
        return t_t <= s.count and (p_t >= s.start and p_t <= s.start + s.duration)

    def membership_bits(self):
        """uint32 per node: bit k set when the node belongs to stimulus k."""
        bits = np.zeros(self.n_nodes, dtype=np.uint32)
        for k, s in enumerate(self.stimulus_list):
            bits[s.region] |= np.uint32(1 << k)
        return bits

    def amplitudes(self):
        a = np.zeros(TCB_MAX_STIMULI, dtype=np.float32)
        for k, s in enumerate(self.stimulus_list):
            a[k] = np.float32(1.0) * np.float32(s.intensity)
        return a

    def schedule(self, nt, dt):
        """(t32[nt+1], mask[nt+1]) for steps n = 1..nt; index 0 is t = 0."""
        t32 = np.zeros(nt + 1, dtype=np.float32)
        mask = np.zeros(nt + 1, dtype=np.uint32)
        t = 0
        for n in range(1, nt + 1):
            t += dt
            t32[n] = t
            m = 0
            for k, s in enumerate(self.stimulus_list):
                if self.is_active(s, t):
                    m |= 1 << k
            mask[n] = m
        return t32, mask

    def apply(self, t):
        """Dense sum of the stimuli active at ``t`` (stimulation.py:51-63)."""
        out = torch.zeros((self.n_nodes,), device=self.device, dtype=self.dtype)
        for s in self.stimulus_list:
            if self.is_active(s, t):
                v = torch.zeros((self.n_nodes,), device=self.device, dtype=self.dtype)
                v[torch.as_tensor(s.region, device=self.device)] = 1.0
                out = out + v * s.intensity
        return out
