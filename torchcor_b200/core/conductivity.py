"""Per-element conductivities with the behaviour of ``torchcor/core/conductivity.py:4-69``.

``add`` sets sigma_l/sigma_t of the listed regions (harmonic mean of intra and
extra values when el/et are given).  The monodomain assembly kernel forms the
tensor sigma = st*I + (sl-st) f f^T itself from (sl, st, fibres);
``calculate_sigma`` returns the (E,3,3) tensors for callers that want them.
"""
from __future__ import annotations

import torch


class Conductivity:
    def __init__(self, regions, dtype):
        self.regions = regions
        self.dtype = dtype
        z = lambda: torch.zeros_like(regions, dtype=dtype)  # noqa: E731
        self.sigma_il, self.sigma_it, self.sigma_el, self.sigma_et = z(), z(), z(), z()
        self.sigma_l, self.sigma_t = z(), z()

    def add(self, region_ids, il, it, el=None, et=None):
        if el is None and et is None:
            self.sigma_il = self.sigma_it = self.sigma_el = self.sigma_et = None
            for rid in region_ids:
                mask = self.regions == rid
                self.sigma_l[mask] = il
                self.sigma_t[mask] = it
        else:
            lv = il * el * (1 / (il + el))
            tv = it * et * (1 / (it + et))
            for rid in region_ids:
                mask = self.regions == rid
                self.sigma_il[mask] = il
                self.sigma_it[mask] = it
                self.sigma_el[mask] = el
                self.sigma_et[mask] = et
                self.sigma_l[mask] = lv
                self.sigma_t[mask] = tv

    def _tensor(self, l, t, fibres):
        E = fibres.shape[0]
        lv, tv = l.view(E, 1, 1), t.view(E, 1, 1)
        s = tv * torch.eye(3, device=fibres.device, dtype=self.dtype).unsqueeze(0).expand(E, 3, 3)
        s += (lv - tv) * fibres.unsqueeze(2) @ fibres.unsqueeze(1)
        return s

    def calculate_sigma(self, fibres):
        if self.sigma_il is None and self.sigma_it is None and self.sigma_el is None and self.sigma_et is None:
            si = se = None
        else:
            si = self._tensor(self.sigma_il, self.sigma_it, fibres)
            se = self._tensor(self.sigma_el, self.sigma_et, fibres)
        return si, se, self._tensor(self.sigma_l, self.sigma_t, fibres)
