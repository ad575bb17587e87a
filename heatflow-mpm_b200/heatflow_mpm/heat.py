"""Temperature on the grid (reference: heatflow_mpm/heat.py).  ``HeatField`` keeps the reference's attributes and
set-up methods; its stages (blend, fixed cells, capped source, advection, implicit diffusion by CG, FLIP particle
update) run in libheatflow_b200 inside ``HeatflowMPM.substep``."""
from __future__ import annotations

import numpy as np
import torch

from .grid import _reported


class HeatField:
    def __init__(self, n: int, h: float, t_init: float, device: str, scene=None):
        self.n, self.h, self.dev = n, h, device
        self.t_init = t_init
        self._scene = scene

    def _bind(self, scene):
        self._scene = scene

    @property
    def T(self):
        return self._scene.current("T")

    @property
    def fixed(self):
        return (self._scene.cell_flags & 1).to(torch.int32)

    @property
    def tfix(self):
        return self._scene.tfix

    @property
    def src(self):
        return ((self._scene.cell_flags >> 1) & 1).to(torch.int32)

    @property
    def rate(self):
        return self._scene.rate

    @property
    def t_cap(self):
        return self._scene.t_cap

    @property
    def kap(self):
        return self._scene.kap

    @property
    def cg_iters(self) -> int:
        """Heat CG iterations of the last substep, quantised like warp's report (check_every=10)."""
        return _reported(self._scene.read_state().heat_iters, 10, self._scene.spec.heat_maxiter)

    @property
    def cg_iters_exact(self) -> int:
        return int(self._scene.read_state().heat_iters)

    def set_fixed(self, fixed: np.ndarray, values: np.ndarray):
        """heat.py:189-192: Dirichlet cells and their values; T takes them at once."""
        self._scene.set_fixed(np.asarray(fixed, bool), np.asarray(values, np.float32))

    def set_source(self, mask: np.ndarray, rate: float, t_cap: float):
        """heat.py:194-196"""
        self._scene.set_source(np.asarray(mask, bool), rate, t_cap)
