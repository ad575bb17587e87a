"""Air on a closed MAC grid (reference: heatflow_mpm/grid.py).  ``GridConfig`` is the reference's dataclass; ``AirGrid``
keeps the reference's attribute and method names as views onto a device scene whose stages run in libheatflow_b200."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class GridConfig:
    """grid.py:13-22 (same fields and defaults)."""
    L: float = 0.48
    h: float = 0.005
    rho: float = 1.2
    t_amb: float = 25.0
    buoyancy: bool = True
    alpha_f_min: float = 0.05
    cg_tol: float = 1e-4
    cg_max_iter: int = 400


def grid_edge(cfg: GridConfig) -> int:
    """grid.py:183: cells per edge."""
    return int(round(cfg.L / cfg.h))


class AirGrid:
    """Face velocities u, v, w and cell pressure p of one scene (grid.py:177-263).

    Fields are torch CUDA tensors in the reference's shapes; ``u``, ``v``, ``w`` return the current buffer.  The stage
    kernels run inside ``HeatflowMPM.substep``; the diagnostics below are the reference's."""

    def __init__(self, cfg: GridConfig, device: str, scene=None, plan=None, index: int = 0):
        self.cfg, self.dev = cfg, device
        self.n = grid_edge(cfg)
        self.h, self.L = cfg.h, cfg.L
        self._scene, self._plan, self._index = scene, plan, index
        self.static = None

    def _bind(self, scene, plan, index=0):
        self._scene, self._plan, self._index = scene, plan, index

    @property
    def u(self):
        return self._scene.current("u")

    @property
    def v(self):
        return self._scene.current("v")

    @property
    def w(self):
        return self._scene.current("w")

    @property
    def p(self):
        return self._scene.p

    @property
    def rhs(self):
        return self._scene.rhs

    @property
    def alpha_s(self):
        return self._scene.alpha_s

    @property
    def ax(self):
        return self._scene.ax

    @property
    def ay(self):
        return self._scene.ay

    @property
    def az(self):
        return self._scene.az

    @property
    def cg_iters(self) -> int:
        """Pressure CG iterations of the last substep, quantised like warp's report (multiples of check_every=20)."""
        return _reported(self._scene.read_state().pressure_iters, 20, self.cfg.cg_max_iter)

    @property
    def cg_iters_exact(self) -> int:
        return int(self._scene.read_state().pressure_iters)

    def set_static(self, alpha, k_faces, m_faces):
        """grid.py:198-200: replace the static obstacle fields (solid fraction (n,n,n); relaxation weights k and
        momentum m on the three face lattices) that every substep adds to the particle contributions (grid.py:206-213).
        The new arrays are copied into the scene's device statics and the obstacle fields, face fractions and
        conductivity are rebuilt from them at once, so the next substep uses them (a recorded substep graph stays
        valid: it reads the same buffers)."""
        n = self.n
        alpha = np.asarray(alpha, np.float32)
        ks = [np.asarray(a, np.float32) for a in k_faces]
        ms = [np.asarray(a, np.float32) for a in m_faces]
        shapes = [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)]
        if alpha.shape != (n, n, n) or [a.shape for a in ks] != shapes or [a.shape for a in ms] != shapes:
            raise ValueError("set_static: alpha (n,n,n) and three k and m face arrays of the MAC lattices expected")
        self.static = (alpha, ks, ms)
        if self._scene is not None:
            self._scene.set_statics(alpha, ks, ms)
            self._plan.prepare_statics()

    def cell_velocity(self) -> np.ndarray:
        """grid.py:253-255: cell-centred velocity (n^3, 3) float32 on the host."""
        return self._plan.cell_velocity(self._index).cpu().numpy()

    def divergence_max(self) -> float:
        """grid.py:257-260"""
        return self._plan.divergence_max(self._index)

    def speed_max(self) -> float:
        """grid.py:262-263"""
        return self._plan.speed_max(self._index)


def _reported(done: int, check_every: int, maxiter: int) -> int:
    """Iteration count warp.optim.linear.cg reports for a solve that converged after `done` iterations: the loop runs
    in pairs and only tests convergence on the host every `check_every` iterations."""
    if done <= 0:
        return 0
    m = maxiter + (maxiter & 1)
    r = -(-done // check_every) * check_every
    return min(r, m)
