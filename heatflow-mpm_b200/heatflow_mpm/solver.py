"""HeatflowMPM: the reference's coupled driver (heatflow_mpm/solver.py:41-110) over the sm_100a air substep.

Same constructor, methods and attributes as the reference.  One extra keyword, ``body``, chooses the material solver:
``"newton"`` (default: Newton's SolverImplicitMPM, as the reference), ``"frozen"`` (particles keep their positions
and velocities; used when Newton is not installed) or a body object of the caller's (``mpm.DLPackBody`` interface).  The air substep itself -- obstacle fields, temperature stages,
heat CG, FLIP particle update, face stage, pressure CG and projection -- is one call into libheatflow_b200, replayed
from a CUDA graph after the first substep at each dt (``graph=False``: launched directly every time; same bits).
``cg="single-reduction"`` solves the pressure system with one grid barrier per CG iteration instead of two (the classic
recurrences with beta from an expansion of the next r.z; the same stopping test; results within ~1e-6 relative of the
classic method, which stays the default)."""
from __future__ import annotations

from dataclasses import asdict

import numpy as np
import torch

from . import _lib
from .grid import AirGrid, GridConfig, grid_edge
from .heat import HeatField
from .heater import Heater
from .mpm import FrozenBody, Material, ThermalMPM
from .scene import DeviceScene, SceneSpec, ScenePlan

KAPPA_AIR = 2.2e-5     # solver.py:15
K_PARTICLE = 1.0e-3    # solver.py:16


def wall_fixed(n: int, cell: np.ndarray, t_rod: float, t_amb: float):
    """solver.py:48-53: rods fixed at t_rod; side walls and ceiling fixed at t_amb (the floor is adiabatic); rods win."""
    rods = cell == 2
    wall = np.zeros((n, n, n), bool)
    wall[[0, -1], :, :] = True
    wall[:, [0, -1], :] = True
    wall[:, :, -1] = True
    fixed = rods | wall
    tfix = np.where(rods, t_rod, np.where(wall, t_amb, 0.0))
    return fixed, tfix


def build_spec(particles, mat: Material, heater, grid: GridConfig, spacing: float, t_init: float, kappa_air: float,
               heat_tol: float = 1e-6, heat_maxiter: int = 200):
    """Host-side scene construction of solver.py:42-61 (no device work): masks, fixed cells, statics, parameters.
    Returns (SceneSpec, cell classes, heater geometry, t_max)."""
    n, h = grid_edge(grid), grid.h
    cell, solid, source, rate, k_faces, m_faces, geom = heater.masks(n, h, (grid.L / 2, grid.L / 2), grid.rho)
    fixed, tfix = wall_fixed(n, cell, heater.t_rod, grid.t_amb)
    t_max = max(heater.t_rod, heater.t_cap, grid.t_amb, t_init)
    spec = SceneSpec(n=n, h=h, rho=grid.rho, t_amb=grid.t_amb, alpha_f_min=grid.alpha_f_min, buoyancy=grid.buoyancy,
                     cg_tol=grid.cg_tol, cg_max_iter=grid.cg_max_iter, heat_tol=heat_tol, heat_maxiter=heat_maxiter,
                     kappa_air=kappa_air, kappa_mat=mat.kappa, fixed=fixed, tfix=tfix, source=source, rate=rate,
                     t_cap=heater.t_cap, static_alpha=solid.astype(np.float32), static_k=k_faces, static_m=m_faces,
                     n_particles=len(particles), spacing=spacing, k_particle=K_PARTICLE, t_sol=mat.t_sol,
                     t_liq=mat.t_liq, y_solid=mat.yield_solid, mu_s=mat.viscosity_solid, mu_l=mat.viscosity_liquid,
                     t_max=t_max)
    return spec, cell, geom, t_max


class HeatflowMPM:
    def __init__(self, particles: np.ndarray, mat: Material = Material(), heater: Heater = Heater(),
                 grid: GridConfig = GridConfig(), spacing: float = 2.5e-3, t_init: float = 20.0,
                 kappa_air: float = KAPPA_AIR, device: str = "cuda:0", *, body: str = "newton",
                 particle_velocities=None, heat_tol: float = 1e-6, heat_maxiter: int = 200, persistent_blocks: int = 0,
                 graph: bool = True, cg: str = "classic"):
        if not torch.cuda.is_available():
            raise RuntimeError("HeatflowMPM needs a CUDA device (sm_100a); there is no CPU path")
        self.mat, self.heater, self.dev, self.spacing, self.kappa_air = mat, heater, device, spacing, kappa_air
        self.use_graph = bool(graph)
        self._graph, self._graph_key = None, None
        self.grid = AirGrid(grid, device)
        self.heat = HeatField(self.grid.n, self.grid.h, grid.t_amb, device)
        particles = np.zeros((0, 3), np.float32) if particles is None else np.asarray(particles, np.float32)
        self.n = len(particles)
        spec, self.cell_type, self.heater_geom, self.t_max = build_spec(particles, mat, heater, grid, spacing, t_init,
                                                                        kappa_air, heat_tol, heat_maxiter)
        with torch.cuda.device(torch.device(device)):
            self.scene = DeviceScene(spec, device)
            self.plan = ScenePlan([self.scene], device, persistent_blocks=persistent_blocks)
            if cg not in ("classic", "single-reduction"):
                raise ValueError("cg must be 'classic' or 'single-reduction'")
            self.plan.single_reduction_cg = cg == "single-reduction"
            self.plan.prepare_statics()
        self.grid._bind(self.scene, self.plan, 0)
        self.heat._bind(self.scene)
        self.grid.static = (spec.static_alpha, spec.static_k, spec.static_m)   # already on the device
        if self.n:
            if not isinstance(body, str):
                self.body = body            # a material solver object (DLPackBody interface) built by the caller
            elif body == "frozen":
                self.body = FrozenBody(particles, spacing, mat, device, particle_velocities)
            else:
                self.body = ThermalMPM(particles, spacing, mat, device)
            self.scene.ptemp.fill_(float(t_init))
            yield_t, visc_t = self.body.material_outputs()
            self.scene.pyield.copy_(yield_t)
            self.scene.pvisc.copy_(visc_t)
        else:
            self.body = None

    # ------------------------------------------------------------------------------------------------ substep
    def substep(self, dt: float):
        """solver.py:63-88: one air substep on the device, then the material step."""
        b, sc = self.body, self.scene
        with torch.cuda.device(torch.device(self.dev)):
            if b is not None:
                pos, vel = b.particle_state()
                sc.pos.copy_(pos)
                sc.pvel.copy_(vel)
            self._air_substep(dt)
            if b is not None:
                ys, vs = b.material_outputs()
                if ys.data_ptr() != sc.pyield.data_ptr():
                    ys.copy_(sc.pyield)
                    vs.copy_(sc.pvisc)
                b.step(dt)

    def _air_substep(self, dt: float):
        """The air substep's launches.  With graph=True the first substep at a given dt (and plan options) runs eagerly
        and is then recorded as a CUDA graph that later substeps replay: the same launches, bit for bit, without the
        host in the loop (the kernels read the buffer parity on the device, so one recording serves every substep).
        A changed scene record (set_source) is uploaded first and drops the recording; inside a caller's own stream
        capture the launches are issued directly."""
        plan = self.plan
        if not self.use_graph or torch.cuda.is_current_stream_capturing():
            plan.substep(dt)
            return
        if any(sc.dirty for sc in plan.scenes):
            plan.upload()
            for sc in plan.scenes:
                sc.dirty = False
            self._graph = None
        key = (float(dt), int(plan.plan.options), int(plan.plan.persistent_blocks), int(plan.plan.group_cells))
        if self._graph is not None and self._graph_key == key:
            self._graph.replay()
            return
        plan.substep(dt)
        dev = torch.device(self.dev)
        cur = torch.cuda.current_stream(dev)
        side = torch.cuda.Stream(dev)
        side.wait_stream(cur)
        g = torch.cuda.CUDAGraph()
        # thread-local capture: a frame writer's thread may wait on its own copies meanwhile
        with torch.cuda.graph(g, stream=side, capture_error_mode="thread_local"):
            plan.substep(dt)
        cur.wait_stream(side)
        self._graph, self._graph_key = g, key

    def status(self) -> dict:
        """Solver status of the last substep: CG iterations, residuals, status bits (0 = converged everywhere)."""
        st = self.scene.read_state()
        return dict(status=int(st.status), substeps=int(st.substeps), heat_iters=int(st.heat_iters),
                    pressure_iters=int(st.pressure_iters), heat_rr=st.heat_rr, heat_atol=st.heat_atol,
                    pressure_rr=st.pressure_rr, pressure_atol=st.pressure_atol, pressure_bb=st.pressure_bb,
                    heat_bb=st.heat_bb, rhs_mean=st.rhs_mean)

    # -------------------------------------------------------------------------------------------------- state
    def positions(self):
        return self.body.positions() if self.body else np.zeros((0, 3), np.float32)

    def velocities(self):
        return self.body.velocities() if self.body else np.zeros((0, 3), np.float32)

    def temperatures(self):
        return self.scene.ptemp.cpu().numpy()[: self.n] if self.n else np.zeros(0, np.float32)

    def melt_fraction(self):
        return self.scene.pmelt.cpu().numpy()[: self.n] if self.n else np.zeros(0, np.float32)

    def grid_T(self, out=None):
        """solver.py:95: grid temperature (n,n,n) on the host.  `out` (optional, e.g. a pinned torch tensor) receives
        the copy instead of a new numpy array."""
        if out is not None:
            out.copy_(self.heat.T)
            return out
        return self.heat.T.cpu().numpy()

    def grid_T_async(self, out):
        """grid_T into `out` (a pinned host tensor of shape (n,n,n)) without waiting: the current temperature is copied
        on the device into one of two staging buffers, then downloaded on a side stream while the next substeps run.
        Returns a torch.cuda.Event that completes when `out` holds the data.  A staging buffer is refilled only after
        its previous download finished, so at most two downloads are in flight."""
        import ctypes as C
        n = self.grid.n
        if not hasattr(self, "_stage"):
            self._stage = [torch.empty((n, n, n), dtype=torch.float32, device=self.dev) for _ in range(2)]
            self._stage_done = [None, None]
            self._stage_k = 0
            self._copy_stream = torch.cuda.Stream(torch.device(self.dev))
        k = self._stage_k % 2
        self._stage_k += 1
        compute = torch.cuda.current_stream(torch.device(self.dev))
        if self._stage_done[k] is not None:
            compute.wait_event(self._stage_done[k])
        buf = self._stage[k]
        _lib.check(self.plan.L.hf_current_field(C.byref(self.plan.plan), 0, 0, buf.data_ptr(),
                                                C.c_void_p(compute.cuda_stream)), "hf_current_field")
        self._copy_stream.wait_stream(compute)
        with torch.cuda.stream(self._copy_stream):
            out.copy_(buf, non_blocking=True)
            done = torch.cuda.Event()
            done.record(self._copy_stream)
        self._stage_done[k] = done
        return done

    def air_velocity(self):
        return self.grid.cell_velocity()

    def static_dict(self) -> dict:
        """solver.py:98-103"""
        hg = self.heater_geom
        return dict(L=self.grid.L, h=self.grid.h, n=self.grid.n, n_particles=self.n, spacing=self.spacing,
                    t_amb=self.grid.cfg.t_amb, cell_type=self.cell_type.astype(np.uint8), heater_on=int(self.heater.on),
                    heater_centre=np.array(hg["centre"], np.float32), heater_facing=np.array(hg["facing"], np.float32),
                    heater_tilt=getattr(self.heater, "tilt", 0.0), heater_radius=getattr(self.heater, "radius", 0.0),
                    heater_length=getattr(self.heater, "length", 0.0),
                    **{f"mat_{k}": v for k, v in asdict(self.mat).items() if not isinstance(v, str)})

    def frame_dict(self, t: float, with_air: bool = True) -> dict:
        """solver.py:105-110"""
        d = dict(t=np.float32(t), pos=self.positions().astype(np.float32), vel=self.velocities().astype(np.float32),
                 temp=self.temperatures().astype(np.float16), melt=self.melt_fraction().astype(np.float16),
                 grid_T=self.grid_T().reshape(-1).astype(np.float16))
        if with_air:
            d["air_u"] = self.air_velocity().astype(np.float16)
        return d
