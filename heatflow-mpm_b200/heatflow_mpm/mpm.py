"""Material particles (reference: heatflow_mpm/mpm.py).  ``Material`` is the reference's dataclass.  ``ThermalMPM`` keeps
NVIDIA Newton's SolverImplicitMPM as the material solver (imported lazily, as the reference does), exchanging particle
arrays with the air path through DLPack.  ``FrozenBody`` is a stand-in body whose particles keep their positions and
velocities; it drives the coupled air path when Newton is not installed (synthetic benchmarks, parity tests).
``DLPackBody`` is the exchange itself, for any material solver whose arrays speak DLPack."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class Material:
    """mpm.py:9-22 (same fields and defaults)."""
    rho: float = 1300.0
    t_sol: float = 30.0
    t_liq: float = 36.0
    yield_solid: float = 2.0e4
    viscosity_solid: float = 5.0
    viscosity_liquid: float = 30.0
    kappa: float = 2.0e-5
    ground_friction: float = 0.3
    strain_basis: str = "Q1"
    voxel_mult: float = 2.0
    max_iterations: int = 250
    tolerance: float = 1.0e-5


class FrozenBody:
    """Particles that do not move: positions and velocities stay as given (torch tensors on the device)."""

    def __init__(self, particles: np.ndarray, spacing: float, mat: Material, device: str, velocities=None):
        self.dev, self.n = device, len(particles)
        self.pos_t = torch.as_tensor(np.asarray(particles, np.float32), device=device).contiguous()
        v = np.zeros_like(particles, dtype=np.float32) if velocities is None else np.asarray(velocities, np.float32)
        self.vel_t = torch.as_tensor(v, device=device).contiguous()
        self.yield_t = torch.full((self.n,), float(mat.yield_solid), device=device)
        self.visc_t = torch.full((self.n,), float(mat.viscosity_solid), device=device)

    def particle_state(self):
        return self.pos_t, self.vel_t

    def set_state(self, positions, velocities):
        """Replace the particle state (host arrays or tensors).  Pinned host tensors are uploaded on a side stream into
        the one of two device buffer pairs that no queued work still reads -- the one the substep before the previous
        call copied from -- so the upload overlaps the substep in flight; work issued afterwards on the current stream
        (the next substep) waits for it.  As with any asynchronous copy, the pinned tensors must not be rewritten until
        that work has run.  Other inputs are copied in stream order."""
        p, v = torch.as_tensor(positions), torch.as_tensor(velocities)
        if p.is_cuda or v.is_cuda or not (p.is_pinned() and v.is_pinned()):
            self.pos_t.copy_(p, non_blocking=True)
            self.vel_t.copy_(v, non_blocking=True)
            return
        dev = torch.device(self.dev)
        if getattr(self, "_up", None) is None:
            self._up = torch.cuda.Stream(dev)
            self._bufs = [(self.pos_t, self.vel_t), (torch.empty_like(self.pos_t), torch.empty_like(self.vel_t))]
            self._free = [None, None]   # event after which no queued work reads the pair
            self._k = 0
        compute = torch.cuda.current_stream(dev)
        k = self._k ^ 1               # the pair not holding the current state
        if self._free[k] is not None:
            self._up.wait_event(self._free[k])
        with torch.cuda.stream(self._up):
            self._bufs[k][0].copy_(p, non_blocking=True)
            self._bufs[k][1].copy_(v, non_blocking=True)
            ready = torch.cuda.Event()
            ready.record(self._up)
        # the current pair is read by work already queued on this stream (the substep issued since the last call)
        freed = torch.cuda.Event()
        freed.record(compute)
        self._free[self._k] = freed
        compute.wait_event(ready)
        self._k = k
        self.pos_t, self.vel_t = self._bufs[k]

    def material_outputs(self):
        return self.yield_t, self.visc_t

    def step(self, dt: float):
        pass

    def positions(self) -> np.ndarray:
        return self.pos_t.cpu().numpy()

    def velocities(self) -> np.ndarray:
        return self.vel_t.cpu().numpy()


def dlpack_view(arr) -> torch.Tensor:
    """A zero-copy torch view of another framework's device array: through the DLPack protocol (``__dlpack__``, which
    Warp, CuPy, JAX and torch arrays implement) or, for arrays without it, Warp's ``to_dlpack`` capsule."""
    if hasattr(arr, "__dlpack__"):
        return torch.from_dlpack(arr)
    import warp as wp
    return torch.from_dlpack(wp.to_dlpack(arr))


class DLPackBody:
    """The material side of the air substep (mpm.py:54-68, heat.py:161-174) for a solver that owns its particle arrays:
    positions and velocities are read, and yield stress and viscosity written, through zero-copy DLPack views of the
    solver's own device arrays -- no host copies and no extra device buffers.  A subclass names the arrays
    (``dlpack_arrays``: particle_q (P,3), particle_qd (P,3), yield_stress (P), viscosity (P)) and advances the solver
    (``step``)."""

    def dlpack_arrays(self):
        raise NotImplementedError

    def particle_state(self):
        q, qd, _, _ = self.dlpack_arrays()
        return dlpack_view(q).view(-1, 3), dlpack_view(qd).view(-1, 3)

    def material_outputs(self):
        _, _, ys, visc = self.dlpack_arrays()
        return dlpack_view(ys), dlpack_view(visc)

    def step(self, dt: float):
        raise NotImplementedError

    def positions(self) -> np.ndarray:
        return self.particle_state()[0].cpu().numpy()

    def velocities(self) -> np.ndarray:
        return self.particle_state()[1].cpu().numpy()


class ThermalMPM(DLPackBody):
    """mpm.py:25-80: Newton implicit MPM body; its particle state is read, and its yield stress and viscosity written,
    through zero-copy DLPack views."""

    def __init__(self, particles: np.ndarray, spacing: float, mat: Material, device: str):
        import warp as wp
        import newton
        from newton.solvers import SolverImplicitMPM
        self._wp = wp
        self.dev, self.n = device, len(particles)
        mass = mat.rho * spacing ** 3
        with wp.ScopedDevice(device):
            b = newton.ModelBuilder()
            SolverImplicitMPM.register_custom_attributes(b)
            b.add_particles(pos=[wp.vec3(*p) for p in particles], vel=[wp.vec3(0.0)] * self.n, mass=[mass] * self.n,
                            radius=[spacing / 2] * self.n)
            b.add_ground_plane(cfg=newton.ModelBuilder.ShapeConfig(mu=mat.ground_friction))
            self.model = b.finalize()
            self.model.set_gravity((0.0, 0.0, -9.81))
            m = self.model.mpm
            m.friction.fill_(0.0)
            m.tensile_yield_ratio.fill_(1.0)
            m.yield_pressure.fill_(1.0e10)
            m.yield_stress.fill_(mat.yield_solid)
            m.viscosity.fill_(mat.viscosity_solid)
            cfg = SolverImplicitMPM.Config()
            cfg.voxel_size = mat.voxel_mult * spacing
            cfg.grid_type = "sparse"
            cfg.transfer_scheme = "apic"
            cfg.max_iterations = mat.max_iterations
            cfg.tolerance = mat.tolerance
            cfg.strain_basis = mat.strain_basis
            self.solver = SolverImplicitMPM(self.model, config=cfg)
            self.s0, self.s1 = self.model.state(), self.model.state()

    def dlpack_arrays(self):
        return self.s0.particle_q, self.s0.particle_qd, self.model.mpm.yield_stress, self.model.mpm.viscosity

    def step(self, dt: float):
        with self._wp.ScopedDevice(self.dev):
            self.solver.step(self.s0, self.s1, None, None, dt)
            self.solver.project_outside(self.s1, self.s1, dt)
        self.s0, self.s1 = self.s1, self.s0

    def positions(self) -> np.ndarray:
        return self.s0.particle_q.numpy()

    def velocities(self) -> np.ndarray:
        return self.s0.particle_qd.numpy()
