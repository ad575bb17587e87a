"""The material side of the air substep without Newton, and AirGrid.set_static.

* DLPack hand-off (reference mpm.py:54-68 and heat.py:161-174): HeatflowMPM drives a stand-in material solver laid out
  like Newton's SolverImplicitMPM (state.particle_q / particle_qd, model.mpm.yield_stress / viscosity), whose arrays
  expose only the DLPack protocol, as Warp arrays do.  Every substep the air path reads the particle state through the
  views and writes yield stress and viscosity into the solver's own arrays in place; the solver then moves its
  particles.  Checked against the oracle driven with the same positions, velocities and temperatures.
* AirGrid.set_static (reference grid.py:198-213): new statics take effect at the next substep, against the oracle
  built with the same statics.
"""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

DT = 2e-3


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


class _DLPackArray:
    """A device array that offers nothing but the DLPack protocol (like a Warp array)."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, stream=None, **kw):
        return self._t.__dlpack__(stream=stream)

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


class _NS:
    pass


def _newton_like(positions, velocities, yield_solid, visc_solid):
    """A material solver with Newton's attribute layout; its step drifts the particles by dt * velocity."""
    import torch
    from heatflow_mpm.mpm import DLPackBody

    class NewtonLike(DLPackBody):
        def __init__(self):
            self.q = torch.as_tensor(positions, device="cuda").contiguous()
            self.qd = torch.as_tensor(velocities, device="cuda").contiguous()
            self.ys = torch.full((len(positions),), yield_solid, device="cuda")
            self.visc = torch.full((len(positions),), visc_solid, device="cuda")
            self.s0, self.model = _NS(), _NS()
            self.model.mpm = _NS()
            self.s0.particle_q, self.s0.particle_qd = _DLPackArray(self.q), _DLPackArray(self.qd)
            self.model.mpm.yield_stress, self.model.mpm.viscosity = _DLPackArray(self.ys), _DLPackArray(self.visc)
            self.steps = 0

        def dlpack_arrays(self):
            return self.s0.particle_q, self.s0.particle_qd, self.model.mpm.yield_stress, self.model.mpm.viscosity

        def step(self, dt):
            self.q.add_(self.qd * dt)
            self.steps += 1

    return NewtonLike()


def _small_scene():
    from heatflow_mpm import GridConfig, Heater, Material
    rng = np.random.default_rng(8)
    grid = GridConfig(L=0.12, h=0.01, cg_tol=1e-5)
    heater = Heater(dist=0.035, z=0.04, radius=0.025, length=0.08, power=50.0, t_cap=120.0, fan=2.0)
    mat = Material(t_sol=28.0, t_liq=34.0)
    g = np.arange(0.045, 0.075, 0.005)
    parts = np.stack(np.meshgrid(g, g, np.arange(0.005, 0.03, 0.005), indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    vel = rng.uniform(-0.2, 0.2, parts.shape).astype(np.float32)
    return grid, heater, mat, parts, vel


def test_dlpack_handoff_with_a_newton_like_solver(torch_cuda):
    torch = torch_cuda
    from heatflow_mpm import HeatflowMPM
    from heatflow_mpm.solver import wall_fixed
    from oracle import oracle as O
    grid, heater, mat, parts, vel = _small_scene()
    body = _newton_like(parts, vel, mat.yield_solid, mat.viscosity_solid)
    ys_ptr, visc_ptr = body.ys.data_ptr(), body.visc.data_ptr()
    sim = HeatflowMPM(parts, mat=mat, heater=heater, grid=grid, spacing=0.005, body=body, t_init=27.8)
    assert sim.body is body
    n = sim.grid.n
    rng = np.random.default_rng(2)
    T0 = (30.0 + rng.uniform(-2, 8, (n, n, n))).astype(np.float32)
    sim.scene.set_current("T", T0)
    cell, solid, source, rate, kf, mf, _ = heater.masks(n, grid.h, (grid.L / 2, grid.L / 2), grid.rho)
    fixed, tfix = wall_fixed(n, cell, heater.t_rod, grid.t_amb)
    orc = O.OracleScene(n, grid.h, cg_tol=grid.cg_tol, fixed=fixed, tfix=tfix, src=source, rate=rate,
                        t_cap=heater.t_cap, static_alpha=solid.astype(np.float32), static_k=kf, static_m=mf,
                        particles=parts, pvel=vel, ptemp=np.full(len(parts), 27.8, np.float32), spacing=0.005,
                        t_sol=28.0, t_liq=34.0, t_max=sim.t_max, kappa_mat=mat.kappa)
    orc.set_state(T=sim.scene.current("T").cpu().numpy())
    for s in range(4):
        q_before = body.q.cpu().numpy()
        orc.a["pos"][...] = q_before           # the oracle sees the positions the solver holds before the substep
        sim.substep(DT)
        orc.substep(DT)
        assert sim.status()["status"] == 0
        assert body.steps == s + 1
        # positions and velocities were read through the views: the scene's copies are the solver's arrays
        assert np.array_equal(sim.scene.pos.cpu().numpy(), q_before)
        assert np.array_equal(sim.scene.pvel.cpu().numpy(), vel)
        # yield stress and viscosity were written into the solver's own arrays, in place
        assert body.ys.data_ptr() == ys_ptr and body.visc.data_ptr() == visc_ptr
        ref = orc.particles()
        assert np.allclose(body.ys.cpu().numpy(), ref["yield_stress"], rtol=1e-6, atol=1e-3)
        assert np.allclose(body.visc.cpu().numpy(), ref["viscosity"], rtol=1e-6, atol=1e-6)
        assert rel_l2(sim.temperatures(), ref["temp"]) <= 1e-6
        assert rel_l2(sim.grid_T(), orc.T) <= 1e-6
    assert body.ys.cpu().numpy().min() < mat.yield_solid     # particles just below T_sol in warm air start to melt
    assert np.allclose(sim.positions(), body.q.cpu().numpy())


def test_set_static_takes_effect(torch_cuda):
    """Replace the heater's statics after construction with the same statics plus a solid block in the middle of the
    box (alpha_s = 1, K_SOLID faces around it): the scene's solid fraction and face fractions change at once, and the
    next substeps equal the oracle built with the new statics."""
    from heatflow_mpm import GridConfig, Heater, HeatflowMPM
    from heatflow_mpm.heater import K_SOLID
    from heatflow_mpm.solver import wall_fixed
    from oracle import oracle as O
    grid = GridConfig(L=0.24, h=0.01, cg_tol=1e-6)
    heater = Heater(power=200.0, t_cap=120.0, fan=1.0, dist=0.06, z=0.05, radius=0.03, length=0.1)
    sim = HeatflowMPM(None, heater=heater, grid=grid)
    n = sim.grid.n
    for _ in range(2):
        sim.substep(DT)
    cell, solid, source, rate, kf, mf, _ = heater.masks(n, grid.h, (grid.L / 2, grid.L / 2), grid.rho)
    alpha = solid.astype(np.float32).copy()
    lo, hi = n // 2 - 3, n // 2 + 3
    alpha[lo:hi, lo:hi, 2:8] = 1.0
    kf = [a.astype(np.float32).copy() for a in kf]
    kf[0][lo:hi + 1, lo:hi, 2:8] = K_SOLID
    kf[1][lo:hi, lo:hi + 1, 2:8] = K_SOLID
    kf[2][lo:hi, lo:hi, 2:9] = K_SOLID
    sim.grid.set_static(alpha, kf, mf)
    assert np.array_equal(sim.grid.alpha_s.cpu().numpy(), alpha)
    ax = sim.grid.ax.cpu().numpy()
    assert ax[n // 2, n // 2, 4] == np.float32(grid.alpha_f_min)      # a face inside the new block
    fixed, tfix = wall_fixed(n, cell, heater.t_rod, grid.t_amb)
    orc = O.OracleScene(n, grid.h, cg_tol=grid.cg_tol, fixed=fixed, tfix=tfix, src=source, rate=rate,
                        t_cap=heater.t_cap, static_alpha=alpha, static_k=kf, static_m=mf)
    orc.set_state(**{nm: sim.scene.current(nm).cpu().numpy() for nm in ("T", "u", "v", "w")})
    orc.a["p"][...] = sim.grid.p.cpu().numpy()
    for _ in range(3):
        sim.substep(DT)
        orc.substep(DT)
        assert sim.status()["status"] == 0
    for nm in ("T", "u", "v", "w"):
        assert rel_l2(sim.scene.current(nm).cpu().numpy(), getattr(orc, nm)) <= 1e-6, nm
    with pytest.raises(ValueError):
        sim.grid.set_static(alpha[:-1], kf, mf)
