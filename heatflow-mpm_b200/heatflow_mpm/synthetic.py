"""Synthetic scenes with the shapes, sizes and value distributions of the benchmark workloads (no dataset is involved).

* ``ellipsoid_particles`` -- a jittered particle lattice filling an ellipsoid that rests on the floor at the box
  centre, built like the reference's mesh fill (shapes.py:33-51: lattice from the bounding box grown by one spacing,
  uniform jitter of +-jitter*spacing, then shifted by (L/2, L/2, spacing/2)).
* ``coupled_default`` -- the default coupled 96^3 scene: h = 5 mm, trough heater 400 W capped at 120 C, fan 2 m/s,
  rods 300 C, room 25 C, a 10 cm tall ellipsoid (semi-axes 4/3/5 cm) of ~16k particles at 20 C with the melt law
  T_sol = 28 C, T_liq = 34 C.
* ``precision_study`` -- the precision-study scene: 160^3, h = 3 mm, trough heater 800 W capped at 120 C, fan 1 m/s,
  the default ellipsoid scaled to a footprint of ~5.8k cells (same 2.5 mm particle spacing), same melt law.
* ``plume_box`` -- the air-only plume scene: 32^3, h = 15 mm, box heater (4x4x2 rod cells on the floor at x = 0.1 m),
  400 W capped at 120 C, T = 25 C plus seeded uniform +-0.01 K noise, CG tolerances 1e-6.
"""
from __future__ import annotations

import numpy as np


def ellipsoid_particles(semi=(0.04, 0.03, 0.05), spacing=2.5e-3, L=0.48, seed=0, jitter=0.2) -> np.ndarray:
    semi = np.asarray(semi, float)
    rng = np.random.default_rng(seed)
    lo, hi = -semi - spacing, semi + spacing
    axes = [np.arange(lo[d] + spacing / 2, hi[d], spacing) for d in range(3)]
    P = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    P = P + rng.uniform(-jitter, jitter, P.shape) * spacing
    P = P[(((P / semi) ** 2).sum(1) <= 1.0)]
    P[:, 2] += semi[2]                    # lowest point on the floor
    return (P + np.array([L / 2, L / 2, spacing / 2])).astype(np.float32)


def coupled_default(device="cuda:0", body="frozen", seed=0, persistent_blocks=0, cg="classic"):
    from .grid import GridConfig
    from .heater import Heater
    from .mpm import Material
    from .solver import HeatflowMPM
    parts = ellipsoid_particles(seed=seed)
    mat = Material(t_sol=28.0, t_liq=34.0)
    heater = Heater(power=400.0, t_cap=120.0, fan=2.0, t_rod=300.0)
    grid = GridConfig(L=0.48, h=0.005, t_amb=25.0)
    return HeatflowMPM(parts, mat=mat, heater=heater, grid=grid, spacing=2.5e-3, t_init=20.0, device=device, body=body,
                       persistent_blocks=persistent_blocks, cg=cg)


PRECISION_FOOTPRINT = 5800     # cells covered by the precision-study body


def precision_particles(n=160, h=0.003, seed=0) -> np.ndarray:
    """The default ellipsoid (semi-axes 4/3/5 cm) scaled so that its volume covers PRECISION_FOOTPRINT cells of edge h."""
    semi = np.array([0.04, 0.03, 0.05])
    scale = (PRECISION_FOOTPRINT * h ** 3 / (4.0 / 3.0 * np.pi * semi.prod())) ** (1.0 / 3.0)
    return ellipsoid_particles(semi=tuple(semi * scale), spacing=2.5e-3, L=n * h, seed=seed)


def precision_build(n=160, h=0.003, seed=0):
    """(particles, Material, Heater, GridConfig) of the precision-study scene (no device work)."""
    from .grid import GridConfig
    from .heater import Heater
    from .mpm import Material
    return (precision_particles(n, h, seed), Material(t_sol=28.0, t_liq=34.0),
            Heater(power=800.0, t_cap=120.0, fan=1.0, t_rod=300.0), GridConfig(L=n * h, h=h, t_amb=25.0))


def precision_study(device="cuda:0", body="frozen", seed=0, n=160, h=0.003):
    from .solver import HeatflowMPM
    parts, mat, heater, grid = precision_build(n, h, seed)
    return HeatflowMPM(parts, mat=mat, heater=heater, grid=grid, spacing=2.5e-3, t_init=20.0, device=device, body=body)


def plume_box(device="cuda:0", seed=0):
    from .grid import GridConfig
    from .heater import BoxHeater
    from .solver import HeatflowMPM
    grid = GridConfig(L=0.48, h=0.015, cg_tol=1e-6)
    sim = HeatflowMPM(np.zeros((0, 3), np.float32), heater=BoxHeater(x=0.10, power=400.0, t_cap=120.0), grid=grid,
                      device=device)
    n = sim.grid.n
    rng = np.random.default_rng(seed)
    T = (25.0 + rng.uniform(-0.01, 0.01, (n, n, n))).astype(np.float32)
    sim.scene.set_current("T", T)
    sim.scene.apply_fixed_to_T()
    return sim
