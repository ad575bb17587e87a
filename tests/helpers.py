"""Shared test helpers: build GPU scenes and oracle scenes from the same inputs."""
from __future__ import annotations

import numpy as np


def spec_from_fixture(fx):
    """SceneSpec of a tests/golden/substep_*.npz fixture (the reference's own inputs)."""
    from heatflow_mpm.scene import SceneSpec
    n = int(fx["n"])
    P = fx["in_pos"].shape[0] if "in_pos" in fx else 0
    return SceneSpec(n=n, h=float(fx["h"]), rho=float(fx["rho"]), t_amb=float(fx["t_amb"]),
                     alpha_f_min=float(fx["alpha_f_min"]), buoyancy=bool(fx["buoyancy"]), cg_tol=float(fx["cg_tol"]),
                     cg_max_iter=int(fx["cg_max_iter"]), kappa_air=float(fx["kappa_air"]), kappa_mat=float(fx["kappa_mat"]),
                     fixed=fx["fixed"] == 1, tfix=fx["tfix"], source=fx["src"] == 1, rate=float(fx["rate"]),
                     t_cap=float(fx["t_cap"]), static_alpha=fx["static_alpha"],
                     static_k=[fx[f"static_k{a}"] for a in range(3)], static_m=[fx[f"static_m{a}"] for a in range(3)],
                     n_particles=P, spacing=float(fx["spacing"]), t_sol=float(fx["t_sol"]), t_liq=float(fx["t_liq"]),
                     y_solid=float(fx["yield_solid"]), mu_s=float(fx["mu_s"]), mu_l=float(fx["mu_l"]),
                     t_max=float(fx["t_max"]))


def device_scene_from_fixture(fx, device="cuda:0"):
    import torch
    from heatflow_mpm.scene import DeviceScene
    spec = spec_from_fixture(fx)
    sc = DeviceScene(spec, device)
    sc.set_current("T", fx["in_T"])
    sc.set_current("u", fx["in_u"])
    sc.set_current("v", fx["in_v"])
    sc.set_current("w", fx["in_w"])
    if spec.n_particles:
        sc.pos.copy_(torch.as_tensor(fx["in_pos"], device=device))
        sc.pvel.copy_(torch.as_tensor(fx["in_pvel"], device=device))
        sc.ptemp.copy_(torch.as_tensor(fx["in_ptemp"], device=device))
        sc.pyield.fill_(float(fx["yield_solid"]))
        sc.pvisc.fill_(float(fx["mu_s"]))
    return sc


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def random_scene_inputs(n, seed, heater_kw=None, L=None, particles=0):
    """A scene of edge n with the reference trough heater scaled into the box, random T and velocities."""
    from heatflow_mpm.heater import Heater
    from heatflow_mpm.solver import wall_fixed
    from heatflow_mpm.scene import SceneSpec
    rng = np.random.default_rng(seed)
    L = L or 0.48
    h = L / n
    kw = dict(power=400.0, t_cap=120.0, fan=2.0)
    kw.update(heater_kw or {})
    heater = Heater(**kw)
    cell, solid, source, rate, kf, mf, geom = heater.masks(n, h, (L / 2, L / 2), 1.2)
    fixed, tfix = wall_fixed(n, cell, heater.t_rod, 25.0)
    spec = SceneSpec(n=n, h=h, fixed=fixed, tfix=tfix, source=source, rate=rate, t_cap=heater.t_cap,
                     static_alpha=solid.astype(np.float32), static_k=kf, static_m=mf)
    T0 = (25.0 + rng.uniform(-2.0, 2.0, (n, n, n))).astype(np.float32)
    uvw = [rng.uniform(-0.3, 0.3, s).astype(np.float32) for s in ((n + 1, n, n), (n, n + 1, n), (n, n, n + 1))]
    return spec, T0, uvw


def oracle_from_spec(spec, precision="f32", mean_mode=0, scatter_mode=0, particles=None, pvel=None, ptemp=None):
    from oracle import oracle as O
    return O.scene_from_spec(spec, precision, mean_mode, scatter_mode, particles, pvel, ptemp)


def coupled_default_oracle(precision="f32"):
    """The default coupled 96^3 scene (heatflow_mpm.synthetic.coupled_default) on the CPU oracle, in the build's
    arithmetic (fp64 rhs mean, fixed-point particle sums): the same spec, particles, velocities and temperatures."""
    from heatflow_mpm.grid import GridConfig
    from heatflow_mpm.heater import Heater
    from heatflow_mpm.mpm import Material
    from heatflow_mpm.solver import KAPPA_AIR, build_spec
    from heatflow_mpm.synthetic import ellipsoid_particles
    from oracle import oracle as O
    parts = ellipsoid_particles(seed=0)
    spec, _, _, _ = build_spec(parts, Material(t_sol=28.0, t_liq=34.0), Heater(power=400.0, t_cap=120.0, fan=2.0),
                               GridConfig(L=0.48, h=0.005, t_amb=25.0), 2.5e-3, 20.0, KAPPA_AIR)
    return O.scene_from_spec(spec, precision, mean_mode=0, scatter_mode=0, particles=parts,
                             pvel=np.zeros_like(parts), ptemp=np.full(len(parts), 20.0, np.float32))
