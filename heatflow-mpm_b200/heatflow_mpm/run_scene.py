"""Melt a body of thermal material in front of an electric heater; write frames (the reference's
scripts/run_scene.py:14-44 on this package: same arguments, defaults and output files).

    python -m heatflow_mpm.run_scene --out data/bunny_fan --fan 2.0 --power 400

Output: static.npz, meta.json, frames/frame_NNNN.npz (pos, vel, temp f16, melt f16, grid_T f16 [n^3], air_u f16
[n^3, 3]).  Frames are packed on the device and written by FrameWriter while the substeps continue.

The body: ``--mesh`` names a Wavefront OBJ file, filled as shapes.py:47-51 fills it (jittered lattice, inside test by
the generalized winding number on the GPU); the default is the reference's bunny when $HEATFLOW_ASSETS/bunny.obj
exists (the mesh is not shipped), otherwise ``ellipsoid``: the 4/3/5 cm ellipsoid scaled to ``--height``.  A ``.npy``
file is taken as particle positions.  The material solver is Newton's implicit MPM when it is installed, otherwise
``--body frozen`` keeps the particles in place.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np


def body_particles(a) -> np.ndarray:
    from .synthetic import ellipsoid_particles
    if a.mesh == "ellipsoid":
        semi = np.array([0.04, 0.03, 0.05]) * (a.height / 0.10)
        P = ellipsoid_particles(semi=tuple(semi), spacing=a.spacing, L=a.L, seed=a.seed)
        if a.yaw:
            c = np.array([a.L / 2, a.L / 2, 0.0], np.float32)
            th = np.deg2rad(a.yaw)
            R = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]], np.float32)
            P = ((P - c) @ R.T + c).astype(np.float32)
        return P
    if a.mesh.endswith(".npy"):
        return np.load(a.mesh).astype(np.float32)
    if not os.path.exists(a.mesh):
        raise SystemExit(f"--mesh {a.mesh}: no such file (give an OBJ mesh, a .npy of particle positions or 'ellipsoid')")
    from .shapes import mesh_particles
    return mesh_particles(a.mesh, a.height, a.spacing, a.L, a.seed, a.yaw, a.device)


def _default_mesh() -> str:
    from .shapes import BUNNY
    return BUNNY if os.path.exists(BUNNY) else "ellipsoid"


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--seconds", type=float, default=20.0)
    ap.add_argument("--frame-dt", type=float, default=0.02)
    ap.add_argument("--dt", type=float, default=2e-3)
    ap.add_argument("--mesh", default=_default_mesh())
    ap.add_argument("--height", type=float, default=0.10)
    ap.add_argument("--yaw", type=float, default=0.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--spacing", type=float, default=2.5e-3)
    ap.add_argument("--L", type=float, default=0.48)
    ap.add_argument("--h", type=float, default=0.005)
    ap.add_argument("--t-amb", type=float, default=25.0)
    ap.add_argument("--t-init", type=float, default=20.0)
    ap.add_argument("--power", type=float, default=400.0)
    ap.add_argument("--t-cap", type=float, default=120.0)
    ap.add_argument("--t-rod", type=float, default=300.0)
    ap.add_argument("--fan", type=float, default=0.0)
    ap.add_argument("--heater-dist", type=float, default=0.21)
    ap.add_argument("--heater-z", type=float, default=0.12)
    ap.add_argument("--no-heater", action="store_true")
    ap.add_argument("--t-sol", type=float, default=30.0)
    ap.add_argument("--t-liq", type=float, default=36.0)
    ap.add_argument("--yield-solid", type=float, default=2e4)
    ap.add_argument("--viscosity-solid", type=float, default=5.0)
    ap.add_argument("--viscosity-liquid", type=float, default=30.0)
    ap.add_argument("--kappa", type=float, default=2e-5)
    ap.add_argument("--no-air-frames", action="store_true")
    ap.add_argument("--device", default="cuda:0")
    ap.add_argument("--body", default="auto", choices=["auto", "newton", "frozen"])
    return ap.parse_args(argv)


def main(argv=None):
    from .frames import FrameWriter
    from .grid import GridConfig
    from .heater import Heater
    from .mpm import Material
    from .solver import HeatflowMPM
    a = parse(argv)
    mat = Material(t_sol=a.t_sol, t_liq=a.t_liq, yield_solid=a.yield_solid, viscosity_solid=a.viscosity_solid,
                   viscosity_liquid=a.viscosity_liquid, kappa=a.kappa)
    heater = Heater(dist=a.heater_dist, z=a.heater_z, t_rod=a.t_rod, power=a.power, t_cap=a.t_cap, fan=a.fan,
                    on=not a.no_heater)
    P = body_particles(a)
    body = a.body
    if body == "auto":
        try:
            import newton  # noqa: F401
            body = "newton"
        except ImportError:
            body = "frozen"
    sim = HeatflowMPM(P, mat, heater, GridConfig(L=a.L, h=a.h, t_amb=a.t_amb), a.spacing, a.t_init, device=a.device,
                      body=body)
    os.makedirs(f"{a.out}/frames", exist_ok=True)
    np.savez(f"{a.out}/static.npz", **sim.static_dict())
    meta = vars(a) | dict(n_particles=int(len(P)), heater=sim.heater_geom, body=body)
    json.dump(meta, open(f"{a.out}/meta.json", "w"), indent=1)
    sub, nf, t0 = int(round(a.frame_dt / a.dt)), int(round(a.seconds / a.frame_dt)), time.time()
    writer = FrameWriter(sim, f"{a.out}/frames")
    writer.write(0, 0.0, not a.no_air_frames)
    print(f"{len(P)} particles, grid {sim.grid.n}^3, body {body}", flush=True)
    for k in range(1, nf + 1):
        for _ in range(sub):
            sim.substep(a.dt)
        writer.write(k, k * a.frame_dt, not a.no_air_frames)
        if k % 50 == 0 or k == nf:
            x, f, T = sim.positions(), sim.melt_fraction(), sim.grid_T()
            c = sim.grid.n // 2
            top = x[:, 2].max() if len(x) else 0.0
            print(f"t {k * a.frame_dt:5.1f} s | height {top * 100:4.1f} cm | melted {100 * (f >= 1).mean() if len(f) else 0.0:5.1f} % | "
                  f"air above the material {T[c, c, min(int(top / a.h) + 1, sim.grid.n - 1)]:5.1f} C | "
                  f"{(time.time() - t0) / k:.3f} s/frame", flush=True)
    writer.close()
    print("done", a.out)


if __name__ == "__main__":
    main()
