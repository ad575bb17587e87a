"""Generate the golden vectors in tests/golden/ from the reference Heatflow-MPM checkout itself.

Run where a checkout of the reference exists (it is read at run time and does not travel with the tests):

    python tests/golden/make_golden.py --reference <path of the Heatflow-MPM checkout>

What it writes (all small, compressed .npz):
  * heater_*.npz  -- ``Heater.masks`` (heatflow_mpm/heater.py:33-65) outputs, produced by the reference module with
    numpy (bit-exact ground truth for cell flags, solid/source masks, source rate and static face weights);
  * kernels.npz   -- every air-path Warp kernel of the reference (grid.py, heat.py, solver.py:19-38) executed through
    ``warp_shim`` (Warp fp32 kernel semantics emulated on the CPU) on seeded random inputs at n = 7;
  * substep_*.npz -- whole ``HeatflowMPM.substep`` calls (solver.py:63-88) of the reference, air-only and coupled
    with a frozen particle body standing in for Newton, at n = 10..12 for a few substeps.

The generator never copies reference source into this repository; it imports the reference package at run time.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import warp_shim  # noqa: E402


def _load_reference(ref_root):
    warp_shim.install()
    sys.path.insert(0, ref_root)
    hm = importlib.import_module("heatflow_mpm")
    return hm


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ------------------------------------------------------------------------------------------------------ heater masks
HEATER_CASES = {
    # name: (L, h, Heater kwargs, store full arrays?)
    "heater_n32_fan0": (0.48, 0.015, dict(power=400.0, t_cap=120.0, fan=0.0), True),
    "heater_n32_fan2": (0.48, 0.015, dict(power=400.0, t_cap=120.0, fan=2.0), True),
    "heater_n96_fan0": (0.48, 0.005, dict(power=400.0, t_cap=120.0, fan=0.0), True),
    "heater_n96_fan2": (0.48, 0.005, dict(power=400.0, t_cap=120.0, fan=2.0), True),
    "heater_n48_misc": (0.48, 0.01, dict(dist=0.17, direction=(0.6, -0.8), z=0.09, tilt=25.0, radius=0.05, length=0.18,
                                          power=250.0, t_cap=90.0, fan=1.3), True),
    "heater_n160_fan1": (0.48, 0.003, dict(power=800.0, t_cap=120.0, fan=1.0), False),
    "heater_n12_small": (0.12, 0.01, dict(dist=0.035, z=0.04, radius=0.025, length=0.08, power=50.0, t_cap=120.0, fan=2.0), True),
    "heater_n60_off": (0.30, 0.005, dict(on=False), False),
}


def make_heater(hm, out):
    for name, (L, h, kw, full) in HEATER_CASES.items():
        heater = hm.Heater(**kw)
        n = int(round(L / h))
        cell, solid, source, rate, kf, mf, geom = heater.masks(n, h, (L / 2, L / 2), 1.2)
        d = dict(L=L, h=h, n=n, rho=1.2, rate=np.float64(rate), counts=np.bincount(cell.ravel(), minlength=5),
                 centre=np.array(geom["centre"]), facing=np.array(geom["facing"]), axis=np.array(geom["axis"]),
                 up=np.array(geom["up"]), kwargs=np.array(repr(kw)))
        arrays = dict(cell=cell.astype(np.int8), solid=solid, source=source, kx=kf[0], ky=kf[1], kz=kf[2],
                      mx=mf[0], my=mf[1], mz=mf[2])
        for k, v in arrays.items():
            d["sha_" + k] = np.array(_sha(v))
            if full:
                d[k] = v
        np.savez_compressed(os.path.join(out, name + ".npz"), **d)
        print(name, n, d["counts"], rate)


# ---------------------------------------------------------------------------------------------- per-kernel fixtures
def make_kernels(hm, out, n=7, seed=7):
    wp = sys.modules["warp"]
    grid = importlib.import_module("heatflow_mpm.grid")
    heat = importlib.import_module("heatflow_mpm.heat")
    solver = importlib.import_module("heatflow_mpm.solver")
    rng = np.random.default_rng(seed)
    F = np.float32
    h, dt = 0.011, 2.0e-3
    fshape = [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)]
    R = lambda shape, lo=-1.0, hi=1.0: rng.uniform(lo, hi, shape).astype(F)
    A = lambda a, dtype=float: wp.array(a, dtype=dtype)
    res = dict(n=n, h=h, dt=dt)

    # velocities with magnitude large enough that back-traces cross cells and leave the box
    uvw = [R(s, -4.0, 4.0) for s in fshape]
    for ax_ in range(3):
        res[f"in_vel{ax_}"] = uvw[ax_]
    # advect faces
    for axis in range(3):
        q = A(uvw[axis]); o = wp.zeros(fshape[axis])
        wp.launch(grid.k_advect_face, dim=fshape[axis], inputs=[q, A(uvw[0]), A(uvw[1]), A(uvw[2]), o, axis, h, n, dt])
        res[f"advect_face{axis}"] = o.numpy().copy()
    # temperature advection
    T = R((n, n, n), 20.0, 80.0); alpha_s = R((n, n, n), 0.0, 1.0)
    res["in_T"], res["in_alpha_s"] = T, alpha_s
    o = wp.zeros((n, n, n))
    wp.launch(heat.k_advect, dim=(n, n, n), inputs=[A(T), A(alpha_s), A(uvw[0]), A(uvw[1]), A(uvw[2]), o, h, n, dt])
    res["advect_T"] = o.numpy().copy()
    # buoyancy
    w = A(uvw[2])
    wp.launch(grid.k_buoyancy, dim=(n, n, n + 1), inputs=[w, A(T), n, dt, 9.81, 25.0])
    res["buoyancy_w"] = w.numpy().copy()
    # face fraction / zero wall / relax
    for axis in range(3):
        af = wp.zeros(fshape[axis])
        wp.launch(grid.k_face_fraction, dim=fshape[axis], inputs=[A(alpha_s), af, axis, n, 0.05])
        res[f"face_fraction{axis}"] = af.numpy().copy()
        q = A(R(fshape[axis]))
        res[f"in_q{axis}"] = q.numpy().copy()
        wp.launch(grid.k_zero_wall, dim=fshape[axis], inputs=[q, axis, n])
        res[f"zero_wall{axis}"] = q.numpy().copy()
        kf = R(fshape[axis], 0.0, 1.0); mf = R(fshape[axis], -0.5, 0.5); afr = R(fshape[axis], 0.0, 1.0)
        res[f"in_kf{axis}"], res[f"in_mf{axis}"], res[f"in_af{axis}"] = kf, mf, afr
        qq = A(uvw[axis])
        wp.launch(grid.k_relax, dim=fshape[axis], inputs=[qq, A(kf), A(mf), A(afr), axis, h, n, dt, 1.2, 0.05])
        res[f"relax{axis}"] = qq.numpy().copy()
    # divergence rhs, laplacian, jacobi, project, cell velocity
    afs = [res[f"face_fraction{a}"] for a in range(3)]
    qs = [R(s, -0.1, 0.1) for s in fshape]
    for a in range(3):
        res[f"in_qdiv{a}"] = qs[a]
    rhs = wp.zeros((n, n, n))
    wp.launch(grid.k_divergence_rhs, dim=(n, n, n), inputs=[A(uvw[0]), A(uvw[1]), A(uvw[2]), A(afs[0]), A(afs[1]), A(afs[2]),
                                                            A(qs[0]), A(qs[1]), A(qs[2]), rhs, h, 1.2 / dt])
    res["divergence_rhs"] = rhs.numpy().copy()
    p = R(n ** 3, -5.0, 5.0); y = R(n ** 3)
    res["in_p"], res["in_y"] = p, y
    o = wp.zeros(n ** 3)
    wp.launch(grid.k_laplacian, dim=n ** 3, inputs=[A(p), A(afs[0]), A(afs[1]), A(afs[2]), o, A(y), 0.75, -0.5, h, n])
    res["laplacian"] = o.numpy().copy()
    d = wp.zeros(n ** 3)
    wp.launch(grid.k_jacobi, dim=n ** 3, inputs=[A(afs[0]), A(afs[1]), A(afs[2]), d, h, n])
    res["jacobi"] = d.numpy().copy()
    for axis in range(3):
        q = A(uvw[axis])
        wp.launch(grid.k_project, dim=fshape[axis], inputs=[q, A(p.reshape(n, n, n)), axis, h, n, dt / 1.2])
        res[f"project{axis}"] = q.numpy().copy()
    cv = wp.zeros(n ** 3, dtype=wp.vec3)
    wp.launch(grid.k_cell_velocity, dim=n ** 3, inputs=[A(uvw[0]), A(uvw[1]), A(uvw[2]), cv, n])
    res["cell_velocity"] = cv.numpy().copy()
    # heat: conductivity, rhs, diag, matvec, blend, fixed, source
    kap = wp.zeros((n, n, n))
    wp.launch(heat.k_conductivity, dim=(n, n, n), inputs=[A(alpha_s), kap, 2.2e-5, 2.0e-5 * 40.0])
    res["conductivity"] = kap.numpy().copy()
    fixed = (rng.uniform(0, 1, (n, n, n)) < 0.2).astype(np.int32); tfix = R((n, n, n), 0.0, 300.0)
    res["in_fixed"], res["in_tfix"] = fixed, tfix
    x = R(n ** 3, 10.0, 60.0)
    res["in_x"] = x
    hrhs = wp.zeros(n ** 3)
    wp.launch(heat.k_heat_rhs, dim=n ** 3, inputs=[A(T), kap, A(fixed, int), A(tfix), A(x), hrhs, h, n, dt])
    res["heat_rhs"] = hrhs.numpy().copy()
    hd = wp.zeros(n ** 3)
    wp.launch(heat.k_heat_diag, dim=n ** 3, inputs=[kap, A(fixed, int), hd, h, n, dt])
    res["heat_diag"] = hd.numpy().copy()
    o = wp.zeros(n ** 3)
    wp.launch(heat.k_heat_matvec, dim=n ** 3, inputs=[A(x), kap, A(fixed, int), A(tfix), o, A(y), -1.0, 1.0, h, n, dt])
    res["heat_matvec"] = o.numpy().copy()
    alpha = R((n, n, n), 0.0, 0.2); tsum = R((n, n, n), 0.0, 10.0)
    res["in_alpha"], res["in_tsum"] = alpha, tsum
    o = wp.zeros((n, n, n))
    wp.launch(heat.k_blend, dim=(n, n, n), inputs=[A(T), A(alpha), A(tsum), o])
    res["blend"] = o.numpy().copy()
    Tf = A(T)
    wp.launch(heat.k_apply_fixed, dim=(n, n, n), inputs=[Tf, A(fixed, int), A(tfix)])
    res["apply_fixed"] = Tf.numpy().copy()
    src = (rng.uniform(0, 1, (n, n, n)) < 0.3).astype(np.int32)
    res["in_src"] = src
    Ts = A(T)
    wp.launch(heat.k_source, dim=(n, n, n), inputs=[Ts, A(src, int), 9000.0, 70.0, dt])
    res["source"] = Ts.numpy().copy()
    # particles: scatter and FLIP update
    P = 40
    pos = rng.uniform(-0.5 * h, (n + 0.5) * h, (P, 3)).astype(F)
    vel = rng.uniform(-1.0, 1.0, (P, 3)).astype(F)
    temp = rng.uniform(15.0, 40.0, P).astype(F)
    res["in_pos"], res["in_pvel"], res["in_ptemp"] = pos, vel, temp
    vol = 0.5 * h ** 3 * 0.3
    res["vol"] = vol
    outs = [wp.zeros((n, n, n))] + [wp.zeros(s) for s in fshape] * 3
    outs = [wp.zeros((n, n, n))] + [wp.zeros(fshape[a % 3]) for a in range(9)]
    wp.launch(solver.k_scatter_particles, dim=P, inputs=[A(pos, wp.vec3), A(vel, wp.vec3), vol, h, n, 1.0e-3] + outs)
    for name, o in zip(["alpha_s", "qx", "qy", "qz", "kx", "ky", "kz", "mx", "my", "mz"], outs):
        res["scatter_" + name] = o.numpy().copy()
    al, ts = wp.zeros((n, n, n)), wp.zeros((n, n, n))
    wp.launch(heat.k_scatter_heat, dim=P, inputs=[A(pos, wp.vec3), A(temp), vol, h, n, al, ts])
    res["scatter_heat_alpha"], res["scatter_heat_tsum"] = al.numpy().copy(), ts.numpy().copy()
    Tb, Ta = R((n, n, n), 20.0, 40.0), R((n, n, n), 20.0, 40.0)
    res["in_Tbefore"], res["in_Tafter"] = Tb, Ta
    tp, melt, ys, vs = A(temp), wp.zeros(P), wp.zeros(P), wp.zeros(P)
    wp.launch(heat.k_particle_update, dim=P, inputs=[A(pos, wp.vec3), A(Tb), A(Ta), h, n, 28.0, 34.0, 2.0e4, 5.0, 30.0, 35.0,
                                                      tp, melt, ys, vs])
    res["pupd_temp"], res["pupd_melt"] = tp.numpy().copy(), melt.numpy().copy()
    res["pupd_yield"], res["pupd_visc"] = ys.numpy().copy(), vs.numpy().copy()
    np.savez_compressed(os.path.join(out, "kernels.npz"), **res)
    print("kernels.npz", len(res), "arrays")


# ------------------------------------------------------------------------------------------------- substep fixtures
class FrozenBody:
    """Stand-in for ThermalMPM (mpm.py:25-80) with Newton absent: particles keep their positions and velocities."""

    def __init__(self, particles, spacing, mat, device):
        wp = sys.modules["warp"]
        self.n = len(particles)
        self.pos = wp.array(np.asarray(particles, np.float32), dtype=wp.vec3)
        self.vel = wp.zeros(self.n, dtype=wp.vec3)
        self.yield_stress = wp.full(self.n, mat.yield_solid)
        self.viscosity = wp.full(self.n, mat.viscosity_solid)

    def step(self, dt):
        pass

    def positions(self):
        return self.pos.numpy().copy()

    def velocities(self):
        return self.vel.numpy().copy()


SUBSTEP_CASES = {
    # name: (GridConfig kwargs, Heater kwargs, particles?, kappa_air, n_substeps, seed, fixed-floor erfc setup?)
    "substep_air_n12": (dict(L=0.12, h=0.01, cg_tol=1e-6), dict(dist=0.035, z=0.04, radius=0.025, length=0.08, power=50.0,
                                                                  t_cap=120.0, fan=0.0), False, 2.2e-5, 3, 11, False),
    "substep_fan_n12": (dict(L=0.12, h=0.01, cg_tol=1e-4), dict(dist=0.035, z=0.04, radius=0.025, length=0.08, power=50.0,
                                                                  t_cap=120.0, fan=2.0), False, 2.2e-5, 3, 12, False),
    "substep_coupled_n12": (dict(L=0.12, h=0.01, cg_tol=1e-5), dict(dist=0.035, z=0.04, radius=0.025, length=0.08, power=50.0,
                                                                      t_cap=120.0, fan=2.0), True, 2.2e-5, 2, 13, False),
    "substep_erfc_n10": (dict(L=0.10, h=0.01, buoyancy=False), dict(on=False), False, 1.0e-3, 3, 14, True),
}


def _ellipsoid_particles(rng, centre, semi, spacing):
    axes = [np.arange(centre[d] - semi[d], centre[d] + semi[d] + 1e-9, spacing) for d in range(3)]
    P = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    P = P + rng.uniform(-0.2, 0.2, P.shape) * spacing
    r = ((P - centre) / semi) ** 2
    return P[r.sum(1) <= 1.0].astype(np.float32)


def make_substeps(hm, out, only=None):
    solver = importlib.import_module("heatflow_mpm.solver")
    solver.ThermalMPM = FrozenBody
    for name, (gkw, hkw, with_particles, kappa_air, nsub, seed, erfc) in SUBSTEP_CASES.items():
        if only and name not in only:
            continue
        rng = np.random.default_rng(seed)
        gcfg = hm.GridConfig(**gkw)
        mat = hm.Material(t_sol=28.0, t_liq=34.0)
        parts = np.zeros((0, 3), np.float32)
        if with_particles:
            parts = _ellipsoid_particles(rng, np.array([gcfg.L / 2, gcfg.L / 2, 0.02]), np.array([0.015, 0.012, 0.018]), 0.005)
        sim = hm.HeatflowMPM(parts, mat=mat, heater=hm.Heater(**hkw), grid=gcfg, spacing=0.005, t_init=20.0,
                             kappa_air=kappa_air, device="cpu")
        n = sim.grid.n
        if erfc:
            fixed = np.zeros((n, n, n), bool)
            fixed[:, :, 0] = True
            sim.heat.set_fixed(fixed, np.where(fixed, 70.0, 0.0))
        d = dict(n=n, L=gcfg.L, h=gcfg.h, rho=gcfg.rho, t_amb=gcfg.t_amb, buoyancy=gcfg.buoyancy, alpha_f_min=gcfg.alpha_f_min,
                 cg_tol=gcfg.cg_tol, cg_max_iter=gcfg.cg_max_iter, kappa_air=kappa_air, kappa_mat=mat.kappa,
                 heater=np.array(repr(hkw)), erfc=erfc, dt=2.0e-3, nsub=nsub, spacing=0.005, t_init=20.0,
                 t_sol=mat.t_sol, t_liq=mat.t_liq, yield_solid=mat.yield_solid, mu_s=mat.viscosity_solid,
                 mu_l=mat.viscosity_liquid, t_max=sim.t_max)
        # seeded initial state (written after construction, as the reference initialises T to t_amb)
        if not erfc:
            for a in ("u", "v", "w"):
                arr = getattr(sim.grid, a).numpy()
                arr[...] = rng.uniform(-0.3, 0.3, arr.shape).astype(np.float32)
            T = sim.heat.T.numpy()
            T[...] = (25.0 + rng.uniform(-3.0, 3.0, T.shape)).astype(np.float32)
        if with_particles:
            sim.body.vel.numpy()[...] = rng.uniform(-0.2, 0.2, sim.body.vel.numpy().shape).astype(np.float32)
            sim.temp.numpy()[...] = rng.uniform(18.0, 36.0, sim.n).astype(np.float32)
            d["in_pos"] = sim.body.pos.numpy().copy()
            d["in_pvel"] = sim.body.vel.numpy().copy()
        d["in_u"], d["in_v"], d["in_w"] = (getattr(sim.grid, a).numpy().copy() for a in ("u", "v", "w"))
        d["in_T"] = sim.heat.T.numpy().copy()
        d["in_ptemp"] = sim.temp.numpy()[: sim.n].copy()
        d["fixed"] = sim.heat.fixed.numpy().copy()
        d["tfix"] = sim.heat.tfix.numpy().copy()
        d["src"] = sim.heat.src.numpy().copy()
        d["rate"] = np.float64(sim.heat.rate)
        d["t_cap"] = np.float64(sim.heat.t_cap)
        st = sim.grid.static
        d["static_alpha"] = st[0].numpy().copy()
        for a in range(3):
            d[f"static_k{a}"] = st[1][a].numpy().copy()
            d[f"static_m{a}"] = st[2][a].numpy().copy()
        for s in range(nsub):
            warp_shim.CG_LOG.clear()
            sim.substep(2.0e-3)
            d[f"T_{s}"] = sim.heat.T.numpy().copy()
            d[f"u_{s}"], d[f"v_{s}"], d[f"w_{s}"] = (getattr(sim.grid, a).numpy().copy() for a in ("u", "v", "w"))
            d[f"p_{s}"] = sim.grid.p.numpy().copy()
            d[f"cglog_{s}"] = np.array(warp_shim.CG_LOG, np.float64)   # rows: heat, pressure
            d[f"heat_iters_{s}"], d[f"grid_iters_{s}"] = sim.heat.cg_iters, sim.grid.cg_iters
            if with_particles:
                d[f"ptemp_{s}"] = sim.temp.numpy()[: sim.n].copy()
                d[f"pmelt_{s}"] = sim.melt.numpy()[: sim.n].copy()
                d[f"pyield_{s}"] = sim.body.yield_stress.numpy().copy()
                d[f"pvisc_{s}"] = sim.body.viscosity.numpy().copy()
                d[f"alpha_s_{s}"] = sim.grid.alpha_s.numpy().copy()
            print(name, "substep", s, "cg", warp_shim.CG_LOG, flush=True)
        d["air_velocity"] = sim.air_velocity()
        d["divergence_max"] = sim.grid.divergence_max()
        d["speed_max"] = sim.grid.speed_max()
        np.savez_compressed(os.path.join(out, name + ".npz"), **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the reference Heatflow-MPM checkout")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", nargs="*", default=None, help="heater | kernels | substep names")
    a = ap.parse_args()
    hm = _load_reference(a.reference)
    np.seterr(all="ignore")
    sel = set(a.only or ["heater", "kernels"] + list(SUBSTEP_CASES))
    if "heater" in sel:
        make_heater(hm, a.out)
    if "kernels" in sel:
        make_kernels(hm, a.out)
    chosen = [s for s in sel if s in SUBSTEP_CASES]
    if chosen:
        make_substeps(hm, a.out, only=chosen)


if __name__ == "__main__":
    main()
