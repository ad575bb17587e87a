"""The CPU oracle against the reference's own golden vectors (tests/golden, made by make_golden.py).

Per-kernel fixtures: every air-path Warp kernel of the reference, run through the Warp-semantics emulation on seeded
inputs; the oracle must be bit-exact.  Substep fixtures: whole reference substeps (air-only, fan, coupled with a
frozen body, erfc setup); the oracle in reference mode (numpy float32 mean, sequential particle scatter) must be
bit-exact, and in the build's deterministic mode (fp64 mean, fixed-point scatter) within 1e-6 relative L2 for T and
the face velocities.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

KER = golden("kernels.npz")
N, H, DT = int(KER["n"]), float(KER["h"]), float(KER["dt"])
FS = O.face_shapes(N)
VEL = [KER[f"in_vel{a}"] for a in range(3)]


def _run(name, *args, out_shape=None, out=None):
    K = O.Kernels("f32")
    o = np.zeros(out_shape, np.float32) if out is None else out
    K.call(name, *args, o) if out is None else K.call(name, *args)
    return o


def _exact(got, ref):
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), f"max diff {np.abs(got.astype(np.float64) - ref).max():.3g}"


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_face_kernels_bit_exact(axis):
    K = O.Kernels("f32")
    o = np.zeros(FS[axis], np.float32)
    K.call("or_advect_face", N, H, DT, VEL[0], VEL[1], VEL[2], axis, VEL[axis], o)
    _exact(o, KER[f"advect_face{axis}"])
    o = np.zeros(FS[axis], np.float32)
    K.call("or_face_fraction", N, KER["in_alpha_s"], axis, 0.05, o)
    _exact(o, KER[f"face_fraction{axis}"])
    q = KER[f"in_q{axis}"].copy()
    K.call("or_zero_wall", N, axis, q)
    _exact(q, KER[f"zero_wall{axis}"])
    q = VEL[axis].copy()
    K.call("or_relax", N, H, DT, 1.2, 0.05, axis, q, KER[f"in_kf{axis}"], KER[f"in_mf{axis}"], KER[f"in_af{axis}"])
    _exact(q, KER[f"relax{axis}"])
    q = VEL[axis].copy()
    K.call("or_project", N, H, DT / 1.2, axis, q, KER["in_p"])
    _exact(q, KER[f"project{axis}"])


def test_cell_kernels_bit_exact():
    K = O.Kernels("f32")
    af = [KER[f"face_fraction{a}"] for a in range(3)]
    qd = [KER[f"in_qdiv{a}"] for a in range(3)]
    o = np.zeros((N, N, N), np.float32)
    K.call("or_advect_T", N, H, DT, KER["in_T"], KER["in_alpha_s"], *VEL, o)
    _exact(o, KER["advect_T"])
    w = VEL[2].copy()
    K.call("or_buoyancy", N, DT, 9.81, 25.0, w, KER["in_T"])
    _exact(w, KER["buoyancy_w"])
    o = np.zeros((N, N, N), np.float32)
    K.call("or_divergence_rhs", N, H, 1.2 / DT, *VEL, *af, *qd, o)
    _exact(o, KER["divergence_rhs"])
    o = np.zeros(N ** 3, np.float32)
    K.call("or_laplacian", N, H, 0.75, -0.5, KER["in_p"], *af, KER["in_y"], o)
    _exact(o, KER["laplacian"])
    o = np.zeros(N ** 3, np.float32)
    K.call("or_jacobi", N, H, *af, o)
    _exact(o, KER["jacobi"])
    o = np.zeros((N ** 3, 3), np.float32)
    K.call("or_cell_velocity", N, *VEL, o)
    _exact(o, KER["cell_velocity"])


def test_heat_kernels_bit_exact():
    K = O.Kernels("f32")
    kap = np.zeros((N, N, N), np.float32)
    K.call("or_conductivity", N, 2.2e-5, 2.0e-5 * 40.0, KER["in_alpha_s"], kap)
    _exact(kap, KER["conductivity"])
    fixed, tfix = KER["in_fixed"], KER["in_tfix"]
    o = np.zeros(N ** 3, np.float32)
    K.call("or_heat_rhs", N, H, DT, KER["in_T"], kap, fixed, tfix, KER["in_x"], o)
    _exact(o, KER["heat_rhs"])
    o = np.zeros(N ** 3, np.float32)
    K.call("or_heat_diag", N, H, DT, kap, fixed, o)
    _exact(o, KER["heat_diag"])
    o = np.zeros(N ** 3, np.float32)
    K.call("or_heat_matvec", N, H, DT, -1.0, 1.0, KER["in_x"], kap, fixed, tfix, KER["in_y"], o)
    _exact(o, KER["heat_matvec"])
    o = np.zeros((N, N, N), np.float32)
    K.call("or_blend", N, KER["in_T"], KER["in_alpha"], KER["in_tsum"], o)
    _exact(o, KER["blend"])
    T = KER["in_T"].copy()
    K.call("or_apply_fixed", N, T, fixed, tfix)
    _exact(T, KER["apply_fixed"])
    T = KER["in_T"].copy()
    K.call("or_source", N, T, KER["in_src"], 9000.0, 70.0, DT)
    _exact(T, KER["source"])


@pytest.mark.parametrize("mode", [1, 0])
def test_particle_kernels(mode):
    """mode 1 (sequential binary32, the reference's order run serially): bit-exact.  mode 0 (fixed-point, the build):
    within 4 binary32 ulps of the largest contribution of each lattice."""
    K = O.Kernels("f32")
    P = KER["in_pos"].shape[0]
    outs = [np.zeros((N, N, N), np.float32)] + [np.zeros(FS[a % 3], np.float32) for a in range(9)] + \
           [np.zeros((N, N, N), np.float32) for _ in range(2)]
    acc = np.zeros(12 * (N + 1) ** 3, np.int64)
    K.call("or_scatter", N, P, H, float(KER["vol"]), 1.0e-3, KER["in_pos"], KER["in_pvel"], KER["in_ptemp"], *outs, mode, acc)
    names = ["alpha_s", "qx", "qy", "qz", "kx", "ky", "kz", "mx", "my", "mz"]
    refs = [KER["scatter_" + nm] for nm in names] + [KER["scatter_heat_alpha"], KER["scatter_heat_tsum"]]
    for got, ref in zip(outs, refs):
        if mode == 1:
            _exact(got, ref)
        else:
            tol = 4 * np.spacing(np.float32(np.abs(ref).max()))
            assert np.abs(got.astype(np.float64) - ref).max() <= tol
    assert not acc.any(), "fixed-point accumulators must be left cleared"
    tp = KER["in_ptemp"].copy()
    melt, ys, vs = (np.zeros(P, np.float32) for _ in range(3))
    K.call("or_particle_update", N, P, H, KER["in_pos"], KER["in_Tbefore"], KER["in_Tafter"], 28.0, 34.0, 2.0e4, 5.0, 30.0,
           35.0, tp, melt, ys, vs)
    for got, nm in ((tp, "temp"), (melt, "melt"), (ys, "yield"), (vs, "visc")):
        _exact(got, KER["pupd_" + nm])


SUBSTEPS = ["substep_air_n12", "substep_fan_n12", "substep_coupled_n12", "substep_erfc_n10"]


@pytest.mark.parametrize("name", SUBSTEPS)
def test_substep_reference_mode_bit_exact(name):
    fx = golden(name + ".npz")
    sc = O.scene_from_fixture(fx, "f32", mean_mode=1, scatter_mode=1)
    for s in range(int(fx["nsub"])):
        sc.substep(float(fx["dt"]))
        for nm, got in (("T", sc.T), ("u", sc.u), ("v", sc.v), ("w", sc.w), ("p", sc.p)):
            _exact(got, fx[f"{nm}_{s}"])
        st, cg = sc.stats(), fx[f"cglog_{s}"]
        assert (st["heat_done"], st["heat_iters"]) == tuple(cg[0, :2].astype(int))
        assert (st["grid_done"], st["grid_iters"]) == tuple(cg[1, :2].astype(int))
        if "ptemp_0" in fx:
            pt = sc.particles()
            _exact(pt["temp"], fx[f"ptemp_{s}"])
            _exact(pt["melt"], fx[f"pmelt_{s}"])


@pytest.mark.parametrize("name", SUBSTEPS)
def test_substep_build_mode_close(name):
    fx = golden(name + ".npz")
    sc = O.scene_from_fixture(fx, "f32", mean_mode=0, scatter_mode=0)
    for s in range(int(fx["nsub"])):
        sc.substep(float(fx["dt"]))
        for nm, got in (("T", sc.T), ("u", sc.u), ("v", sc.v), ("w", sc.w)):
            ref = fx[f"{nm}_{s}"].astype(np.float64)
            rel = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
            assert rel < 1e-6, (nm, s, rel)


def test_fixture_diagnostics():
    fx = golden("substep_air_n12.npz")
    sc = O.scene_from_fixture(fx, "f32", mean_mode=1, scatter_mode=1)
    for _ in range(int(fx["nsub"])):
        sc.substep(float(fx["dt"]))
    assert np.array_equal(sc.cell_velocity(), fx["air_velocity"])
    assert sc.divergence_max() == pytest.approx(float(fx["divergence_max"]), rel=1e-6)
    assert sc.speed_max() == float(fx["speed_max"])


def test_numpy_mean_restatement():
    """or_mean(mode=1) is numpy's float32 pairwise mean (grid.py:239)."""
    rng = np.random.default_rng(3)
    L = O.lib("f32")
    import ctypes as C
    for n in (5, 9, 100, 128, 129, 1000, 1728, 4096, 32768, 100003):
        a = (rng.standard_normal(n) * 1000).astype(np.float32)
        got = L.or_mean(a.ctypes.data_as(C.c_void_p), n, 1)
        assert np.float32(got) == a.mean()
