"""GPU parity: libheatflow_b200 against the reference's golden vectors and the CPU oracle.

Tolerances (binary32 fields):
  * single kernels through the C ABI vs the reference kernels (golden): bit-exact;
  * whole substeps vs the oracle in the build's arithmetic (fp64 mean, fixed-point particle sums, fp64 CG scalars):
    relative L2 <= 1e-6 for T and the face velocities (the only difference is the summation order of fp64 dot products,
    which moves alpha/beta by ~1e-16 before they are rounded to binary32);
  * whole substeps vs the reference itself (golden): relative L2 <= 1e-5 (the reference sums the pressure rhs mean in
    float32 and the particle weights in float32 atomic order);
  * CG exits at ||r|| <= atol = max(tol ||b||, tol) in every solve (warp.optim.linear.cg's criterion).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden
from helpers import device_scene_from_fixture, oracle_from_spec, rel_l2, random_scene_inputs, spec_from_fixture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_kernels_bit_exact_vs_reference(torch_cuda):
    torch = torch_cuda
    from heatflow_mpm import _lib
    L = _lib.load()
    fx = golden("kernels.npz")
    n, h, dt = int(fx["n"]), float(fx["h"]), float(fx["dt"])
    D = lambda a, dt_=torch.float32: torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=dt_)
    af = [D(fx[f"face_fraction{a}"]) for a in range(3)]
    p, y = D(fx["in_p"]), D(fx["in_y"])
    out = torch.zeros(n ** 3, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.hf_k_laplacian(n, h, 0.75, -0.5, _ptr(p), _ptr(af[0]), _ptr(af[1]), _ptr(af[2]), _ptr(y), _ptr(out), s))
    assert np.array_equal(out.cpu().numpy(), fx["laplacian"])
    kap = D(fx["conductivity"])
    flags = D(fx["in_fixed"].astype(np.uint8), torch.uint8)
    x = D(fx["in_x"])
    _lib.check(L.hf_k_heat_matvec(n, h, dt, -1.0, 1.0, _ptr(x), _ptr(kap), _ptr(flags), _ptr(y), _ptr(out), s))
    assert np.array_equal(out.cpu().numpy(), fx["heat_matvec"])


FIXTURES = ["substep_air_n12", "substep_fan_n12", "substep_coupled_n12", "substep_erfc_n10"]


@pytest.mark.parametrize("name", FIXTURES)
def test_substeps_vs_reference_and_oracle(torch_cuda, name):
    from heatflow_mpm.scene import ScenePlan
    from oracle import oracle as O
    fx = golden(name + ".npz")
    sc = device_scene_from_fixture(fx)
    plan = ScenePlan([sc])
    plan.prepare_statics()
    orc = O.scene_from_fixture(fx, "f32", mean_mode=0, scatter_mode=0)
    for s in range(int(fx["nsub"])):
        plan.substep(float(fx["dt"]))
        orc.substep(float(fx["dt"]))
        st = sc.read_state()
        assert st.status == 0
        for nm, ref in (("T", fx[f"T_{s}"]), ("u", fx[f"u_{s}"]), ("v", fx[f"v_{s}"]), ("w", fx[f"w_{s}"])):
            got = sc.current(nm).cpu().numpy()
            assert rel_l2(got, getattr(orc, nm)) <= 1e-6, (nm, s, rel_l2(got, getattr(orc, nm)))
            assert rel_l2(got, ref) <= 1e-5, (nm, s, rel_l2(got, ref))
        assert st.pressure_rr <= st.pressure_atol ** 2 * (1 + 1e-12)
        assert st.heat_rr <= st.heat_atol ** 2 * (1 + 1e-12)
        # the reference reports warp's quantised counts; ours performs exactly the iterations until convergence
        cg = fx[f"cglog_{s}"]
        assert abs(st.heat_iters - int(cg[0, 0])) <= 1 and abs(st.pressure_iters - int(cg[1, 0])) <= 2
        if sc.spec.n_particles:
            assert rel_l2(sc.ptemp.cpu().numpy(), fx[f"ptemp_{s}"]) <= 1e-6
            assert np.allclose(sc.pmelt.cpu().numpy(), fx[f"pmelt_{s}"], atol=1e-5)


@pytest.mark.parametrize("cg", ["classic", "single-reduction"])
def test_larger_scene_vs_oracle(torch_cuda, cg):
    """n = 32 with the reference trough heater (fan on), pressure tolerance 1e-6 (~170 iterations), 4 substeps: GPU vs
    oracle (build arithmetic).  The single-reduction pressure solve takes beta from an expansion instead of a direct
    inner product (binary32 rounding of r differs by ~1e-7): relative L2 <= 1e-5 for it."""
    from heatflow_mpm.scene import DeviceScene, ScenePlan
    spec, T0, uvw = random_scene_inputs(32, seed=21)
    spec.cg_tol = 1e-6
    sc = DeviceScene(spec)
    for nm, a in zip("uvw", uvw):
        sc.set_current(nm, a)
    sc.set_current("T", T0)
    plan = ScenePlan([sc])
    plan.single_reduction_cg = cg == "single-reduction"
    tol = 1e-6 if cg == "classic" else 1e-5
    plan.prepare_statics()
    orc = oracle_from_spec(spec)
    orc.set_state(T=T0, u=uvw[0], v=uvw[1], w=uvw[2])
    for s in range(4):
        plan.substep(2e-3)
        orc.substep(2e-3)
        for nm in ("T", "u", "v", "w"):
            got = sc.current(nm).cpu().numpy()
            assert rel_l2(got, getattr(orc, nm)) <= tol, (nm, s, rel_l2(got, getattr(orc, nm)))
        st, ost = sc.read_state(), orc.stats()
        assert st.status == 0
        assert st.pressure_rr <= st.pressure_atol ** 2 * (1 + 1e-12)
        assert abs(st.pressure_iters - ost["grid_done"]) <= 2


def test_cell_velocity_and_diagnostics(torch_cuda):
    from heatflow_mpm.scene import ScenePlan
    from oracle import oracle as O
    fx = golden("substep_air_n12.npz")
    sc = device_scene_from_fixture(fx)
    plan = ScenePlan([sc])
    plan.prepare_statics()
    orc = O.scene_from_fixture(fx, "f32", mean_mode=0, scatter_mode=0)
    for _ in range(int(fx["nsub"])):
        plan.substep(float(fx["dt"]))
        orc.substep(float(fx["dt"]))
    cv = plan.cell_velocity(0).cpu().numpy()
    assert rel_l2(cv, fx["air_velocity"]) <= 1e-5
    assert np.array_equal(cv, orc.cell_velocity())
    # after the projection |div| sits at the CG tolerance: the reference's own threshold (tests/test_solver.py:39)
    assert plan.divergence_max(0) < 1e-3 and float(fx["divergence_max"]) < 1e-3
    assert plan.speed_max(0) == pytest.approx(float(fx["speed_max"]), rel=1e-5)
    # the diagnostic kernels themselves, on a field that is not divergence-free: same value as the oracle
    rng = np.random.default_rng(9)
    for nm in "uvw":
        a = rng.uniform(-1, 1, sc.current(nm).shape).astype(np.float32)
        sc.set_current(nm, a)
        orc.cur(nm)[...] = a
    assert plan.divergence_max(0) == orc.divergence_max()
    assert plan.speed_max(0) == orc.speed_max()


def test_deterministic_and_batch_invariant(torch_cuda):
    """The same scene gives bit-identical results run twice, and alone vs inside a batch of uneven scenes."""
    from heatflow_mpm.scene import DeviceScene, ScenePlan

    def make(n, seed):
        spec, T0, uvw = random_scene_inputs(n, seed)
        sc = DeviceScene(spec)
        sc.set_current("T", T0)
        for nm, a in zip("uvw", uvw):
            sc.set_current(nm, a)
        return sc

    alone = make(24, 3)
    p1 = ScenePlan([alone])
    p1.prepare_statics()
    again = make(24, 3)
    p2 = ScenePlan([again])
    p2.prepare_statics()
    mixed = [make(16, 1), make(24, 3), make(20, 7)]
    p3 = ScenePlan(mixed)
    p3.prepare_statics()
    for _ in range(3):
        p1.substep(2e-3)
        p2.substep(2e-3)
        p3.substep(2e-3)
    for nm in ("T", "u", "v", "w"):
        a = alone.current(nm).cpu().numpy()
        assert np.array_equal(a, again.current(nm).cpu().numpy())
        assert np.array_equal(a, mixed[1].current(nm).cpu().numpy())


@pytest.mark.parametrize("n", [17, 32, 48, 96])
def test_resident_cg_matches_streaming_cg(torch_cuda, n):
    """Single-scene plans use the register-resident CG variant (TMA-staged for the pressure when n % 4 == 0), with 1-3
    tiles per 256-thread group; every choice must give the streaming kernel's bits."""
    from heatflow_mpm.scene import DeviceScene, ScenePlan
    scenes, plans = [], []
    for streaming, tiles in ((True, 0), (False, 0), (False, 3)):
        spec, T0, uvw = random_scene_inputs(n, seed=40 + n)
        sc = DeviceScene(spec)
        sc.set_current("T", T0)
        for nm, a in zip("uvw", uvw):
            sc.set_current(nm, a)
        pl = ScenePlan([sc], streaming_cg=streaming)
        pl.resident_tiles = tiles
        pl.prepare_statics()
        scenes.append(sc)
        plans.append(pl)
    for _ in range(3):
        for pl in plans:
            pl.substep(2e-3)
    a = scenes[0]
    sa = a.read_state()
    for b in scenes[1:]:
        for nm in ("T", "u", "v", "w"):
            assert np.array_equal(a.current(nm).cpu().numpy(), b.current(nm).cpu().numpy()), nm
        assert np.array_equal(a.p.cpu().numpy(), b.p.cpu().numpy())
        sb = b.read_state()
        assert (sa.pressure_iters, sa.heat_iters, sa.status) == (sb.pressure_iters, sb.heat_iters, sb.status)


def test_config1_air_only_plume_100_substeps(torch_cuda):
    """The CPU-runnable configuration end to end: 32^3 air-only plume (h = 15 mm, box heater of 4x4x2 rod cells at
    x = 0.1 m with its trough layer, 400 W capped at 120 C, fan 0), seeded +-0.01 K noise, pressure and heat CG tol
    1e-6, 100 substeps through HeatflowMPM.substep against the oracle in the build's arithmetic: T, u, v, w within
    relative L2 1e-6 every 20 substeps; every solve converged; the plume rises above the heater."""
    from heatflow_mpm.synthetic import plume_box
    sim = plume_box()
    sc = sim.scene
    orc = oracle_from_spec(sc.spec)
    orc.set_state(T=sc.current("T").cpu().numpy())
    for s in range(1, 101):
        sim.substep(2e-3)
        orc.substep(2e-3)
        assert sc.read_state().status == 0, s
        if s % 20 == 0:
            for nm in ("T", "u", "v", "w"):
                assert rel_l2(sc.current(nm).cpu().numpy(), getattr(orc, nm)) <= 1e-6, (nm, s)
    w = sc.current("w").cpu().numpy()
    i0, j0 = int(round(0.10 / sim.grid.h)) - 2, sim.grid.n // 2 - 2
    assert w[i0:i0 + 4, j0:j0 + 4, 4:10].mean() > 1e-3              # warm air rising above the block
    assert sim.grid.divergence_max() < 1e-3


@pytest.mark.parametrize("cg", ["classic", "single-reduction"])
def test_headline_coupled96_vs_oracle(torch_cuda, cg):
    """The benchmark's own configuration -- the default coupled 96^3 scene (h = 5 mm, trough heater 400 W capped at
    120 C, fan 2 m/s, ~16k-particle ellipsoid, frozen body) -- through HeatflowMPM.substep (CUDA-graph replay, the
    TMA-staged resident CG variants, the footprint-box obstacle rebuild): 30 spin-up substeps, then 20 substeps on the
    GPU and on the oracle from the same state.  Every substep: the same CG iteration counts (within 2 for the pressure
    solve, 1 for heat), every solve converged (r.r <= atol^2, status 0); at the end relative L2 <= 1e-6 for T, u, v,
    w and the particle temperatures with the classic pressure solve (the oracle's method), <= 1e-5 with the
    single-reduction one (beta from an expansion, ~1e-7 apart)."""
    torch = torch_cuda
    from heatflow_mpm.synthetic import coupled_default
    from oracle import oracle as O
    from helpers import coupled_default_oracle
    import os
    O.set_threads(len(os.sched_getaffinity(0)))
    tol = 1e-6 if cg == "classic" else 1e-5
    sim = coupled_default(cg=cg)
    sc = sim.scene
    for _ in range(30):
        sim.substep(2e-3)
    torch.cuda.synchronize()
    orc = coupled_default_oracle()
    orc.set_state(**{nm: sc.current(nm).cpu().numpy() for nm in ("T", "u", "v", "w")})
    orc.a["p"][...] = sc.p.cpu().numpy()
    orc.a["ptemp"][: sim.n] = sc.ptemp.cpu().numpy()
    for s in range(20):
        sim.substep(2e-3)
        orc.substep(2e-3)
        st, ost = sc.read_state(), orc.stats()
        assert st.status == 0, (s, st.status)
        assert abs(st.pressure_iters - ost["grid_done"]) <= 2, (s, st.pressure_iters, ost["grid_done"])
        assert abs(st.heat_iters - ost["heat_done"]) <= 1, (s, st.heat_iters, ost["heat_done"])
        assert st.pressure_rr <= st.pressure_atol ** 2 * (1 + 1e-12)
        assert st.heat_rr <= st.heat_atol ** 2 * (1 + 1e-12)
    for nm in ("T", "u", "v", "w"):
        got = sc.current(nm).cpu().numpy()
        assert rel_l2(got, getattr(orc, nm)) <= tol, (nm, rel_l2(got, getattr(orc, nm)))
    assert rel_l2(sc.ptemp.cpu().numpy(), orc.a["ptemp"][: sim.n]) <= tol


def test_divide_by_constant_matches_ieee(torch_cuda):
    """The sampling stages divide every sample coordinate by the cell size with a precomputed reciprocal pair and one
    correction step instead of an IEEE division; the result must be the correctly rounded quotient bit for bit.
    Reference: the binary64 quotient of the two binary32 operands rounded to binary32 (double rounding is harmless for
    division when the intermediate has >= 2p + 2 bits).  Every binary32 value in [2^-12, 2^9) (both signs) and 16 M
    random bit patterns over the whole range (zeros, subnormals, infinities and NaNs included), for the cell sizes of
    the test and benchmark scenes, their squares (the CG stencils divide by h^2) and the buoyancy denominator."""
    torch = torch_cuda
    from heatflow_mpm import _lib
    L = _lib.load()
    L.hf_k_divide_by.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    hs = {np.float32(v) for v in (0.01, 0.015, 0.005, 0.003, 0.02)} | {np.float32(0.48 / n) for n in (32, 48, 64, 96, 128, 160)}
    divisors = hs | {np.float32(h * h) for h in hs} | {np.float32(298.15)}   # h, h^2 (the CG stencils), buoyancy
    gen = torch.Generator(device="cuda").manual_seed(3)
    rnd = torch.randint(-2 ** 31, 2 ** 31 - 1, (1 << 24,), device="cuda", dtype=torch.int64, generator=gen).to(torch.int32)
    lo, hi = np.float32(2.0 ** -12).view(np.int32), np.float32(2.0 ** 9).view(np.int32)
    chunk = 1 << 24
    for y in sorted(divisors):
        def check(xbits):
            x = xbits.view(torch.float32)
            out = torch.empty_like(x)
            _lib.check(L.hf_k_divide_by(x.numel(), C.c_void_p(x.data_ptr()), C.c_float(float(y)),
                                        C.c_void_p(out.data_ptr()), stream))
            ref = (x.double() / float(y)).float()
            same = (out.view(torch.int32) == ref.view(torch.int32)) | (torch.isnan(out) & torch.isnan(ref))
            bad = int((~same).sum())
            if bad:
                i = int((~same).nonzero()[0])
                raise AssertionError(f"y={y!r}: {bad} mismatches, e.g. x={float(x[i])!r}: {float(out[i])!r} "
                                     f"vs {float(ref[i])!r}")
        for start in range(int(lo), int(hi), chunk):
            b = torch.arange(start, min(start + chunk, int(hi)), device="cuda", dtype=torch.int64).to(torch.int32)
            check(b)
            check(b | torch.tensor(-2 ** 31, dtype=torch.int32, device="cuda"))   # negative values
        check(rnd)
        check(torch.tensor([0, -2 ** 31, 1, 0x7F800000, -8388608, 0x7FC00000], dtype=torch.int32, device="cuda"))


@pytest.mark.parametrize("n,vmax", [(20, 3.0), (20, 40.0), (40, 6.0)])
def test_sampling_stages_bit_exact_vs_oracle(torch_cuda, n, vmax):
    """The face stage (semi-Lagrangian advection of u, v, w + buoyancy + relaxation, grid.py:25-79) and the temperature
    stage's advection (heat.py:21-41 with the blend, fixed cells and source) against the oracle's kernels, bit for bit
    (compared as integers), on a random air-only scene whose velocities carry back-traces outside the domain.  The
    face stage samples from velocity boxes staged around each tile with a two-cell halo: |u| dt / h is 0.25 cells at
    (20, 3 m/s), so every back-trace stays in the boxes; 3.3 cells at (20, 40 m/s), so most leave them and read the
    lattice; up to 1 cell at (40, 6 m/s), a mix."""
    torch = torch_cuda
    from heatflow_mpm.scene import DeviceScene, ScenePlan
    from oracle.oracle import Kernels
    dt = 2e-3
    spec, T0, uvw = random_scene_inputs(n, seed=9)
    rng = np.random.default_rng(4)
    uvw = [rng.uniform(-vmax, vmax, a.shape).astype(np.float32) for a in uvw]
    sc = DeviceScene(spec)
    plan = ScenePlan([sc])
    plan.prepare_statics()
    par = sc.parity()
    for nm, a in zip("uvw", uvw):
        getattr(sc, nm)[par].copy_(torch.as_tensor(a, device="cuda"))
    Tn = (25.0 + rng.uniform(-5, 30, (n, n, n))).astype(np.float32)
    sc.T[par ^ 1].copy_(torch.as_tensor(Tn, device="cuda"))
    plan.face_stage(dt)
    torch.cuda.synchronize()
    K = Kernels("f32")
    af = [a.cpu().numpy() for a in (sc.ax, sc.ay, sc.az)]
    kf = [np.ascontiguousarray(a, np.float32) for a in spec.static_k]
    mf = [np.ascontiguousarray(a, np.float32) for a in spec.static_m]
    outs = []
    for axis in range(3):
        o = np.zeros_like(uvw[axis])
        K.call("or_advect_face", n, float(spec.h), dt, uvw[0], uvw[1], uvw[2], axis, uvw[axis], o)
        outs.append(o)
    K.call("or_buoyancy", n, dt, 9.81, float(spec.t_amb), outs[2], Tn)
    for axis in range(3):
        K.call("or_relax", n, float(spec.h), dt, float(spec.rho), float(spec.alpha_f_min), axis, outs[axis], kf[axis],
               mf[axis], af[axis])
    for nm, ref in zip("uvw", outs):
        got = getattr(sc, nm)[par ^ 1].cpu().numpy()
        assert np.array_equal(got.view(np.int32), ref.view(np.int32)), (nm, int((got != ref).sum()))
    # temperature stage: blend (air-only: Tw = T), fixed cells, capped source, then the RK2 advection into T[par ^ 1]
    T = (25.0 + rng.uniform(-5, 30, (n, n, n))).astype(np.float32)
    sc.T[par].copy_(torch.as_tensor(T, device="cuda"))
    plan.temperature_stage(dt)
    torch.cuda.synchronize()
    Tw = T.copy()
    K.call("or_apply_fixed", n, Tw, np.ascontiguousarray(spec.fixed, np.int32), np.ascontiguousarray(spec.tfix, np.float32))
    K.call("or_source", n, Tw, np.ascontiguousarray(spec.source, np.int32), float(spec.rate), float(spec.t_cap), dt)
    T2 = np.zeros_like(T)
    K.call("or_advect_T", n, float(spec.h), dt, Tw, np.ascontiguousarray(spec.static_alpha, np.float32), uvw[0], uvw[1],
           uvw[2], T2)
    got = sc.T[par ^ 1].cpu().numpy()
    assert np.array_equal(got.view(np.int32), T2.view(np.int32)), int((got != T2).sum())


@pytest.mark.parametrize("n,tol", [(36, 1e-6), (44, 1e-6), (92, 1e-4)])
def test_single_reduction_partial_tiles_vs_oracle(torch_cuda, n, tol):
    """The single-reduction pressure solve on edges whose tiles are cut by the domain (n % 8 != 0, n % 32 != 0: partial
    tiles in j and k, face-neighbour points outside the domain; 92: three tiles per group, ~250-280 iterations per
    solve from the random start at the reference tolerance -- at 1e-6 the classic solve itself stops at maxiter), 3
    substeps: GPU vs oracle, relative L2 <= 1e-5, every solve converged, iteration counts within 2 of the classic
    method's."""
    import os
    from heatflow_mpm.scene import DeviceScene, ScenePlan
    from oracle import oracle as O
    O.set_threads(len(os.sched_getaffinity(0)))
    spec, T0, uvw = random_scene_inputs(n, seed=40 + n)
    spec.cg_tol = tol
    sc = DeviceScene(spec)
    for nm, a in zip("uvw", uvw):
        sc.set_current(nm, a)
    sc.set_current("T", T0)
    plan = ScenePlan([sc])
    plan.single_reduction_cg = True
    plan.prepare_statics()
    orc = oracle_from_spec(spec)
    orc.set_state(T=T0, u=uvw[0], v=uvw[1], w=uvw[2])
    for s in range(3):
        plan.substep(2e-3)
        orc.substep(2e-3)
        st, ost = sc.read_state(), orc.stats()
        assert st.status == 0, (s, st.status)
        assert st.pressure_rr <= st.pressure_atol ** 2 * (1 + 1e-12)
        assert abs(st.pressure_iters - ost["grid_done"]) <= 2, (s, st.pressure_iters, ost["grid_done"])
        for nm in ("T", "u", "v", "w"):
            got = sc.current(nm).cpu().numpy()
            assert rel_l2(got, getattr(orc, nm)) <= 1e-5, (nm, s, rel_l2(got, getattr(orc, nm)))
