"""Failure detection of the air solves, in forms that fault, trap or hang no GPU.

The reference is silent when a solve fails (grid.py:248-249 stores warp's iteration count and never checks it); here
every CG solve reports status bits in the scene's state block (HF_SCENE_*), and every spin-wait of the persistent CG
kernels is bounded.  The failures are made on the host: a maxiter that cannot reach the tolerance, a NaN written into
one scene's temperature, and a wait limit of 1 ms with one block kept from its first grid barrier (a barrier that
nothing completes).  In each case the status says what happened, the other scenes of a batch are untouched, and the
next substep on the same device runs normally.
"""
import time

import numpy as np
import pytest

from helpers import random_scene_inputs

pytestmark = pytest.mark.gpu

DT = 2e-3


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


def _plain(n=32, seed=3, **spec_kw):
    from heatflow_mpm.scene import DeviceScene, ScenePlan
    spec, T0, uvw = random_scene_inputs(n, seed=seed)
    for k, v in spec_kw.items():
        setattr(spec, k, v)
    sc = DeviceScene(spec)
    sc.set_current("T", T0)
    for nm, a in zip("uvw", uvw):
        sc.set_current(nm, a)
    plan = ScenePlan([sc])
    plan.prepare_statics()
    return sc, plan


@pytest.mark.parametrize("variant", ["resident", "single-reduction", "streaming"])
def test_maxiter_is_reported(torch_cuda, variant):
    """cg_max_iter = 1 (run as 2: warp's iterations come in pairs) cannot reach tol 1e-4 from a random velocity field:
    the pressure solve stops at 2 iterations and sets HF_SCENE_PRESSURE_MAXITER; a heat tolerance of 1e-14 with
    heat_maxiter = 1 sets HF_SCENE_HEAT_MAXITER."""
    from heatflow_mpm import _lib
    sc, plan = _plain(cg_max_iter=1, heat_maxiter=1, heat_tol=1e-14)
    if variant == "single-reduction":
        plan.single_reduction_cg = True
    elif variant == "streaming":
        plan.plan.options |= _lib.HF_PLAN_STREAMING_CG
    plan.substep(DT)
    st = sc.read_state()
    assert st.status & _lib.HF_SCENE_PRESSURE_MAXITER, st.status
    assert st.status & _lib.HF_SCENE_HEAT_MAXITER, st.status
    assert not st.status & (_lib.HF_SCENE_NONFINITE | _lib.HF_SCENE_BARRIER_TIMEOUT)
    assert st.pressure_iters == 2 and st.pressure_rr > st.pressure_atol ** 2


def test_nonfinite_scene_is_flagged_alone(torch_cuda):
    """Three scenes in one batch; a NaN written on the host into the middle scene's temperature.  After two batched
    substeps that scene carries HF_SCENE_NONFINITE, and the other two are bit-identical (fields, iteration counts,
    status 0) to the same scenes run alone."""
    from heatflow_mpm import _lib
    from heatflow_mpm.batch import AirBatch, AirScenario
    scs = [AirScenario(n=32, heater_x=0.1, power=300.0, seed=1), AirScenario(n=24, heater_x=0.12, fan=1.5, seed=2),
           AirScenario(n=40, power=500.0, fan=2.0, seed=3)]
    alone = []
    for s in scs[0::2]:
        b = AirBatch([s])
        for _ in range(2):
            b.substep(DT)
        alone.append(({nm: b.scenes[0].current(nm).cpu().numpy() for nm in ("T", "u", "v", "w")}, b.scenes[0].read_state()))
    batch = AirBatch(scs)
    T = batch.scenes[1].current("T").cpu().numpy()
    T[5, 7, 9] = np.nan
    batch.scenes[1].set_current("T", T)
    for _ in range(2):
        batch.substep(DT)
    bad = batch.scenes[1].read_state()
    assert bad.status & _lib.HF_SCENE_NONFINITE, bad.status
    for s, (ref, rst) in zip(batch.scenes[0::2], alone):
        st = s.read_state()
        assert st.status == 0
        assert (st.pressure_iters, st.heat_iters) == (rst.pressure_iters, rst.heat_iters)
        for nm in ("T", "u", "v", "w"):
            assert np.array_equal(s.current(nm).cpu().numpy(), ref[nm]), nm


@pytest.mark.parametrize("variant", ["resident", "single-reduction", "batch"])
def test_barrier_timeout_is_reported_and_the_device_stays_usable(torch_cuda, variant):
    """A wait limit of 1 ms and block 0 kept from the first grid barrier of every CG launch: the barrier cannot
    complete, every other block gives up after the limit, the launch returns and the scene's status carries
    HF_SCENE_BARRIER_TIMEOUT (the substep is not counted and the buffer parity does not flip).  With the defaults put
    back, a new scene on the same device substeps normally."""
    torch = torch_cuda
    from heatflow_mpm import _lib
    from heatflow_mpm.batch import AirBatch, AirScenario
    L = _lib.load()
    if variant == "batch":
        batch = AirBatch([AirScenario(n=32, heater_x=0.1, seed=4), AirScenario(n=48, fan=1.0, seed=5)], lanes=2)
        scenes, plan = batch.scenes, batch.plan
    else:
        sc, plan = _plain()
        plan.single_reduction_cg = variant == "single-reduction"
        scenes = [sc]
    par0 = [s.read_state().parity for s in scenes]
    torch.cuda.synchronize()
    _lib.check(L.hf_set_wait_limit(1_000_000, 0), "hf_set_wait_limit")
    try:
        t0 = time.perf_counter()
        plan.substep(DT)
        torch.cuda.synchronize()
        took = time.perf_counter() - t0
    finally:
        _lib.check(L.hf_set_wait_limit(_lib.WAIT_LIMIT_NS, -1), "hf_set_wait_limit")
    assert took < 5.0, took
    states = [s.read_state() for s in scenes]
    assert any(st.status & _lib.HF_SCENE_BARRIER_TIMEOUT for st in states), [st.status for st in states]
    for st, p in zip(states, par0):
        if st.status & _lib.HF_SCENE_BARRIER_TIMEOUT:
            assert st.parity == p and st.substeps == 0
    # the device is usable: a new scene substeps normally and converges
    sc2, plan2 = _plain(seed=11)
    plan2.substep(DT)
    st2 = sc2.read_state()
    assert st2.status == 0 and st2.substeps == 1
    assert np.isfinite(sc2.current("T").cpu().numpy()).all()
