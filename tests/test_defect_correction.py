"""Outer defect correction (HF_FLAG_DEFECT_CORRECTION; not in the reference, off by default): after each CG solve the
true residual b - A x is formed in fp64; above the tolerance the solve restarts from x with it.

* At the reference tolerances the binary32 recurrence and the true residual agree, no restart happens, and the fields
  are bit-identical to the same solves without the check; the fp64 true residual is reported (<= atol^2).
* Below what binary32 vectors can reach (tol 1e-8), the check restarts the solves (status bit HF_SCENE_CORRECTED), at
  most twice per solve; the result stays finite and within 1e-4 relative L2 of an all-fp64 oracle run."""
import dataclasses

import numpy as np
import pytest

from helpers import random_scene_inputs, rel_l2

pytestmark = pytest.mark.gpu


def _pair(n, seed, **spec_kw):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from heatflow_mpm.scene import DeviceScene, ScenePlan
    out = []
    for dc in (False, True):
        spec, T0, uvw = random_scene_inputs(n, seed)
        spec = dataclasses.replace(spec, defect_correction=dc, **spec_kw)
        sc = DeviceScene(spec)
        sc.set_current("T", T0)
        for nm, a in zip("uvw", uvw):
            sc.set_current(nm, a)
        pl = ScenePlan([sc], streaming_cg=True)
        pl.prepare_statics()
        out.append((sc, pl))
    return out


def test_no_restart_at_reference_tolerances():
    from heatflow_mpm import _lib
    (a, pa), (b, pb) = _pair(32, 11)
    for _ in range(3):
        pa.substep(2e-3)
        pb.substep(2e-3)
        sa, sb = a.read_state(), b.read_state()
        assert sa.pressure_true_rr == -1.0 and sa.heat_true_rr == -1.0
        assert not (sb.status & _lib.HF_SCENE_CORRECTED)
        assert 0.0 <= sb.pressure_true_rr <= sb.pressure_atol ** 2
        assert 0.0 <= sb.heat_true_rr <= sb.heat_atol ** 2
        for nm in ("T", "u", "v", "w"):
            assert np.array_equal(a.current(nm).cpu().numpy(), b.current(nm).cpu().numpy()), nm
        assert (sa.pressure_iters, sa.heat_iters) == (sb.pressure_iters, sb.heat_iters)


def test_restart_below_binary32_reach():
    """tol 1e-8: the check restarts the solves; the result stays finite and within 1e-4 relative L2 of an all-fp64
    oracle run at the same tolerance."""
    from heatflow_mpm import _lib
    from helpers import oracle_from_spec
    (_, _), (b, pb) = _pair(24, 12, cg_tol=1e-8, heat_tol=1e-8)
    spec = b.spec
    orc = oracle_from_spec(spec, "f64")
    orc.set_state(T=b.current("T").cpu().numpy(), u=b.current("u").cpu().numpy(), v=b.current("v").cpu().numpy(),
                  w=b.current("w").cpu().numpy())
    corrected = 0
    for _ in range(3):
        pb.substep(2e-3)
        orc.substep(2e-3)
        sb = b.read_state()
        corrected += bool(sb.status & _lib.HF_SCENE_CORRECTED)
        assert not (sb.status & _lib.HF_SCENE_NONFINITE)
        assert np.isfinite(sb.pressure_true_rr) and sb.pressure_true_rr >= 0.0
        for nm in ("T", "u", "v", "w"):
            got = b.current(nm).cpu().numpy()
            assert np.isfinite(got).all()
            assert rel_l2(got, getattr(orc, nm)) <= 1e-4, nm
    assert corrected >= 1
