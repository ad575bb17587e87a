"""hf_pressure_solve_noalloc against hf_pressure_solve, through the C ABI.

The no-allocation entry point exists for callers that cannot call cudaMalloc (code running inside an allocator
callback, under a device-memory budget someone else owns, or in a host that plans all device memory up front): it
runs the pressure stage of one scene with its scratch in a fixed device array inside the library.  This test checks
that it gives the results of the ordinary entry point (which uses caller-allocated buffers) on two calls in a row,
within the tolerance of the other GPU parity tests (relative L2 <= 1e-6 for p and u, v, w), and that scenes beyond
its stated maximum are rejected with a clear error.  It sits last in collection order so that a failure here leaves
every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import random_scene_inputs, rel_l2

pytestmark = pytest.mark.gpu


def _bind():
    from heatflow_mpm import _lib
    L = _lib.load()
    f = L.hf_pressure_solve_noalloc
    f.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int] + [C.c_void_p] * 12
    f.restype = C.c_int
    L.hf_noalloc_scratch_bytes.restype = C.c_size_t
    return L, _lib


@pytest.mark.parametrize("n", [32, 37, 63, 64])
def test_no_alloc_matches_allocating_entry_point(n):
    """n = 64 is the stated maximum (the scratch layout's largest fill); 37 and 63 give partial tiles and a partial
    last chunk, so the tile and chunk tables written on the device are compared with hf_plan_upload's."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    from heatflow_mpm.scene import DeviceScene, ScenePlan
    L, _lib = _bind()
    dt = 2e-3
    spec, T0, uvw = random_scene_inputs(n, seed=77 + n)
    sc = DeviceScene(spec)
    plan = ScenePlan([sc])
    plan.prepare_statics()               # alpha_f of the static heater body
    rng = np.random.default_rng(5)
    p0 = rng.uniform(-1.0, 1.0, (n, n, n)).astype(np.float32)
    # the ordinary entry point works on the velocity buffer the face stage wrote (u[parity ^ 1]) and on p
    par = sc.parity()
    for nm, a in zip("uvw", uvw):
        getattr(sc, nm)[par ^ 1].copy_(torch.as_tensor(a, device="cuda"))
    sc.p.copy_(torch.as_tensor(p0, device="cuda"))
    # the no-allocation entry point works in place on copies of the same inputs
    U = [torch.as_tensor(a, device="cuda").clone() for a in uvw]
    P = torch.as_tensor(p0, device="cuda").clone()
    ptr = lambda t: C.c_void_p(t.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st_dev = torch.zeros(C.sizeof(_lib.SceneState), dtype=torch.uint8, device="cuda")
    for call in range(2):
        plan.divergence_stage(dt)
        plan.pressure_cg(dt)             # projects u[parity ^ 1] and flips the parity
        rc = L.hf_pressure_solve_noalloc(n, spec.h, spec.rho, dt, spec.cg_tol, spec.cg_max_iter, ptr(U[0]), ptr(U[1]),
                                         ptr(U[2]), ptr(sc.ax), ptr(sc.ay), ptr(sc.az), None, None, None, ptr(P),
                                         ptr(st_dev), stream)
        assert rc == 0, L.hf_last_error().decode()
        torch.cuda.synchronize()
        cur = sc.parity()                # the ordinary call projected u[old parity ^ 1], now the current buffer
        ref = [getattr(sc, nm)[cur].cpu().numpy() for nm in "uvw"]
        assert rel_l2(P.cpu().numpy(), sc.p.cpu().numpy()) <= 1e-6, call
        for a, b in zip(U, ref):
            assert rel_l2(a.cpu().numpy(), b) <= 1e-6, call
        mine = _lib.SceneState.from_buffer_copy(st_dev.cpu().numpy().tobytes())
        theirs = sc.read_state()
        assert mine.pressure_iters == theirs.pressure_iters and mine.status == (theirs.status & 6)
        assert mine.pressure_rr <= mine.pressure_atol ** 2 * (1 + 1e-12)
        # next call: same inputs for both paths (the projected velocities, p as warm start)
        for nm, a in zip("uvw", U):
            getattr(sc, nm)[sc.parity() ^ 1].copy_(a)


def test_no_alloc_rejects_scenes_beyond_its_scratch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    L, _lib = _bind()
    assert L.hf_noalloc_max_edge() == 64 and L.hf_noalloc_scratch_bytes() == 9 * 1024 * 1024
    n = 65
    dummy = torch.zeros(1, device="cuda")
    d = C.c_void_p(dummy.data_ptr())
    rc = L.hf_pressure_solve_noalloc(n, 0.005, 1.2, 2e-3, 1e-4, 400, d, d, d, d, d, d, None, None, None, d, None, None)
    assert rc == _lib.HF_ERR_ARG
    assert b"2..64" in L.hf_last_error()
