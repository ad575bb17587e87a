"""Batched and served air scenes: scenario construction, admission logic (CPU), and on the GPU that every scene of a
batch or of a served trace ends bit-identical to the same scene run alone, that a CUDA-graph replay gives the eager
bits, and that an air-only scenario with a fan and a static solid sphere matches the oracle (relative L2 <= 1e-6, the
bound used for every whole-substep comparison)."""
import numpy as np
import pytest

from helpers import oracle_from_spec, rel_l2


# ------------------------------------------------------------------------------------------------------ CPU
def test_box_heater_fan_layer():
    from heatflow_mpm.heater import BoxHeater, FAN, K_FAN, K_SOLID, ROD, TROUGH
    n, h = 24, 0.02
    hot = BoxHeater(x=0.2, fan=2.0, power=300.0)
    cells, solid, source, rate, kf, mf, _ = hot.masks(n, h, (0.24, 0.24), 1.2)
    i0, j0 = 10 - 2, 12 - 2
    assert (cells[i0:i0 + 4, j0:j0 + 4, 0:2] == ROD).all()
    assert (cells[i0:i0 + 4, j0:j0 + 4, 2] == TROUGH).all()
    assert (cells[i0:i0 + 4, j0:j0 + 4, 3] == FAN).all()
    assert source.sum() == 32 and solid.sum() == 32
    assert rate == pytest.approx(300.0 / (1.2 * 1005.0 * 32 * h ** 3))
    # the face between the fan layer and the air above: K_FAN, blowing upward at 2 m/s
    assert kf[2][i0 + 1, j0 + 1, 4] == np.float32(K_FAN)
    assert mf[2][i0 + 1, j0 + 1, 4] == np.float32(K_FAN * 2.0)
    assert mf[0][i0 + 1, j0 + 1, 3] == 0.0          # no momentum across the sideways faces
    assert kf[2][i0 + 1, j0 + 1, 2] == np.float32(K_SOLID)   # rod top
    still = BoxHeater(x=0.2, fan=0.0).masks(n, h, (0.24, 0.24), 1.2)[0]
    assert (still == FAN).sum() == 0


def test_sphere_scenario_spec():
    from heatflow_mpm.batch import AirScenario
    from heatflow_mpm.heater import K_SOLID
    sc = AirScenario(n=24, sphere_radius=0.06, sphere_t=12.0, heater_x=0.1)
    spec = sc.spec()
    g = (np.arange(24) + 0.5) * sc.h
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    ball = (X - 0.24) ** 2 + (Y - 0.24) ** 2 + (Z - 0.06) ** 2 <= 0.06 ** 2
    assert ball.sum() > 50
    assert spec.fixed[ball].all() and (spec.tfix[ball] == np.float32(12.0)).all()
    assert (spec.static_alpha[ball] == 1.0).all()
    c = np.argwhere(ball)[0]
    assert spec.static_k[0][c[0], c[1], c[2]] == np.float32(K_SOLID)
    assert spec.static_k[0][c[0] + 1, c[1], c[2]] == np.float32(K_SOLID)
    assert spec.static_m[0][c[0], c[1], c[2]] == 0.0
    T0 = sc.initial_T()
    assert T0.dtype == np.float32 and np.abs(T0 - 25.0).max() <= 0.0101
    assert np.array_equal(T0, AirScenario(n=24, seed=sc.seed).initial_T())


def test_traces_are_seeded():
    from heatflow_mpm.batch import ensemble
    from heatflow_mpm.serve import poisson_trace
    a, b = poisson_trace(rate=50, duration=20, seed=3), poisson_trace(rate=50, duration=20, seed=3)
    assert [(r.arrival, r.scenario.n, r.scenario.horizon) for r in a] == \
           [(r.arrival, r.scenario.n, r.scenario.horizon) for r in b]
    arr = np.array([r.arrival for r in a])
    assert (np.diff(arr) > 0).all() and 700 < len(a) < 1300
    e = ensemble(count=64, seed=1)
    assert len(e) == 64 and {s.n for s in e} <= {32, 48, 64, 96, 128}
    assert [s.power for s in e] == [s.power for s in ensemble(count=64, seed=1)]


def test_admission_respects_slots_and_hbm_budget(monkeypatch):
    """Host logic of the server with fake scenes: FIFO admission bounded by slots and by the HBM budget; scenes
    retire after exactly their horizon; the plan is rebuilt only when the membership changes."""
    from heatflow_mpm import serve
    from heatflow_mpm.batch import AirScenario

    built = []

    class FakePlan:
        def __init__(self, scenes, device=None, **kw):
            self.scenes = list(scenes)
            built.append(len(self.scenes))

        def prepare_statics(self):
            pass

    setups = []
    monkeypatch.setattr(serve, "make_scene", lambda sc, dev, **kw: setups.append(kw.get("setup")) or object())
    monkeypatch.setattr(serve, "ScenePlan", FakePlan)

    class Landed:                                          # a result copy that has already landed
        def query(self):
            return True

        def synchronize(self):
            pass

    class Server(serve.AirServer):
        def _advance(self):
            pass

        def _copy_back(self, req, slot):
            return Landed(), {}

    big, small = AirScenario(n=96, horizon=3), AirScenario(n=32, horizon=2)
    srv = Server(device="cpu", hbm_budget=big.device_bytes() + 2 * small.device_bytes(), max_slots=3, result_fields=())
    reqs = [serve.Request(big, 0.0, 0), serve.Request(big, 0.0, 1), serve.Request(small, 0.0, 2)]
    for r in reqs:
        srv.submit(r)
    srv.step(0.0)
    assert [r.rid for r in srv.active] == [0]          # the second big one does not fit; FIFO blocks the small one
    srv.step(0.1)
    srv.step(0.2)                                        # request 0 retires after its 3rd substep
    assert reqs[0].done_at == 0.2 and reqs[0].substeps_done == 3 and srv.active == []
    srv.step(0.3)
    assert [r.rid for r in srv.active] == [1, 2]
    for t in (0.4, 0.5):
        srv.step(t)
    assert reqs[2].done_at == 0.4 and reqs[1].done_at == 0.5
    assert srv.scene_substeps == 3 + 3 + 2 and srv.used == 0
    s = srv.summary()
    assert s["requests_done"] == 3 and s["batched_substeps"] == 6
    # statics built on the device by default: only the initial temperature is uploaded per admitted scene
    from heatflow_mpm.batch import upload_bytes
    assert setups == ["device"] * 3 and s["setup"] == "device" and s["admit_ms_p50"] is not None
    assert srv.h2d_bytes == 2 * 4 * 96 ** 3 + 4 * 32 ** 3
    assert upload_bytes(small, "host") > upload_bytes(small, "device") == 4 * 32 ** 3


# ------------------------------------------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


def _scenarios():
    from heatflow_mpm.batch import AirScenario
    return [AirScenario(n=17, heater_x=0.12, fan=2.0, power=250.0, seed=1),
            AirScenario(n=24, sphere_radius=0.05, fan=1.0, seed=2),
            AirScenario(n=32, heater_x=0.2, sphere_radius=0.04, sphere_t=15.0, power=600.0, seed=3),
            AirScenario(n=20, seed=4)]


def _alone(sc, steps, dt=2e-3):
    from heatflow_mpm.batch import AirBatch
    b = AirBatch([sc])
    for _ in range(steps):
        b.substep(dt)
    s = b.scenes[0]
    return {nm: s.current(nm).cpu().numpy() for nm in ("T", "u", "v", "w")}, s.read_state()


def _same(fields, state, ref):
    rf, rs = ref
    for nm in ("T", "u", "v", "w"):
        assert np.array_equal(fields[nm], rf[nm]), nm
    assert (state.pressure_iters, state.heat_iters, state.status) == (rs.pressure_iters, rs.heat_iters, rs.status)


@pytest.mark.gpu
def test_batch_matches_alone(cuda):
    from heatflow_mpm.batch import AirBatch
    scs = _scenarios()
    b = AirBatch(scs)
    for _ in range(4):
        b.substep(2e-3)
    for sc, s in zip(scs, b.scenes):
        st = s.read_state()
        assert st.status == 0
        _same({nm: s.current(nm).cpu().numpy() for nm in ("T", "u", "v", "w")}, st, _alone(sc, 4))


@pytest.mark.gpu
def test_sphere_fan_scene_vs_oracle(cuda):
    from heatflow_mpm.batch import AirBatch, AirScenario
    sc = AirScenario(n=24, heater_x=0.12, fan=2.5, sphere_radius=0.05, sphere_t=10.0, cg_tol=1e-6, seed=5)
    b = AirBatch([sc])
    spec = sc.spec()
    orc = oracle_from_spec(spec)
    s = b.scenes[0]
    orc.set_state(T=s.current("T").cpu().numpy())
    for k in range(4):
        b.substep(2e-3)
        orc.substep(2e-3)
        for nm in ("T", "u", "v", "w"):
            assert rel_l2(s.current(nm).cpu().numpy(), getattr(orc, nm)) <= 1e-6, (nm, k)
    assert float(np.abs(s.current("w").cpu().numpy()).max()) > 0.0


@pytest.mark.gpu
def test_graph_replay_matches_eager(cuda):
    from heatflow_mpm.batch import AirBatch
    scs = _scenarios()[:3]
    g, e = AirBatch(scs), AirBatch(scs)
    g.run(2e-3, 7, use_graph=True, graph_steps=3)      # 1 warm-up + 2 replays of 3
    e.run(2e-3, 7, use_graph=False)
    for a, c in zip(g.scenes, e.scenes):
        for nm in ("T", "u", "v", "w"):
            assert np.array_equal(a.current(nm).cpu().numpy(), c.current(nm).cpu().numpy()), nm
        assert a.read_state().pressure_iters == c.read_state().pressure_iters


@pytest.mark.gpu
def test_served_scenes_match_alone(cuda):
    """Two slots for five requests: scenes join and leave a running batch; each ends as if run alone."""
    import dataclasses
    from heatflow_mpm.serve import AirServer, Request
    horizons = [3, 5, 2, 4, 3]
    scs = [dataclasses.replace(sc, horizon=h) for sc, h in zip(_scenarios() + [_scenarios()[0]], horizons)]
    scs[4] = dataclasses.replace(scs[4], n=16, seed=9)
    srv = AirServer(max_slots=2, keep_results=True)
    out = srv.serve([Request(sc, 0.0, i) for i, sc in enumerate(scs)], time_limit=120.0)
    assert out["requests_done"] == 5 and out["requests_unfinished"] == 0
    assert out["scene_substeps"] == sum(horizons) and out["plan_builds"] >= 3
    for r in srv.finished:
        assert r.substeps_done == r.scenario.horizon
        _same(r.result, r.result["state"], _alone(r.scenario, r.scenario.horizon))


@pytest.mark.gpu
def test_autotune_keeps_results(cuda):
    """Tuning leaves the batch where it was, and every launch shape (blocks, group size, lanes) computes the same
    bits: two substeps under each candidate, from the restored start, equal two substeps of an untuned batch."""
    from heatflow_mpm.batch import AirBatch, autotune
    scs = _scenarios()
    b = AirBatch(scs)
    sms = cuda.cuda.get_device_properties(0).multi_processor_count
    cands = [(2 * sms, 1, 4), (4 * sms, 0, 1), (sms, 20_000, 2), (3 * sms, 1, 3), (2 * sms, 0, 8)]
    ref = AirBatch(scs)
    same = lambda x, y: all(np.array_equal(a.current(nm).cpu().numpy(), c.current(nm).cpu().numpy())
                            for a, c in zip(x.scenes, y.scenes) for nm in ("T", "u", "v", "w"))
    best, timings = autotune(b, reps=1, candidates=cands, cache=False)
    assert best in cands and len(timings) == len(cands)
    assert same(b, ref)
    start = b.snapshot()
    for _ in range(2):
        ref.substep(2e-3)
    for pb, gc, ln in cands:
        b.restore(start)
        b.plan.plan.persistent_blocks, b.plan.plan.group_cells, b.plan.lanes = pb, gc, ln
        for _ in range(2):
            b.substep(2e-3)
        assert same(b, ref), (pb, gc, ln)
        assert [s.read_state().pressure_iters for s in b.scenes] == [s.read_state().pressure_iters for s in ref.scenes]


@pytest.mark.gpu
def test_served_failure_is_reported_for_that_request_only(cuda):
    """Three requests served together; after the first batched substep a NaN is written on the host into the middle
    request's temperature.  The server's status check finds HF_SCENE_NONFINITE, that request leaves the batch as
    failed (its result carries the status), and the other two finish with results bit-identical to running alone."""
    import dataclasses
    from heatflow_mpm import _lib
    from heatflow_mpm.serve import AirServer, Request
    scs = [dataclasses.replace(sc, horizon=h) for sc, h in zip(_scenarios()[:3], (5, 6, 4))]
    srv = AirServer(max_slots=3, keep_results=True, status_every=2)
    reqs = [Request(sc, 0.0, i) for i, sc in enumerate(scs)]
    for r in reqs:
        srv.submit(r)
    t = 0.0
    srv.step(t)
    bad = reqs[1]
    T = bad.scene.current("T").cpu().numpy()
    T[3, 4, 5] = np.nan
    bad.scene.set_current("T", T)
    while srv.queue or srv.active or srv.retiring:
        t += 0.01
        srv.step(t)
        srv._collect(t, wait=not srv.active)
    cuda.cuda.synchronize()
    assert [r.rid for r in srv.failed] == [1] and sorted(r.rid for r in srv.finished) == [0, 2]
    assert bad.result["failed"] and bad.result["status"] & _lib.HF_SCENE_NONFINITE
    assert bad.substeps_done < bad.scenario.horizon          # it left the batch before its horizon
    for r in srv.finished:
        assert r.substeps_done == r.scenario.horizon
        _same(r.result, r.result["state"], _alone(r.scenario, r.scenario.horizon))
    s = srv.summary()
    assert s["requests_failed"] == 1 and s["requests_done"] == 2
