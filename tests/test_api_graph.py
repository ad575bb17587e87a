"""HeatflowMPM.substep replays a recorded CUDA graph of the air substep after the first substep at each dt: the
fields, particle temperatures and solver statistics equal those of direct launches (graph=False) bit for bit, through
a change of dt and a change of the heater source (which uploads the scene record and records a new graph).  Particle
states set from pinned host memory (uploaded on a side stream) give the same bits as states copied in stream order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(graph):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from heatflow_mpm import GridConfig, Heater, HeatflowMPM, Material
    from heatflow_mpm.synthetic import ellipsoid_particles
    P = ellipsoid_particles(semi=(0.03, 0.02, 0.04), spacing=4e-3, L=0.24)
    return HeatflowMPM(P, Material(t_sol=28.0, t_liq=34.0), Heater(dist=0.1, z=0.06, radius=0.03, length=0.1, fan=2.0),
                       GridConfig(L=0.24, h=0.01), 4e-3, 20.0, body="frozen", graph=graph)


def test_graph_replay_equals_direct_launches():
    a, b = _sim(True), _sim(False)
    for sim in (a, b):
        for _ in range(3):
            sim.substep(2e-3)
        for _ in range(2):
            sim.substep(1e-3)
        src = sim.heat.src.cpu().numpy().astype(bool)
        sim.heat.set_source(src, 0.5 * float(sim.heat.rate), 90.0)
        for _ in range(3):
            sim.substep(1e-3)
    assert a._graph is not None and b._graph is None
    for nm in ("T", "u", "v", "w"):
        assert np.array_equal(a.scene.current(nm).cpu().numpy(), b.scene.current(nm).cpu().numpy()), nm
    assert np.array_equal(a.temperatures(), b.temperatures())
    sa, sb = a.status(), b.status()
    assert sa == sb and sa["substeps"] == 8


def test_pinned_particle_uploads_equal_in_order_copies():
    """FrozenBody.set_state with pinned host tensors uploads on a side stream into one of two device buffer pairs,
    overlapping the substep in flight.  With a different particle state before every substep (positions shifted and
    velocities changed), the result equals that of the same states copied in stream order from numpy arrays, bit for
    bit: no substep reads a pair while it is being refilled."""
    import torch
    a, b = _sim(True), _sim(True)
    P0 = a.body.pos_t.cpu().numpy().copy()
    V0 = a.body.vel_t.cpu().numpy().copy()
    rng = np.random.default_rng(3)
    states = []
    for s in range(6):
        shift = np.float32(2e-3) * np.float32(s % 3)
        states.append(((P0 + shift).astype(np.float32), rng.uniform(-0.2, 0.2, V0.shape).astype(np.float32)))
    pinned = [(torch.from_numpy(p).pin_memory(), torch.from_numpy(v).pin_memory()) for p, v in states]
    for s in range(6):
        a.body.set_state(*pinned[s])
        a.substep(2e-3)
        b.body.set_state(*states[s])
        b.substep(2e-3)
    torch.cuda.synchronize()
    for nm in ("T", "u", "v", "w"):
        assert np.array_equal(a.scene.current(nm).cpu().numpy(), b.scene.current(nm).cpu().numpy()), nm
    assert np.array_equal(a.temperatures(), b.temperatures())
    assert np.array_equal(a.body.pos_t.cpu().numpy(), states[-1][0])
    assert a.status() == b.status()
