"""HeatflowMPM.substep replays a recorded CUDA graph of the air substep after the first substep at each dt: the
fields, particle temperatures and solver statistics equal those of direct launches (graph=False) bit for bit, through
a change of dt and a change of the heater source (which uploads the scene record and records a new graph)."""
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
