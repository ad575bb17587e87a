"""Frame output (the reference's run_scene.py frames and solver.py:105-110 frame_dict): frames packed on the device and
written asynchronously are bit-identical to frame_dict at the same state, through a reused ring of slots; the CLI
writes the reference's files.  CPU part: the CLI's body construction and its refusal of mesh files."""
import os

import numpy as np
import pytest


def test_cli_body_and_mesh_refusal():
    from heatflow_mpm.run_scene import body_particles, parse
    a = parse(["--out", "x", "--mesh", "ellipsoid"])
    assert (a.seconds, a.frame_dt, a.dt, a.h, a.L, a.power, a.t_cap, a.t_sol, a.t_liq) == \
           (20.0, 0.02, 2e-3, 0.005, 0.48, 400.0, 120.0, 30.0, 36.0)
    P = body_particles(a)
    assert P.dtype == np.float32 and 10_000 < len(P) < 25_000 and P[:, 2].min() >= 0.0
    a2 = parse(["--out", "x", "--mesh", "no_such_mesh.obj"])
    with pytest.raises(SystemExit):
        body_particles(a2)


@pytest.mark.gpu
def test_cli_fills_obj_mesh(tmp_path):
    """--mesh file.obj: the body is shapes.py's mesh_particles of that file with the CLI's height, spacing, box, seed
    and yaw."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from heatflow_mpm.run_scene import body_particles, parse
    from heatflow_mpm.shapes import mesh_particles
    from test_scene_setup import torus, write_obj
    p = tmp_path / "t.obj"
    write_obj(p, *torus())
    a = parse(["--out", "x", "--mesh", str(p), "--height", "0.05", "--yaw", "20", "--seed", "4"])
    P = body_particles(a)
    assert len(P) > 1000 and np.array_equal(P, mesh_particles(str(p), 0.05, 2.5e-3, 0.48, 4, 20.0))


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.gpu
def test_async_frames_equal_frame_dict(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from heatflow_mpm import GridConfig, Heater, HeatflowMPM, Material
    from heatflow_mpm.frames import FrameWriter
    from heatflow_mpm.synthetic import ellipsoid_particles
    P = ellipsoid_particles(semi=(0.03, 0.02, 0.04), spacing=4e-3, L=0.24)
    sim = HeatflowMPM(P, Material(), Heater(dist=0.1, z=0.06, radius=0.03, length=0.1, fan=2.0),
                      GridConfig(L=0.24, h=0.01), 4e-3, 20.0, body="frozen")
    w = FrameWriter(sim, str(tmp_path), depth=2)
    expected = {}
    for k in range(4):                       # 4 frames through 2 slots: every slot reused
        for _ in range(2):
            sim.substep(2e-3)
        torch.cuda.synchronize()
        expected[k] = sim.frame_dict(0.004 * (k + 1), with_air=(k != 2))
        w.write(k, 0.004 * (k + 1), with_air=(k != 2))
    w.close()
    for k, ref in expected.items():
        got = np.load(os.path.join(tmp_path, f"frame_{k:04d}.npz"))
        assert sorted(got.files) == sorted(ref.keys()), k
        for key, val in ref.items():
            assert _same(got[key], val), (k, key)


@pytest.mark.gpu
def test_run_scene_cli(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from heatflow_mpm.run_scene import main
    out = str(tmp_path / "scene")
    main(["--out", out, "--seconds", "0.06", "--frame-dt", "0.02", "--L", "0.24", "--h", "0.012", "--height", "0.05",
          "--heater-dist", "0.1", "--heater-z", "0.06", "--fan", "1.0", "--spacing", "4e-3"])
    frames = sorted(os.listdir(os.path.join(out, "frames")))
    assert frames == [f"frame_{k:04d}.npz" for k in range(4)]
    st = np.load(os.path.join(out, "static.npz"))
    n = int(st["n"])
    f = np.load(os.path.join(out, "frames", frames[-1]))
    assert f["grid_T"].dtype == np.float16 and f["grid_T"].shape == (n ** 3,)
    assert f["air_u"].shape == (n ** 3, 3) and f["temp"].dtype == np.float16 and f["pos"].dtype == np.float32
    assert float(f["t"]) == pytest.approx(0.06) and np.isfinite(f["grid_T"].astype(np.float32)).all()
    assert os.path.exists(os.path.join(out, "meta.json"))


@pytest.mark.gpu
def test_grid_T_async_matches_grid_T():
    """grid_T_async (device-side copy of the current buffer, download on a side stream) delivers what grid_T reads,
    through both staging buffers."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from heatflow_mpm import GridConfig, Heater, HeatflowMPM, Material
    from heatflow_mpm.synthetic import ellipsoid_particles
    P = ellipsoid_particles(semi=(0.03, 0.02, 0.04), spacing=4e-3, L=0.24)
    sim = HeatflowMPM(P, Material(), Heater(dist=0.1, z=0.06, radius=0.03, length=0.1, fan=2.0),
                      GridConfig(L=0.24, h=0.01), 4e-3, 20.0, body="frozen")
    n = sim.grid.n
    bufs = [torch.empty((n, n, n), dtype=torch.float32).pin_memory() for _ in range(2)]
    for k in range(5):
        sim.substep(2e-3)
        ev = sim.grid_T_async(bufs[k % 2])
        ref = sim.grid_T()
        ev.synchronize()
        assert np.array_equal(bufs[k % 2].numpy(), ref), k
