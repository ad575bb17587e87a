"""Precision study: the CUDA path (binary32 stencils and CG vectors; fp64 inner products, alpha/beta and rhs mean)
against an all-fp64 oracle run of the same scene -- the trough heater at 800 W capped at 120 C, fan 1 m/s, the default
ellipsoid scaled to a ~5.8k-cell footprint at 20 C, frozen body, dt = 2 ms.

Bound (stated for T and the face velocities): relative L2 <= 1e-4 against the fp64 run; the pressure and heat CG
iteration counts within 2 of the fp64 run's; and the largest |div(alpha_f u + alpha_s v_s)| of both runs at the same
level (within 25 %: both sit at the CG tolerance, not at round-off).

The default case is the 64^3 grid of the same box (h = 7.5 mm) over 60 substeps.  HF_PRECISION_FULL=1 runs the full
study instead -- 160^3, h = 3 mm, 300 substeps -- and HF_PRECISION_OUT=<file> writes its figures as JSON.
"""
import json
import os
import time

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def test_fp32_path_vs_fp64_oracle():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from heatflow_mpm.solver import KAPPA_AIR, build_spec
    from heatflow_mpm.synthetic import precision_build, precision_study
    from oracle import oracle as O
    full = os.environ.get("HF_PRECISION_FULL") == "1"
    n, h, steps = (160, 0.003, 300) if full else (64, 0.0075, 60)
    sim = precision_study(n=n, h=h)
    parts, mat, heater, grid = precision_build(n, h)
    spec, _, _, _ = build_spec(parts, mat, heater, grid, 2.5e-3, 20.0, KAPPA_AIR)
    O.set_threads(len(os.sched_getaffinity(0)))
    ref = O.scene_from_spec(spec, "f64", particles=parts, pvel=np.zeros_like(parts),
                            ptemp=np.full(len(parts), 20.0, np.float32))
    log, worst = [], {"T": 0.0, "u": 0.0, "v": 0.0, "w": 0.0}
    t0 = time.time()
    for k in range(1, steps + 1):
        sim.substep(2e-3)
        ref.substep(2e-3)
        st, rs = sim.scene.read_state(), ref.stats()
        assert abs(st.pressure_iters - rs["grid_done"]) <= 2 and abs(st.heat_iters - rs["heat_done"]) <= 2, k
        if k % 20 == 0 or k == steps:
            row = {"substep": k, "pressure_iters": int(st.pressure_iters), "heat_iters": int(st.heat_iters)}
            for nm in ("T", "u", "v", "w"):
                e = rel_l2(sim.scene.current(nm).cpu().numpy(), getattr(ref, nm))
                worst[nm] = max(worst[nm], e)
                row["rel_l2_" + nm] = e
            row["div_max"], row["div_max_fp64"] = sim.grid.divergence_max(), float(ref.divergence_max())
            row["seconds"] = round(time.time() - t0, 1)
            log.append(row)
    last = log[-1]
    if os.environ.get("HF_PRECISION_OUT"):
        with open(os.environ["HF_PRECISION_OUT"], "w") as f:
            json.dump({"n": n, "h": h, "substeps": steps, "worst_rel_l2": worst, "log": log,
                       "particles": int(len(parts)), "oracle_threads": O.num_threads()}, f, indent=1)
    for nm, e in worst.items():
        assert e <= 1e-4, (nm, e)
    assert abs(last["div_max"] - last["div_max_fp64"]) <= 0.25 * last["div_max_fp64"]
