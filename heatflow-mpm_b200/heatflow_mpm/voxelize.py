"""Scene set-up on the device: heater voxelisation, walls and the static sphere (hf_scene_statics).

The reference builds these statics on the host with numpy (heater.py:33-65 ``Heater.masks``; solver.py:48-56 walls and
the fixed-cell priority).  ``device_statics`` computes the same arrays with two kernels straight into device memory:
cell classes and flags, Dirichlet values, the static solid fraction and the static face weights.  Only the heater's
frame and thresholds travel to the device (a few hundred bytes), and one 8-byte read-back brings the source-cell count
from which the host forms heater.py:52's rate.  The arrays equal ``Heater.masks`` / ``BoxHeater.masks`` +
``wall_fixed`` (+ the sphere of ``AirScenario``) bit for bit; ``ambiguous`` counts the cells whose class depends on a
comparison within 1e-12 m of its threshold (0: the classes do not depend on the host CPU's evaluation order).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .heater import K_FAN, K_SOLID, BoxHeater, source_rate

__all__ = ["SceneStatics", "heater_geometry", "device_statics", "sphere_bounds"]


@dataclass
class SceneStatics:
    """Device statics of one scene (torch tensors on its device)."""
    n: int
    h: float
    cell_class: torch.Tensor      # uint8 (n,n,n): heater cell type 0-4, + 8 on sphere cells
    cell_flags: torch.Tensor      # uint8 (n,n,n): bit0 fixed, bit1 source
    tfix: torch.Tensor            # float32 (n,n,n)
    alpha: torch.Tensor           # float32 (n,n,n) static solid fraction
    k: list                       # 3 float32 face arrays
    m: list                       # 3 float32 face arrays
    n_source: int
    ambiguous: int
    rate: float
    geom: dict

    def cell_type(self) -> np.ndarray:
        """The reference's cell classes (heater.py:40, int32 on the host)."""
        return (self.cell_class & 7).to(torch.int32).cpu().numpy()


def sphere_bounds(n: int, h: float, L: float, radius: float):
    """Candidate box of a solid sphere of `radius` resting on the floor at the centre of a box of edge L: i, j in
    [lo, hi), k in [0, top); centre (L/2, L/2, radius)."""
    c = L / 2
    lo, hi = max(0, int((c - radius) / h) - 1), min(n, int((c + radius) / h) + 2)
    top = min(n, int(2 * radius / h) + 2)
    return lo, hi, top


def heater_geometry(heater, n: int, h: float, centre_xy, t_amb: float, sphere=None) -> tuple[_lib.HeaterGeometry, dict]:
    """The hf_heater_geometry record of a Heater / BoxHeater on an n^3 grid of cell size h, and the heater geometry
    dict of heater.py:64.  sphere = (radius, temperature, L) adds the static sphere of AirScenario."""
    G = _lib.HeaterGeometry()
    G.k_solid, G.k_fan = float(np.float32(K_SOLID)), float(np.float32(K_FAN))
    G.t_rod, G.t_amb = float(heater.t_rod), float(t_amb)
    G.fan = 1 if heater.fan > 0 else 0
    if isinstance(heater, BoxHeater):
        bx, by, bz = heater.block
        i0 = int(round(heater.x / h)) - bx // 2
        j0 = int(round(centre_xy[1] / h)) - by // 2
        facing = (0.0, 0.0, 1.0)
        geom = dict(centre=[(i0 + bx / 2) * h, (j0 + by / 2) * h, bz * h / 2], facing=list(facing),
                    axis=[1.0, 0.0, 0.0], up=[0.0, 0.0, 1.0])
        if heater.on:
            if bz + (2 if heater.fan > 0 else 1) > n:
                raise IndexError("box heater layers above the grid")
            G.kind = 2
            for d, (a, b) in enumerate(((i0, i0 + bx), (j0, j0 + by), (0, bz))):
                start, stop, _ = slice(a, b).indices(n)    # numpy slice semantics of BoxHeater.masks
                G.box_lo[d], G.box_hi[d] = start, max(start, stop)
            G.box_trough = bz
    else:
        centre, facing, axis, up = heater.frame(centre_xy)
        geom = dict(centre=centre.tolist(), facing=facing.tolist(), axis=axis.tolist(), up=up.tolist())
        if heater.on:
            G.kind = 1
            for name, v in (("centre", centre), ("facing", facing), ("axis", axis), ("up", up)):
                arr = getattr(G, name)
                for d in range(3):
                    arr[d] = float(v[d])
            R, L2 = heater.radius, heater.length / 2
            # heater.py:43-49, each threshold by the expression written there
            G.half_length = L2
            G.shell_in, G.shell_out = R - h / 2, R + 0.006 + h / 2
            G.cap_half, G.cap_radius = h / 2, R + 0.006
            G.rod_half, G.rod_radius, G.rod_front, G.rod_dz = L2 - 0.015, 0.007 + h / 2, 0.03, 0.03
            G.fan_half, G.fan_high, G.fan_depth = L2 - 0.02, R - 0.01, 0.015
            G.trough_half, G.trough_radius = L2 - 0.015, R - 0.004
    for d in range(3):
        G.m_face[d] = float(np.float32(K_FAN * heater.fan * facing[d])) if heater.fan > 0 else 0.0
    if sphere is not None and sphere[0] > 0:
        radius, t_sphere, L = sphere
        G.sphere = 1
        G.sphere_lo, G.sphere_hi, G.sphere_top = sphere_bounds(n, h, L, radius)
        G.sphere_c, G.sphere_zc, G.sphere_rr = L / 2, radius, radius * radius
        G.sphere_t = float(np.float32(t_sphere))
    return G, geom


def device_statics(heater, n: int, h: float, centre_xy, rho_air: float, t_amb: float, sphere=None,
                   device="cuda:0", stream=None) -> SceneStatics:
    """heater.py:33-65 + solver.py:48-56 (+ the sphere) computed on the device; see the module docstring."""
    L = _lib.load()
    dev = torch.device(device)
    G, geom = heater_geometry(heater, n, h, centre_xy, t_amb, sphere)
    u8 = dict(dtype=torch.uint8, device=dev)
    f32 = dict(dtype=torch.float32, device=dev)
    fs = [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)]
    cls, flags = torch.empty((n, n, n), **u8), torch.empty((n, n, n), **u8)
    tfix, alpha = torch.empty((n, n, n), **f32), torch.empty((n, n, n), **f32)
    k = [torch.empty(s, **f32) for s in fs]
    m = [torch.empty(s, **f32) for s in fs]
    counts = torch.empty(2, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev) if stream is None else stream
    P = _lib.ptr
    _lib.check(L.hf_scene_statics(C.byref(G), n, float(h), P(cls), P(flags), P(tfix), P(alpha), *(P(a) for a in k),
                                  *(P(a) for a in m), P(counts), C.c_void_p(st.cuda_stream)), "hf_scene_statics")
    n_source, ambiguous = (int(x) for x in counts.cpu().tolist())
    rate = source_rate(heater.power, rho_air, n_source, h) if heater.on else 0.0
    return SceneStatics(n=n, h=h, cell_class=cls, cell_flags=flags, tfix=tfix, alpha=alpha, k=k, m=m,
                        n_source=n_source, ambiguous=ambiguous, rate=rate, geom=geom)

