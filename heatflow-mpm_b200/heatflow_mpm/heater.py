"""Heater geometry as grid masks (reference: heatflow_mpm/heater.py:1-65), plus a box heater for synthetic scenes.

``Heater.masks`` must reproduce the reference's cell classes, solid/source masks, source rate and static face weights
bit for bit, so the geometric tests below use the same floating-point primitives in the same order as the reference
(projection of cell centres onto the heater frame with ``@``, distances with ``np.hypot``); the code around them is
organised differently.  Cell classes: 0 air, 1 reflector shell, 2 rod, 3 fan outlet, 4 trough air.
"""
from __future__ import annotations

from dataclasses import dataclass
import numpy as np

K_SOLID = 1.0     # face relaxation weight next to solid cells [kg/s] (heater.py:7)
K_FAN = 0.05      # face relaxation weight in the fan outlet [kg/s] (heater.py:7)
CP_AIR = 1005.0   # heat capacity of air [J/(kg K)] (heater.py:7)

AIR, SHELL, ROD, FAN, TROUGH = 0, 1, 2, 3, 4


def face_masks(solid: np.ndarray, fan: np.ndarray) -> tuple[list, list]:
    """Per face lattice: does the face touch a solid cell, and does it touch a fan cell but no solid one
    (heater.py:54-63; domain faces see the outside as empty)."""
    touch_solid, touch_fan = [], []
    for axis in range(3):
        widths = [(0, 0), (0, 0), (0, 0)]
        widths[axis] = (1, 1)
        sp, fp = np.pad(solid, widths), np.pad(fan, widths)
        n_faces = solid.shape[axis] + 1
        lo, hi = np.arange(0, n_faces), np.arange(1, n_faces + 1)
        ts = np.take(sp, lo, axis=axis) | np.take(sp, hi, axis=axis)
        touch_solid.append(ts)
        touch_fan.append((np.take(fp, lo, axis=axis) | np.take(fp, hi, axis=axis)) & ~ts)
    return touch_solid, touch_fan


def fan_momentum(touch_fan: list, fan_speed: float, facing) -> list:
    """Momentum weights K_FAN * fan_speed * facing[axis] on the fan faces of face_masks (heater.py:61-62)."""
    return [np.where(touch_fan[axis], K_FAN * fan_speed * facing[axis], 0.0).astype(np.float32) for axis in range(3)]


def face_weights(solid: np.ndarray, fan: np.ndarray, fan_speed: float, facing) -> tuple[list, list]:
    """Static relaxation weights of the three face lattices (heater.py:54-63).

    A face touching a solid cell gets K_SOLID; otherwise a face touching a fan cell gets K_FAN, and its
    momentum weight K_FAN * fan_speed * facing[axis]."""
    touch_solid, touch_fan = face_masks(solid, fan)
    k_faces = [np.where(ts, K_SOLID, np.where(tf, K_FAN, 0.0)).astype(np.float32)
               for ts, tf in zip(touch_solid, touch_fan)]
    return k_faces, fan_momentum(touch_fan, fan_speed, facing)


def source_rate(power: float, rho_air: float, n_source: int, h: float) -> float:
    """Volumetric heating rate [K/s] of the source cells (heater.py:51-52)."""
    return power / (rho_air * CP_AIR * max(int(n_source), 1) * h ** 3)


@dataclass
class Heater:
    """Electric trough heater (reference heater.py:10-21); same fields and defaults."""
    dist: float = 0.21
    direction: tuple = (-0.423, 0.906)
    z: float = 0.12
    tilt: float = 15.0
    radius: float = 0.055
    length: float = 0.22
    t_rod: float = 300.0
    power: float = 400.0
    t_cap: float = 120.0
    fan: float = 0.0
    on: bool = True

    def frame(self, centre_xy):
        """Head centre and the unit vectors (facing, axis, up) of the trough (heater.py:23-30)."""
        d = np.asarray(self.direction, float) / np.linalg.norm(self.direction)
        centre = np.array([centre_xy[0] + self.dist * d[0], centre_xy[1] + self.dist * d[1], self.z])
        tl = np.deg2rad(self.tilt)
        facing = np.array([-d[0] * np.cos(tl), -d[1] * np.cos(tl), -np.sin(tl)])
        axis = np.array([d[1], -d[0], 0.0])
        return centre, facing, axis, np.cross(axis, facing)

    def _classify(self, n: int, h: float, centre, facing, axis, up) -> np.ndarray:
        cells = np.zeros((n, n, n), np.int32)
        if not self.on:
            return cells
        g = (np.arange(n) + 0.5) * h
        rel = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1) - centre
        along, front, high = rel @ axis, rel @ facing, rel @ up   # coordinates in the heater frame
        radial = np.hypot(front, high)
        half = self.length / 2
        behind = front <= 0
        # reflector: half-cylinder shell of thickness 6 mm plus the two end caps
        shell = (np.abs(along) <= half) & behind & (radial >= self.radius - h / 2) & (radial <= self.radius + 0.006 + h / 2)
        caps = (np.abs(np.abs(along) - half) <= h / 2) & behind & (radial <= self.radius + 0.006)
        cells[shell] = SHELL
        cells[caps] = SHELL
        # two heating rods, 3 cm in front of the back wall, 3 cm above and below the axis
        for dz in (-0.03, 0.03):
            cells[(np.abs(along) <= half - 0.015) & (np.hypot(front + 0.03, high - dz) <= 0.007 + h / 2)] = ROD
        if self.fan > 0:
            outlet = (np.abs(along) <= half - 0.02) & (np.abs(high) <= self.radius - 0.01) & (front > 0) & (front <= 0.015)
            cells[(cells == AIR) & outlet] = FAN
        trough = (np.abs(along) <= half - 0.015) & (radial <= self.radius - 0.004) & behind
        cells[(cells == AIR) & trough] = TROUGH
        return cells

    def masks(self, n: int, h: float, centre_xy, rho_air: float):
        """(cell classes, solid, source, rate [K/s], k_faces, m_faces, geometry) as heater.py:33-65 returns them."""
        centre, facing, axis, up = self.frame(centre_xy)
        cells = self._classify(n, h, centre, facing, axis, up)
        solid = (cells == SHELL) | (cells == ROD)
        source = (cells == FAN) | (cells == TROUGH)
        rate = source_rate(self.power, rho_air, int(source.sum()), h) if self.on else 0.0
        k_faces, m_faces = face_weights(solid, cells == FAN, self.fan, facing)
        geom = dict(centre=centre.tolist(), facing=facing.tolist(), axis=axis.tolist(), up=up.tolist())
        return cells, solid, source, rate, k_faces, m_faces, geom


@dataclass
class BoxHeater:
    """Box heater of the synthetic air-only scenes: a block of rod cells on the floor with a layer of heated air on
    top.  Block cells i in [round(x/h) - bx//2, +bx), j in [n//2 - by//2, +by), k in [0, bz) are rods (solid, fixed at
    t_rod); the bx x by layer at k = bz is trough air (the power source); with fan > 0 the layer above it is a fan
    outlet blowing upward (class 3, relaxation weight K_FAN toward fan m/s, as heater.py:54-63 does for the trough
    heater).  Same interface as Heater."""
    x: float = 0.10
    block: tuple = (4, 4, 2)
    t_rod: float = 300.0
    power: float = 400.0
    t_cap: float = 120.0
    fan: float = 0.0
    on: bool = True

    def masks(self, n: int, h: float, centre_xy, rho_air: float):
        bx, by, bz = self.block
        i0 = int(round(self.x / h)) - bx // 2
        j0 = int(round(centre_xy[1] / h)) - by // 2
        cells = np.zeros((n, n, n), np.int32)
        if self.on:
            cells[i0:i0 + bx, j0:j0 + by, 0:bz] = ROD
            cells[i0:i0 + bx, j0:j0 + by, bz] = TROUGH
            if self.fan > 0:
                cells[i0:i0 + bx, j0:j0 + by, bz + 1] = FAN
        solid = cells == ROD
        source = (cells == TROUGH) | (cells == FAN)
        rate = source_rate(self.power, rho_air, int(source.sum()), h) if self.on else 0.0
        facing = (0.0, 0.0, 1.0)
        k_faces, m_faces = face_weights(solid, cells == FAN, self.fan, facing)
        c = [(i0 + bx / 2) * h, (j0 + by / 2) * h, bz * h / 2]
        geom = dict(centre=c, facing=list(facing), axis=[1.0, 0.0, 0.0], up=[0.0, 0.0, 1.0])
        return cells, solid, source, rate, k_faces, m_faces, geom
