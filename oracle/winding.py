"""Generalized winding number of points against a triangle soup, in numpy fp64.  TEST INFRASTRUCTURE ONLY.

Checker for hf_winding_inside (the inside test of the reference's shapes.py:13-17 _inside, which calls warp-lang's
``mesh_query_point_sign_winding_number(mesh, p, max_dist, 2.0, 0.5)``; warp-lang >= 1.7 per the reference's
pyproject.toml, not installable here).  Warp evaluates the winding number of Jacobson et al. (2013) with the fast
approximation of Barill et al. (2018, accuracy beta = 2.0) and calls a point inside when it exceeds 0.5; this oracle
sums it exactly: w(p) = sum over triangles of Omega / (4 pi), each solid angle by van Oosterom and Strackee (1983),
tan(Omega / 2) = a.(b x c) / (|a||b||c| + (a.b)|c| + (b.c)|a| + (c.a)|b|) with a, b, c the corners relative to p.
Parity with Warp's approximation itself is unpinned (no Warp here); known answers pin the formula (tests).
"""
from __future__ import annotations

import numpy as np


def winding_numbers(tri: np.ndarray, points: np.ndarray, chunk: int = 2048) -> np.ndarray:
    """w for every point: tri (F, 3, 3) corners, points (P, 3); fp64 throughout."""
    T = np.asarray(tri, np.float64).reshape(-1, 3, 3)
    Pts = np.asarray(points, np.float64).reshape(-1, 3)
    out = np.empty(len(Pts))
    for s in range(0, len(Pts), chunk):
        p = Pts[s:s + chunk, None, None, :]                  # (c, 1, 1, 3)
        d = T[None, :, :, :] - p                             # (c, F, 3, 3)
        a, b, c = d[:, :, 0], d[:, :, 1], d[:, :, 2]
        la, lb, lc = (np.sqrt((x * x).sum(-1)) for x in (a, b, c))
        det = (a * np.cross(b, c)).sum(-1)
        den = la * lb * lc + (a * b).sum(-1) * lc + (b * c).sum(-1) * la + (c * a).sum(-1) * lb
        out[s:s + chunk] = (2.0 * np.arctan2(det, den)).sum(-1) / (4.0 * np.pi)
    return out
