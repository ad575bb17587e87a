"""Particles filling a mesh (reference: heatflow_mpm/shapes.py:1-51): a jittered lattice kept where it lies inside the
mesh, the inside test on the GPU.

The reference reads meshes with trimesh and tests points with Warp's ``mesh_query_point_sign_winding_number`` (accuracy
2.0, threshold 0.5).  Neither library is used here:

* ``load_obj`` reads Wavefront OBJ vertices and faces (polygons fanned into triangles, ``v/vt/vn`` and negative
  indices accepted) and drops vertices no face uses, as trimesh's processing does; ``load_mesh`` then applies
  shapes.py:20-31's transform (Z-up, yaw, scale to `height`, centred in xy, lowest point at z = 0) step for step;
* the inside test is ``hf_winding_inside``: the generalized winding number of every candidate summed exactly over all
  triangles on the device (Warp evaluates the same number with Barill et al.'s fast approximation), inside when above
  0.5.  The two agree except at points within the approximation error of the surface.

``sample_interior`` and ``mesh_particles`` keep the reference's signatures, lattice, seeded jitter and offsets, so the
same mesh and seed give the same candidates.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

ASSETS = os.environ.get("HEATFLOW_ASSETS", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                        "assets"))
BUNNY = os.path.join(ASSETS, "bunny.obj")   # not shipped: set HEATFLOW_ASSETS to a folder holding it


@dataclass
class Mesh:
    """A triangle mesh: vertices (V, 3) float64, faces (F, 3) int64 (0-based)."""
    vertices: np.ndarray
    faces: np.ndarray


def load_obj(path: str) -> Mesh:
    """Vertices and triangles of a Wavefront OBJ file; unreferenced vertices are dropped."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"mesh file {path} not found")
    verts, faces = [], []
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "v" and len(tok) >= 4:
                verts.append((float(tok[1]), float(tok[2]), float(tok[3])))
            elif tok[0] == "f" and len(tok) >= 4:
                idx = []
                for t in tok[1:]:
                    k = int(t.split("/")[0])
                    idx.append(k - 1 if k > 0 else len(verts) + k)
                for a in range(1, len(idx) - 1):          # fan a polygon into triangles
                    faces.append((idx[0], idx[a], idx[a + 1]))
    V = np.asarray(verts, np.float64).reshape(-1, 3)
    F = np.asarray(faces, np.int64).reshape(-1, 3)
    if len(F) == 0:
        raise ValueError(f"{path}: no faces")
    if F.min() < 0 or F.max() >= len(V):
        raise ValueError(f"{path}: face index out of range")
    used, inverse = np.unique(F.ravel(), return_inverse=True)
    return Mesh(V[used], inverse.reshape(-1, 3).astype(np.int64))


def load_mesh(path: str = BUNNY, height: float = 0.10, yaw_deg: float = 0.0, y_up: bool = True) -> Mesh:
    """shapes.py:20-31: the mesh scaled to `height` [m], Z-up, yawed, centred in xy with its lowest point at z = 0."""
    m = load_obj(path)
    v = np.asarray(m.vertices, float)
    if y_up:
        v = np.stack([v[:, 0], -v[:, 2], v[:, 1]], 1)
    c, s = np.cos(np.deg2rad(yaw_deg)), np.sin(np.deg2rad(yaw_deg))
    v = np.stack([c * v[:, 0] - s * v[:, 1], s * v[:, 0] + c * v[:, 1], v[:, 2]], 1)
    v -= v.min(0)
    v *= height / v[:, 2].max()
    v[:, :2] -= v.max(0)[:2] / 2
    return Mesh(v, m.faces)


def winding_inside(mesh: Mesh, points: np.ndarray, threshold: float = 0.5, device="cuda:0",
                   return_winding: bool = False):
    """Inside flags (bool) of float32 points against the mesh by the generalized winding number (hf_winding_inside);
    with return_winding, also the numbers themselves."""
    L = _lib.load()
    dev = torch.device(device)
    tri = torch.as_tensor(np.ascontiguousarray(mesh.vertices.astype(np.float32)[mesh.faces].reshape(-1, 9)), device=dev)
    pts = torch.as_tensor(np.ascontiguousarray(points, np.float32).reshape(-1, 3), device=dev)
    flag = torch.empty(len(pts), dtype=torch.int32, device=dev)
    wind = torch.empty(len(pts), dtype=torch.float32, device=dev) if return_winding else None
    stream = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(L.hf_winding_inside(_lib.ptr(tri), len(tri), _lib.ptr(pts), len(pts), float(threshold), _lib.ptr(flag),
                                   _lib.ptr(wind), stream), "hf_winding_inside")
    inside = flag.cpu().numpy().astype(bool)
    return (inside, wind.cpu().numpy()) if return_winding else inside


def lattice_candidates(mesh: Mesh, spacing: float, jitter: float, rng: np.random.Generator) -> np.ndarray:
    """shapes.py:35-38: the jittered lattice over the mesh's bounds grown by one spacing (float64)."""
    lo, hi = mesh.vertices.min(0) - spacing, mesh.vertices.max(0) + spacing
    axes = [np.arange(lo[d] + spacing / 2, hi[d], spacing) for d in range(3)]
    P = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    return P + rng.uniform(-jitter, jitter, P.shape) * spacing


def sample_interior(mesh: Mesh, spacing: float, jitter: float, rng: np.random.Generator, device: str) -> np.ndarray:
    """shapes.py:34-44: lattice candidates inside the mesh, as float32."""
    P = lattice_candidates(mesh, spacing, jitter, rng)
    keep = winding_inside(mesh, P.astype(np.float32), 0.5, device)
    return P[keep].astype(np.float32)


def mesh_particles(path: str = BUNNY, height: float = 0.10, spacing: float = 2.5e-3, L: float = 0.48, seed: int = 0,
                   yaw_deg: float = 0.0, device: str = "cuda:0") -> np.ndarray:
    """shapes.py:47-51: particles filling the mesh, standing on the floor at the centre of a box of edge L."""
    P = sample_interior(load_mesh(path, height, yaw_deg), spacing, 0.2, np.random.default_rng(seed), device)
    return (P + np.array([L / 2, L / 2, spacing / 2], np.float32)).astype(np.float32)
