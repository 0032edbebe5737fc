"""Triangle meshes for the AIFMM solver: readers/writers for the reference's
``nodeList<N>.txt`` / ``patchList<N>.txt`` text format and deterministic
generators for the synthetic workloads (icospheres and ellipsoids).

Format (vaishna77/RCS src/EFIEMatrix.cpp:31-44 and :72-95): one vertex per
line ``x y z``; one triangle per line ``v1 v2 v3 [conductor]`` with ONE-based
vertex ids.  Arrays in this module follow that convention: ``nodes`` is an
``(nv, 3)`` float64 array and ``tris`` an ``(nt, 3)`` int32 array of one-based
vertex ids, so that the RWG numbering built from them is the reference's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh:
    nodes: np.ndarray  # (nv, 3) float64
    tris: np.ndarray  # (nt, 3) int32, one-based vertex ids
    cond: np.ndarray | None = None  # (nt,) conductor index per triangle

    @property
    def n_nodes(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def n_tris(self) -> int:
        return int(self.tris.shape[0])


def read_mesh(node_file: str, patch_file: str) -> Mesh:
    nodes = []
    with open(node_file) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3:
                nodes.append([float(p) for p in parts[:3]])
    tris, cond = [], []
    with open(patch_file) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3:
                tris.append([int(p) for p in parts[:3]])
                cond.append(int(parts[3]) if len(parts) > 3 else 0)
    return Mesh(np.asarray(nodes, dtype=np.float64), np.asarray(tris, dtype=np.int32),
                np.asarray(cond, dtype=np.int32))


def write_mesh(mesh: Mesh, node_file: str, patch_file: str) -> None:
    with open(node_file, "w") as f:
        for x, y, z in mesh.nodes:
            f.write(f"{x:.18e} {y:.18e} {z:.18e}\n")
    with open(patch_file, "w") as f:
        for t, (a, b, c) in enumerate(mesh.tris):
            if mesh.cond is not None:
                f.write(f"{a} {b} {c} {int(mesh.cond[t])}\n")
            else:
                f.write(f"{a} {b} {c}\n")


def icosphere(subdivisions: int, radius: float = 1.0) -> Mesh:
    """Regular icosahedron (12 golden-ratio vertices, 20 faces, outward
    orientation) refined ``subdivisions`` times by 4:1 midpoint splits, every
    new vertex projected back to the sphere.  Triangles: 20*4^s; closed
    surface so every edge is an RWG edge: N = 1.5 * triangles."""
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, phi, 0), (1, phi, 0), (-1, -phi, 0), (1, -phi, 0),
         (0, -1, phi), (0, 1, phi), (0, -1, -phi), (0, 1, -phi),
         (phi, 0, -1), (phi, 0, 1), (-phi, 0, -1), (-phi, 0, 1)]
    verts = [np.asarray(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            idx = cache.get(key)
            if idx is None:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                idx = len(verts) - 1
                cache[key] = idx
            return idx

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    nodes = np.stack(verts) * radius
    tris = np.asarray(faces, dtype=np.int32) + 1
    return Mesh(nodes, tris, np.ones(len(faces), dtype=np.int32))


def ellipsoid(subdivisions: int, axes: tuple[float, float, float]) -> Mesh:
    """Unit icosphere scaled by the semi-axes (a, b, c)."""
    m = icosphere(subdivisions, 1.0)
    m.nodes = m.nodes * np.asarray(axes, dtype=np.float64)[None, :]
    return m


def rwg_count(mesh: Mesh) -> int:
    """Number of RWG unknowns: edges shared by at least two triangles
    (EFIEMatrix.cpp:199-209 keeps every edge with more than one patch)."""
    t = mesh.tris
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    e.sort(axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    return int((counts > 1).sum())
