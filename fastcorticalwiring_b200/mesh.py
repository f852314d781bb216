"""Host-side mesh preparation for the per-source hot path.

Everything here runs once per hemisphere and produces the inputs the device
kernels consume. Each function states the reference code whose result it
reproduces:

* cortical submesh extraction        core_analysis.py:859-911
* per-face area / max edge            core_analysis.py:913-957
* barycentric vertex areas            core_analysis.py:959-978
* boundary vertices (free edges)      core_analysis.py:651-665
* BFS source order over components    core_analysis.py:1336-1417 (1385-1417)
* mean unique-edge length             distance_engines.py:17-21
* lean face metric + bucket width     lean_geometry.py:44-63, 99-114
"""

from __future__ import annotations

from collections import deque
from dataclasses import dataclass, field

import numpy as np


def validate_mesh_inputs(vertices, faces, cortex_mask):
    """Shape/range checks with the reference's error messages (core_analysis.py:771-807)."""
    V = np.asarray(vertices, dtype=np.float64)
    F_raw = np.asarray(faces)
    M = np.asarray(cortex_mask)
    if V.ndim != 2 or V.shape[1] != 3:
        raise ValueError(f"Invalid vertex array shape {V.shape}; expected (N, 3).")
    if F_raw.ndim != 2 or F_raw.shape[1] != 3:
        raise ValueError(f"Invalid face array shape {F_raw.shape}; expected (M, 3).")
    if F_raw.shape[0] == 0:
        raise ValueError("Face array is empty.")
    if M.ndim != 1:
        raise ValueError(f"Invalid cortex mask shape {M.shape}; expected (N,).")
    if M.shape[0] != V.shape[0]:
        raise ValueError(f"Mask length mismatch: mask has {M.shape[0]} entries, vertices has {V.shape[0]}.")
    if not np.issubdtype(F_raw.dtype, np.integer):
        if np.any(np.abs(F_raw - np.rint(F_raw)) > 0):
            raise ValueError("Face indices must be integers.")
        F = np.rint(F_raw).astype(np.int32)
    else:
        F = F_raw.astype(np.int32, copy=False)
    if np.any(F < 0):
        raise ValueError("Face indices contain negative values.")
    if np.any(F >= V.shape[0]):
        raise ValueError(
            f"Face indices out of range: max face index {int(np.max(F))}, "
            f"but only {V.shape[0]} vertices provided.")
    M = M.astype(bool, copy=False)
    if not np.any(M):
        raise ValueError("Cortex mask is empty (no True vertices).")
    return V, F, M


def cortex_submesh(vertices, faces, cortex_mask):
    """Faces with all corners cortical and area > 1e-12, re-indexed to used vertices.

    Returns (V_sub, F_sub int32, sub_to_orig int32, orig_to_sub int32 with -1).
    Follows core_analysis.py:859-911.
    """
    keep = cortex_mask[faces].all(axis=1)
    Fk = faces[keep]
    nfull = vertices.shape[0]
    empty = (np.empty((0, 3)), np.empty((0, 3), np.int32), np.empty(0, np.int32),
             np.full(nfull, -1, np.int32))
    if Fk.shape[0] == 0:
        return empty
    p0, p1, p2 = vertices[Fk[:, 0]], vertices[Fk[:, 1]], vertices[Fk[:, 2]]
    area = 0.5 * np.linalg.norm(np.cross(p1 - p0, p2 - p0), axis=1)
    Fk = Fk[area > 1e-12]
    if Fk.shape[0] == 0:
        return empty
    used = np.unique(Fk)
    sub_to_orig = used.astype(np.int32)
    orig_to_sub = np.full(nfull, -1, dtype=np.int32)
    orig_to_sub[sub_to_orig] = np.arange(sub_to_orig.shape[0], dtype=np.int32)
    return vertices[sub_to_orig], orig_to_sub[Fk].astype(np.int32), sub_to_orig, orig_to_sub


def face_areas_and_max_edge(V, F):
    """Per-face area (0 for degenerate) and longest edge (core_analysis.py:913-957)."""
    p0, p1, p2 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    e01, e12, e20 = p1 - p0, p2 - p1, p0 - p2
    nrm = np.linalg.norm(np.cross(e01, p2 - p0), axis=1)
    Lmax = np.maximum.reduce([np.linalg.norm(e01, axis=1), np.linalg.norm(e12, axis=1),
                              np.linalg.norm(e20, axis=1)])
    tiny = np.finfo(np.float64).eps * (Lmax * Lmax) * 10.0
    area = 0.5 * nrm
    area[nrm < tiny] = 0.0
    return area, Lmax


def vertex_areas(nv, F, face_area):
    """One third of each incident face's area (core_analysis.py:959-978).

    The reference adds the three corners of each face before moving to the
    next face; np.add.at over the flattened face array applies the additions
    in that same order, so the sums agree bit for bit.
    """
    a = np.zeros(nv, dtype=np.float64)
    third = face_area / 3.0
    flat = F.reshape(-1)
    np.add.at(a, flat, np.repeat(third, 3))
    return a


def _edge_keys(F):
    """Undirected edges of the faces as sorted int64 keys lo * n + hi (n = max vertex id + 1)."""
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0).astype(np.int64)
    e.sort(axis=1)
    n = int(F.max()) + 1 if F.size else 1
    return np.sort(e[:, 0] * n + e[:, 1]), n


def boundary_vertices(F):
    """Vertices on free edges (edges used by exactly one face), sorted (core_analysis.py:651-665)."""
    key, n = _edge_keys(F)
    if key.size == 0:
        return np.empty(0, dtype=np.int32)
    first = np.ones(key.size, dtype=bool)
    first[1:] = key[1:] != key[:-1]
    starts = np.flatnonzero(first)
    cnt = np.diff(np.append(starts, key.size))
    be = key[starts[cnt == 1]]
    if be.size == 0:
        return np.empty(0, dtype=np.int32)
    return np.unique(np.concatenate([be // n, be % n])).astype(np.int32)


def mean_edge_length(V, F):
    """Mean length over unique undirected edges (distance_engines.py:17-21)."""
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0).astype(np.int64)
    e.sort(axis=1)
    e = np.unique(e, axis=0)
    return float(np.mean(np.linalg.norm(V[e[:, 1]] - V[e[:, 0]], axis=1)))


def vertex_adjacency_csr(nv, F):
    """Sorted neighbour lists as CSR (indptr int64, indices int32)."""
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]],
                        F[:, [1, 0]], F[:, [2, 1]], F[:, [0, 2]]], axis=0).astype(np.int64)
    key = np.sort(e[:, 0] * nv + e[:, 1])
    if key.size:
        keep = np.ones(key.size, dtype=bool)
        keep[1:] = key[1:] != key[:-1]
        key = key[keep]
    rows = key // nv
    cols = (key % nv).astype(np.int32)
    indptr = np.zeros(nv + 1, dtype=np.int64)
    indptr[1:] = np.cumsum(np.bincount(rows, minlength=nv))
    return indptr, cols


def bfs_order(nv, F, start=0):
    """BFS over all components, neighbours in ascending order (core_analysis.py:1385-1417).

    Level by level: the next frontier is the frontier's neighbour lists, in frontier
    order, unvisited, each vertex at its first appearance -- exactly the order a FIFO
    queue visits them in.
    """
    indptr, nbr = vertex_adjacency_csr(nv, F)
    visited = np.zeros(nv, dtype=bool)
    order = []
    deg = np.diff(indptr)

    def run(s):
        visited[s] = True
        front = np.array([s], dtype=np.int64)
        while front.size:
            order.append(front)
            d = deg[front]
            tot = int(d.sum())
            if tot == 0:
                break
            # positions of the frontier's neighbour lists, concatenated in frontier order
            off = np.repeat(indptr[front] - np.cumsum(d) + d, d) + np.arange(tot)
            cand = nbr[off].astype(np.int64)
            cand = cand[~visited[cand]]
            if cand.size == 0:
                break
            _, first = np.unique(cand, return_index=True)
            front = cand[np.sort(first)]
            visited[front] = True

    s0 = int(start) if 0 <= int(start) < nv else 0
    if nv:
        run(s0)
        nxt = 0
        while True:
            rest = np.flatnonzero(~visited[nxt:])
            if rest.size == 0:
                break
            nxt += int(rest[0])
            run(nxt)
    return np.concatenate(order) if order else np.empty(0, dtype=np.int64)


def lean_face_metric(V, F):
    """Face area and inverse-Gram coefficients g11, g12, g22 (lean_geometry.py:44-63)."""
    e1 = V[F[:, 1]] - V[F[:, 0]]
    e2 = V[F[:, 2]] - V[F[:, 0]]
    a11 = np.einsum("ij,ij->i", e1, e1)
    a22 = np.einsum("ij,ij->i", e2, e2)
    a12 = np.einsum("ij,ij->i", e1, e2)
    det = a11 * a22 - a12 * a12
    area = 0.5 * np.sqrt(np.maximum(det, 0.0))
    inv = np.zeros_like(det)
    good = det > 0.0
    inv[good] = 1.0 / det[good]
    return area, a22 * inv, -a12 * inv, a11 * inv


def lean_bin_width(V, F, quantile=0.999, pad=1.05):
    """Bucket width: 0.999 quantile of per-face max edge, padded 5% (lean_geometry.py:99-114)."""
    L = np.maximum.reduce([
        np.linalg.norm(V[F[:, 1]] - V[F[:, 0]], axis=1),
        np.linalg.norm(V[F[:, 2]] - V[F[:, 1]], axis=1),
        np.linalg.norm(V[F[:, 0]] - V[F[:, 2]], axis=1),
    ])
    return float(np.quantile(L, quantile) * pad)


# The batch runner's default 12 log-spaced area fractions (run_pipeline.py:249-266).
RUNNER_SCALES = (0.00200000, 0.00267988, 0.00359088, 0.00481157, 0.00644721, 0.00863888,
                 0.01157558, 0.01551059, 0.02078326, 0.02784833, 0.03731509, 0.05000000)


def default_scales():
    return RUNNER_SCALES


@dataclass
class PreparedMesh:
    """Cortical submesh plus every per-mesh array the hot path reads."""
    vertices_full: np.ndarray
    faces_full: np.ndarray
    cortex_mask_full: np.ndarray
    V: np.ndarray
    F: np.ndarray
    sub_to_orig: np.ndarray
    orig_to_sub: np.ndarray
    face_area: np.ndarray
    face_L: np.ndarray
    vertex_area: np.ndarray
    boundary: np.ndarray
    health_h: float
    lean_area: np.ndarray
    g11: np.ndarray
    g12: np.ndarray
    g22: np.ndarray
    bin_width: float
    _bfs: np.ndarray | None = field(default=None, repr=False)

    @property
    def n_vertices(self):
        return int(self.V.shape[0])

    @property
    def n_faces(self):
        return int(self.F.shape[0])

    @property
    def bfs(self):
        if self._bfs is None:
            self._bfs = bfs_order(self.n_vertices, self.F, 0)
        return self._bfs

    def targets(self, scales):
        total = float(np.sum(self.vertex_area))
        return np.array([total * float(s) for s in scales], dtype=np.float64)


def prepare(vertices, faces, cortex_mask) -> PreparedMesh:
    """Validate, cut the cortical submesh and precompute per-mesh arrays."""
    Vf, Ff, Mf = validate_mesh_inputs(vertices, faces, cortex_mask)
    V, F, s2o, o2s = cortex_submesh(Vf, Ff, Mf)
    if V.shape[0] == 0:
        raise ValueError("Cortex mask produced an empty cortical submesh.")
    if F.shape[0] == 0:
        raise ValueError("No valid cortical faces remain after applying cortex mask.")
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int32)
    fa, fL = face_areas_and_max_edge(V, F)
    va = vertex_areas(V.shape[0], F, fa)
    la, g11, g12, g22 = lean_face_metric(V, F)
    return PreparedMesh(
        vertices_full=Vf, faces_full=Ff, cortex_mask_full=Mf, V=V, F=F,
        sub_to_orig=s2o, orig_to_sub=o2s, face_area=fa, face_L=fL, vertex_area=va,
        boundary=boundary_vertices(F), health_h=float(np.median(fL)),
        lean_area=np.ascontiguousarray(la), g11=np.ascontiguousarray(g11),
        g12=np.ascontiguousarray(g12), g22=np.ascontiguousarray(g22),
        bin_width=float(np.quantile(fL, 0.999) * 1.05),  # lean_bin_width(V, F): the same edge lengths
    )
