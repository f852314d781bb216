"""Seeded synthetic hemisphere meshes: folded icospheres with a medial-wall cap.

The workloads this engine is measured on are synthetic stand-ins for cortical
surfaces (no subject data ships with the project):

* an order-``level`` icosphere (10*4**level + 2 vertices), radius 70 mm;
* radially folded, r = R * (1 + 0.15 * sum_{l=4..12} sum_m a_lm Y_lm) with
  a_lm ~ N(0, 1) / l drawn from the job seed (real spherical harmonics);
* optionally jittered in the tangent plane by up to ``jitter`` x the mean edge
  length before folding, which gives irregular (non-Delaunay) triangles;
* a spherical cap holding ``cap_fraction`` of the vertices is masked out as the
  "medial wall", so the cortical submesh has a boundary.

The returned ``cortex_mask`` plays the role of the FreeSurfer cortex label that
``io_utils.load_surface_and_mask`` returns in the reference pipeline.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_PHI = (1.0 + 5.0 ** 0.5) / 2.0
_BASE_V = np.array(
    [(-1, _PHI, 0), (1, _PHI, 0), (-1, -_PHI, 0), (1, -_PHI, 0),
     (0, -1, _PHI), (0, 1, _PHI), (0, -1, -_PHI), (0, 1, -_PHI),
     (_PHI, 0, -1), (_PHI, 0, 1), (-_PHI, 0, -1), (-_PHI, 0, 1)], dtype=np.float64)
_BASE_F = np.array(
    [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
     (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
     (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)


def unit_icosphere(level: int):
    """Unit icosphere by ``level`` rounds of 1:4 midpoint subdivision.

    Returns (V float64 (10*4**level+2, 3), F int32 (20*4**level, 3)), outward
    oriented. Each round adds one vertex per edge, projected to the sphere.
    """
    V = _BASE_V / np.linalg.norm(_BASE_V, axis=1, keepdims=True)
    F = _BASE_F.copy()
    for _ in range(int(level)):
        nF = F.shape[0]
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0)
        e.sort(axis=1)
        key = e[:, 0] * (V.shape[0] + 1) + e[:, 1]
        uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
        ue = e[first]
        mid = V[ue[:, 0]] + V[ue[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = V.shape[0]
        V = np.concatenate([V, mid], axis=0)
        m01 = inv[:nF] + base
        m12 = inv[nF:2 * nF] + base
        m20 = inv[2 * nF:] + base
        F = np.concatenate([
            np.stack([F[:, 0], m01, m20], axis=1),
            np.stack([F[:, 1], m12, m01], axis=1),
            np.stack([F[:, 2], m20, m12], axis=1),
            np.stack([m01, m12, m20], axis=1),
        ], axis=0)
    return V, F.astype(np.int32)


def _real_sph_harm(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    from scipy.special import sph_harm_y

    if m == 0:
        return np.real(sph_harm_y(l, 0, theta, phi))
    y = sph_harm_y(l, abs(m), theta, phi)
    return np.sqrt(2.0) * (np.real(y) if m > 0 else np.imag(y))


def _mean_edge(V, F):
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0).astype(np.int64)
    e.sort(axis=1)
    e = np.unique(e, axis=0)
    return float(np.mean(np.linalg.norm(V[e[:, 1]] - V[e[:, 0]], axis=1)))


@dataclass
class HemisphereMesh:
    vertices: np.ndarray      # (N, 3) float64, mm
    faces: np.ndarray         # (M, 3) int32
    cortex_mask: np.ndarray   # (N,) bool; False on the medial-wall cap
    level: int
    seed: int
    jitter: float


def folded_icosphere(level: int, seed: int = 0, radius: float = 70.0, amplitude: float = 0.15,
                     lmin: int = 4, lmax: int = 12, jitter: float = 0.0,
                     cap_fraction: float = 0.10) -> HemisphereMesh:
    """Seeded folded icosphere with a medial-wall cap (see module docstring)."""
    rng = np.random.default_rng(int(seed))
    V, F = unit_icosphere(level)
    if jitter > 0.0:
        h = _mean_edge(V, F)
        g = rng.standard_normal(V.shape)
        g -= np.sum(g * V, axis=1, keepdims=True) * V
        g /= np.maximum(np.linalg.norm(g, axis=1, keepdims=True), 1e-300)
        mag = rng.uniform(0.0, float(jitter) * h, size=(V.shape[0], 1))
        V = V + mag * g
        V /= np.linalg.norm(V, axis=1, keepdims=True)
    theta = np.arccos(np.clip(V[:, 2], -1.0, 1.0))
    phi = np.arctan2(V[:, 1], V[:, 0])
    s = np.zeros(V.shape[0])
    for l in range(lmin, lmax + 1):
        for m in range(-l, l + 1):
            s += (rng.standard_normal() / l) * _real_sph_harm(l, m, theta, phi)
    r = radius * (1.0 + amplitude * s)
    centre = rng.standard_normal(3)
    centre /= np.linalg.norm(centre)
    closeness = V @ centre
    n_cap = int(round(cap_fraction * V.shape[0]))
    mask = np.ones(V.shape[0], dtype=bool)
    if n_cap > 0:
        mask[np.argsort(-closeness, kind="stable")[:n_cap]] = False
    return HemisphereMesh(V * r[:, None], F, mask, int(level), int(seed), float(jitter))


# The measured workloads: order-5/6/7/8 folded icospheres (jitter on 6 and 8).
WORKLOADS = {
    "L5": dict(level=5, jitter=0.0),
    "L6": dict(level=6, jitter=0.2),
    "L7": dict(level=7, jitter=0.0),
    "L8": dict(level=8, jitter=0.2),
}


def workload_mesh(name: str, seed: int = 0) -> HemisphereMesh:
    cfg = WORKLOADS[name]
    return folded_icosphere(cfg["level"], seed=seed, jitter=cfg["jitter"])
