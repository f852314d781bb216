"""Per-vertex (radius, area) sample assembly -- CPU restatement for the tests.

TEST INFRASTRUCTURE ONLY (what the device assembly kernel is compared with).

Restates, from the reference's core_analysis.py:
  * FastCorticalWiringAnalysis.boundary_area_loss_fraction   (core_analysis.py:759-777)
  * FastCorticalWiringAnalysis._clean_vertex_samples         (core_analysis.py:1424-1439)
  * the per-source pair list and boundary cap                 (core_analysis.py:1599-1611)
  * the CSR layout of the flat sample arrays                  (core_analysis.py:1619-1632)

Pinned against golden_samples_L5.npz, written by the reference's own code.
"""

from __future__ import annotations

import math

import numpy as np


def boundary_area_loss_fraction(radius, boundary_distance):
    """Disc-area fraction cut off by a straight boundary at distance d from the centre."""
    r = float(radius)
    d = float(boundary_distance)
    if not math.isfinite(r) or r <= 0.0:
        return math.nan
    if not math.isfinite(d):
        return 0.0
    if d >= r:
        return 0.0
    x = min(1.0, max(0.0, d / r))
    # NumPy's arccos/sqrt, as the reference evaluates them (bit-identical results)
    return float((np.arccos(x) - x * np.sqrt(max(0.0, 1.0 - x * x))) / np.pi)


def clean_vertex_samples(pairs):
    """Stable sort by radius; drop radii within max(1e-12, 1e-9 * span) of their predecessor."""
    if not pairs:
        return []
    arr = np.asarray(pairs, dtype=np.float64)
    arr = arr[np.argsort(arr[:, 0], kind="stable")]
    if arr.shape[0] == 1:
        return [(float(arr[0, 0]), float(arr[0, 1]))]
    r = arr[:, 0]
    tol = max(1e-12, 1e-9 * float(r[-1] - r[0]))
    keep = np.empty(arr.shape[0], dtype=bool)
    keep[0] = True
    keep[1:] = np.diff(r) > tol
    return [(float(a), float(b)) for a, b in arr[keep]]


def vertex_samples(radii, targets, extra_r, extra_a, dist_to_boundary_f32, cap=None):
    """The cleaned (radius, area) pairs of one healthy source.

    radii / targets: the solved scales; extra_r / extra_a: the supplementary samples;
    dist_to_boundary_f32: the float32 value the analysis stored for the source.
    """
    pairs = [(float(r), float(a)) for r, a in zip(radii, targets) if np.isfinite(r)]
    extra_r = np.asarray(extra_r, np.float64)
    extra_a = np.asarray(extra_a, np.float64)
    if extra_r.size:
        ok = np.isfinite(extra_r) & np.isfinite(extra_a)
        if cap is not None:
            d_b = float(np.float32(dist_to_boundary_f32))
            for j in np.flatnonzero(ok):
                if boundary_area_loss_fraction(float(extra_r[j]), d_b) > cap:
                    ok[j] = False
        pairs.extend(zip(extra_r[ok].tolist(), extra_a[ok].tolist()))
    return clean_vertex_samples(pairs)


def csr(rows, n):
    """rows: {vertex: list of pairs} -> (indptr int64 (n+1,), radii float32, areas float32)."""
    indptr = np.zeros(n + 1, dtype=np.int64)
    for i in range(n):
        indptr[i + 1] = indptr[i] + len(rows.get(i) or [])
    r = np.empty(int(indptr[-1]), dtype=np.float32)
    a = np.empty(int(indptr[-1]), dtype=np.float32)
    for i, row in rows.items():
        if row:
            lo = int(indptr[i])
            r[lo:lo + len(row)] = np.asarray([x[0] for x in row], dtype=np.float32)
            a[lo:lo + len(row)] = np.asarray([x[1] for x in row], dtype=np.float32)
    return indptr, r, a
