"""All-sources wiring costs on the B200 engine, with FastCorticalWiring's result layout.

`WiringAnalysis.compute_all_wiring_costs` is the batched counterpart of
`FastCorticalWiringAnalysis.compute_all_wiring_costs` (core_analysis.py:1441-1672):
the same arguments and validation, the same float32 result arrays over the full
mesh (NaN where not computed), the same health flags, and the same sample CSR
(sample_indptr / sample_radii_flat / sample_areas_flat). Sources run through the
engine in blocks; the per-source samples are assembled on the device.

`save_analysis_npz` writes the reference's NPZ schema v3 (io_utils.py:436-477).
"""

from __future__ import annotations

import json
import os
import time
import warnings

import numpy as np

from . import mesh as M
from .engine import B200DistanceEngine

GEOMETRY_METHOD = "lean_closed_form_v1"  # core_analysis.py:57
MAX_TARGETS = 32                         # scales per run the device kernels hold
MAX_BETWEEN = 8                          # supplementary samples per gap


def classify_nonmanifold_vertices(vertices, faces):
    """Boundary and non-manifold vertices of a triangle mesh (core_analysis.py:60-110).

    Returns sets: boundary_verts (on an edge of one face), non_manifold_verts (on an
    edge of more than two faces), also_boundary (both) and interior (non-manifold only).
    """
    V = np.asarray(vertices)
    F = np.asarray(faces)
    if V.ndim != 2 or V.shape[1] != 3:
        raise ValueError(f"Invalid vertex array shape {V.shape}; expected (N, 3).")
    if F.ndim != 2 or F.shape[1] != 3:
        raise ValueError(f"Invalid face array shape {F.shape}; expected (M, 3).")
    if F.size == 0:
        return {"boundary_verts": set(), "non_manifold_verts": set(), "also_boundary": set(), "interior": set()}
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]]).astype(np.int64)
    e.sort(axis=1)
    edges, counts = np.unique(e, axis=0, return_counts=True)
    boundary = set(np.unique(edges[counts == 1]).tolist())
    non_manifold = set(np.unique(edges[counts > 2]).tolist())
    return {"boundary_verts": boundary, "non_manifold_verts": non_manifold,
            "also_boundary": non_manifold & boundary, "interior": non_manifold - boundary}


def report_components(pm, quiet=False):
    """Print the cortical submesh's connected components, as the reference's analysis does at
    construction (core_analysis.py:1349-1381), unless quiet; returns their sizes, largest
    first. Every source still yields a field over the whole submesh."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    n = pm.n_vertices
    if n == 0:
        if not quiet:
            print("Connected components in cortical submesh: 0")
        return np.zeros(0, dtype=np.int64)
    F = np.asarray(pm.F)
    G = coo_matrix((np.ones(F.size, dtype=np.uint8), (F.ravel(), F[:, [1, 2, 0]].ravel())), shape=(n, n))
    ncomp, label = connected_components(G, directed=False)
    sizes = np.sort(np.bincount(label, minlength=ncomp))[::-1]
    if quiet:
        return sizes
    print(f"Connected components in cortical submesh: {int(ncomp)}")
    if ncomp > 1:
        more = " ..." if ncomp > 20 else ""
        print("Component sizes: " + ", ".join(str(int(x)) for x in sizes[:20]) + more)
    return sizes


def check_interior_nonmanifold(pm, engine_type="b200", allow=False):
    """Count the cortical submesh's interior non-manifold vertices and warn about them unless
    allowed, as the reference does for engines without the robust fallback
    (core_analysis.py:609-636). Returns the count."""
    n = len(classify_nonmanifold_vertices(pm.V, pm.F)["interior"])
    if n and not allow:
        warnings.warn(
            "Interior non-manifold vertices detected in cortical submesh. "
            "Automatic use_robust fallback is only available for the potpourri engine; "
            f"continuing with engine_type={engine_type!r}.",
            RuntimeWarning,
        )
    return n


class WiringAnalysis:
    """A cortical mesh, its B200 engine and the per-vertex wiring metrics.

    The constructor takes FastCorticalWiringAnalysis's arguments (core_analysis.py:545-586):
    engine_type must name this engine ("b200"); metadata is kept; a cortical submesh with
    interior non-manifold vertices warns unless allow_interior_nonmanifold, as the
    reference does for engines without the robust operators (core_analysis.py:609-636).
    precision and block_sources are this engine's own settings.
    """

    # core_analysis.py:536-543
    DEFAULT_SCALES = (0.0006, 0.001, 0.002, 0.004, 0.008, 0.016)

    def __init__(self, vertices, faces, cortex_mask, engine_type="b200", engine_kwargs=None, eps=1e-6,
                 metadata=None, allow_interior_nonmanifold=False, precision="mixed", block_sources=16384):
        key = str(engine_type).strip().lower()
        if key != "b200":
            raise ValueError(f"Unknown engine_type '{engine_type}'. Valid options: b200")
        self.engine_type = key
        self.metadata = dict(metadata or {})
        self.allow_interior_nonmanifold = bool(allow_interior_nonmanifold)
        self.mesh = M.prepare(vertices, faces, cortex_mask)
        pm = self.mesh
        self.n_interior_nonmanifold = check_interior_nonmanifold(pm, self.engine_type,
                                                                 self.allow_interior_nonmanifold)
        self.quiet = getattr(self, "quiet", False)  # no printed reports (a subclass may set it first)
        self.component_sizes = report_components(pm, quiet=self.quiet)
        self.distance_engine = B200DistanceEngine(pm.V, pm.F, **dict(engine_kwargs or {}))
        self.eps = float(eps)
        self.precision = precision
        self.block_sources = int(block_sources)
        self.cortex_mask_full = np.asarray(pm.cortex_mask_full, dtype=bool)
        self.sub_to_orig = np.asarray(pm.sub_to_orig, dtype=np.int32)
        self.orig_to_sub = np.asarray(pm.orig_to_sub)
        self.n_vertices_full = int(self.cortex_mask_full.shape[0])
        self.vertex_areas_sub = pm.vertex_area
        n = self.n_vertices_full
        self.msd_unweighted = np.full(n, np.nan, dtype=np.float32)
        self.msd_weighted = np.full(n, np.nan, dtype=np.float32)
        self.dist_to_boundary = np.full(n, np.nan, dtype=np.float32)
        self.radius_function = {}
        self.perimeter_function = {}
        self.field_flag = np.zeros(n, dtype=np.uint8)
        self.n_flagged_fields = 0
        self.active_scales = ()
        self.n_samples_between_scales = 0
        self.boundary_cap_fraction = None
        self.sample_radii_flat = None
        self.sample_areas_flat = None
        self.sample_indptr = None

    # -- helpers with the reference's semantics ---------------------------
    @staticmethod
    def scale_token(scale):
        """core_analysis.py:754-757."""
        return format(float(scale), "g")

    @staticmethod
    def normalize_scales(scale):
        """core_analysis.py:727-752: an ascending tuple of unique fractions in (0, 1]."""
        if scale is None:
            raw = list(WiringAnalysis.DEFAULT_SCALES)
        elif np.isscalar(scale):
            raw = [scale]
        else:
            raw = list(scale)
        if not raw:
            raise ValueError("At least one scale must be provided.")
        normalized, seen = [], set()
        for item in raw:
            value = float(item)
            if not np.isfinite(value):
                raise ValueError(f"Invalid scale {item!r}: must be finite.")
            if value <= 0.0 or value > 1.0:
                raise ValueError(f"Invalid scale {item!r}: expected 0 < scale <= 1.")
            if value not in seen:
                seen.add(value)
                normalized.append(value)
        normalized.sort()
        return tuple(normalized)

    def _sources(self, vertex_subset):
        """Cortical sub-indices in BFS order, restricted as core_analysis.py:1519-1533 does."""
        order = np.asarray(self.mesh.bfs, dtype=np.int64)
        if vertex_subset is None:
            return order
        keep = np.zeros(self.mesh.n_vertices, dtype=bool)
        for raw in vertex_subset:
            try:
                o = int(raw)
            except Exception:
                continue
            if o < 0 or o >= self.n_vertices_full or not self.cortex_mask_full[o]:
                continue
            s = int(self.orig_to_sub[o])
            if s >= 0:
                keep[s] = True
        return order[keep[order]]

    # -- the computation -----------------------------------------------------
    def compute_all_wiring_costs(self, scale=None, area_tol=None, vertex_subset=None, n_samples_between_scales=3,
                                 boundary_cap_fraction=None, batch_size=None, verbose=False):
        """MSD, distance to boundary, radius, perimeter and (radius, area) samples of every source.

        Arguments and validation follow core_analysis.py:1441-1500; area_tol and batch_size are
        accepted and ignored as there. The engine solves blocks of sources, so verbose prints one
        timing line per block instead of one per source. Prints the end-of-run report and returns
        ((msd_unweighted, msd_weighted), radius_function, perimeter_function), as
        core_analysis.py:1634-1672 does.
        """
        t0 = time.perf_counter()
        scales, m, cap = self.run_arguments(scale, n_samples_between_scales, boundary_cap_fraction)
        targets = self._reset(scales, m, cap)
        order = self._sources(vertex_subset)
        eng = self.distance_engine.engine
        for b0 in range(0, order.size, self.block_sources):
            tb = time.perf_counter()
            sub = order[b0:b0 + self.block_sources]
            rec = eng.compute_metrics(sub, targets, n_between=m, eps=self.eps, precision=self.precision)
            self._absorb(sub, rec, eng.assemble_samples(rec, targets, n_between=m, boundary_cap=cap))
            if verbose:
                print(f"[{b0 + sub.size}/{order.size}] block of {sub.size} sources: "
                      f"{1e3 * (time.perf_counter() - tb):.2f}ms")
        flagged = self._finish(order.size)
        self.report(order.size, flagged, time.perf_counter() - t0)
        return (self.msd_unweighted, self.msd_weighted), self.radius_function, self.perimeter_function

    def report(self, n_sources, flagged, seconds):
        """The end-of-run printout of core_analysis.py:1634-1670: the flagged fields (the first ten
        with their health fractions), the run time, and min/max/mean of MSD, radius and perimeter."""
        if self.quiet:
            return
        if flagged:
            print(f"WARNING: {len(flagged)} of {n_sources} source vertices had corrupted distance fields; "
                  "all metrics for them were set to NaN (see field_flag).")
            for orig_idx, neg, viol in flagged[:10]:
                print(f"  vertex {orig_idx}: negative fraction {neg:.4f}, chord-violation fraction {viol:.4f}")
        if n_sources > 0:
            print(f"Timing over {n_sources} vertices: {seconds:.1f}s ({1e3 * seconds / n_sources:.3f} ms/vertex) "
                  f"on the {getattr(self.distance_engine, 'name', 'b200')} engine, {self.precision}")

        def stats(prefix, values):
            v = values[np.isfinite(values)]
            if v.size:
                print(f"{prefix}min={np.min(v):.2f}, max={np.max(v):.2f}, mean={np.mean(v):.2f}")

        if np.isfinite(self.msd_unweighted).any():
            print("MSD (unweighted, Ecker 2013 definition):")
            stats("  ", self.msd_unweighted)
        if np.isfinite(self.msd_weighted).any():
            print("MSD (area-weighted, resampling-invariant):")
            stats("  ", self.msd_weighted)
        for s in self.active_scales:
            stats(f"Radius stats @ {s * 100:.2f}%: ", self.radius_function[float(s)])
            stats(f"Perimeter stats @ {s * 100:.2f}%: ", self.perimeter_function[float(s)])

    @classmethod
    def run_arguments(cls, scale, n_samples_between_scales, boundary_cap_fraction):
        """Validated (scales, n_between, cap) of a run (core_analysis.py:1441-1500)."""
        scales = cls.normalize_scales(scale)
        m = int(n_samples_between_scales)
        if m < 0:
            raise ValueError("n_samples_between_scales must be >= 0.")
        if boundary_cap_fraction is None:
            cap = None
        else:
            cap = float(boundary_cap_fraction)
            if not np.isfinite(cap) or cap < 0.0 or cap >= 0.5:
                raise ValueError(
                    "boundary_cap_fraction must be in [0, 0.5), or None. "
                    "Values >= 0.5 are not geometrically meaningful; use None for no cap."
                )
        if len(scales) > MAX_TARGETS:
            raise ValueError(f"at most {MAX_TARGETS} scales per run on this engine, got {len(scales)}")
        if m > MAX_BETWEEN:
            raise ValueError(f"n_samples_between_scales must be <= {MAX_BETWEEN} on this engine, got {m}")
        return scales, m, cap

    # -- the steps of compute_all_wiring_costs (also driven by runner.py) ------
    def _reset(self, scales, m, cap):
        """Fresh result arrays for a run; returns the target areas of the scales."""
        n = self.n_vertices_full
        self.active_scales = scales
        self.n_samples_between_scales = m
        self.boundary_cap_fraction = cap
        self.msd_unweighted = np.full(n, np.nan, dtype=np.float32)
        self.msd_weighted = np.full(n, np.nan, dtype=np.float32)
        self.dist_to_boundary = np.full(n, np.nan, dtype=np.float32)
        self.radius_function = {float(s): np.full(n, np.nan, dtype=np.float32) for s in scales}
        self.perimeter_function = {float(s): np.full(n, np.nan, dtype=np.float32) for s in scales}
        self.field_flag = np.zeros(n, dtype=np.uint8)
        self._counts = np.zeros(n, dtype=np.int64)
        self._rows = []
        self._flagged = []
        total_area = float(np.sum(self.vertex_areas_sub))
        return np.array([total_area * float(s) for s in scales], dtype=np.float64)

    def _absorb(self, sub, rec, samples):
        """Records of the cortical sources `sub` (and their assembled samples) into the arrays."""
        nt = len(self.active_scales)
        orig = self.sub_to_orig[sub]
        bad = rec[:, 5] != 0.0
        ok = ~bad
        self.field_flag[orig[bad]] = 1
        self._flagged.extend(zip(orig[bad].tolist(), rec[bad, 3].tolist(), rec[bad, 4].tolist()))
        good = orig[ok]
        self.dist_to_boundary[good] = rec[ok, 2].astype(np.float32)
        self.msd_unweighted[good] = rec[ok, 0].astype(np.float32)
        self.msd_weighted[good] = rec[ok, 1].astype(np.float32)
        for i, s in enumerate(self.active_scales):
            self.radius_function[float(s)][good] = rec[ok, 7 + i].astype(np.float32)
            self.perimeter_function[float(s)][good] = rec[ok, 7 + nt + i].astype(np.float32)
        r, a, c = samples
        self._counts[orig] = c
        self._rows.append((r, a, orig))

    def _finish(self, n_sources):
        """The sample CSR over the full mesh, rows in vertex order (core_analysis.py:1619-1632)."""
        n = self.n_vertices_full
        counts = self._counts
        self.sample_indptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(counts, out=self.sample_indptr[1:])
        total = int(self.sample_indptr[-1])
        self.sample_radii_flat = np.empty(total, dtype=np.float32)
        self.sample_areas_flat = np.empty(total, dtype=np.float32)
        for r, a, orig in self._rows:
            c = counts[orig]
            used = np.arange(r.shape[1])[None, :] < c[:, None]
            dst = (self.sample_indptr[orig][:, None] + np.arange(r.shape[1])[None, :])[used]
            self.sample_radii_flat[dst] = r[used]
            self.sample_areas_flat[dst] = a[used]
        flagged = self._flagged
        self._counts, self._rows, self._flagged = None, None, None
        self.n_flagged_fields = len(flagged)
        if flagged:
            msg = (f"{len(flagged)} of {n_sources} source vertices had corrupted distance fields; "
                   "all metrics for them were set to NaN (see field_flag).")
            warnings.warn(msg, RuntimeWarning)
        return flagged

    # -- results -------------------------------------------------------------
    def provenance(self):
        """core_analysis.py:1674-1687."""
        eng = self.distance_engine
        return {
            "geometry_method": GEOMETRY_METHOD,
            "engine": getattr(eng, "name", "b200"),
            "use_robust": getattr(eng, "use_robust", None),
            "diffusion_length_mm": getattr(eng, "diffusion_length_mm", None),
            "t_coef": getattr(eng, "t_coef", None),
            "mean_edge_length_mm": getattr(eng, "mean_edge_length", None),
            "n_flagged_fields": int(self.n_flagged_fields),
            "health_neg_frac_tol": 1e-3,
            "health_chord_frac_tol": 1e-3,
        }

    def get_metric_arrays(self):
        """core_analysis.py:1693-1705."""
        out = {
            "msd_unweighted": self.msd_unweighted,
            "msd_weighted": self.msd_weighted,
            "dist_to_boundary": self.dist_to_boundary,
        }
        for scale in self.active_scales:
            token = self.scale_token(scale)
            out[f"radius_{token}"] = self.radius_function[float(scale)]
            out[f"perimeter_{token}"] = self.perimeter_function[float(scale)]
        return out

    def get_vertex_samples(self, orig_idx):
        """core_analysis.py:1707-1713: (radii, areas) float32 of one full-mesh vertex."""
        if self.sample_indptr is None:
            return np.empty(0, dtype=np.float32), np.empty(0, dtype=np.float32)
        lo = int(self.sample_indptr[int(orig_idx)])
        hi = int(self.sample_indptr[int(orig_idx) + 1])
        return self.sample_radii_flat[lo:hi], self.sample_areas_flat[lo:hi]


def save_analysis_npz(output_dir, npz_filename, analysis, n_samples_between_scales=None):
    """Scalar metrics plus the sample CSR in the reference's NPZ schema v3 (io_utils.py:436-477)."""
    os.makedirs(output_dir, exist_ok=True)
    path = os.path.join(output_dir, npz_filename)
    payload = dict(analysis.get_metric_arrays())
    m = analysis.n_samples_between_scales if n_samples_between_scales is None else n_samples_between_scales
    cap = getattr(analysis, "boundary_cap_fraction", None)
    payload.update({
        "fastcw_output_schema_version": np.asarray(3, dtype=np.int32),
        "sample_storage_layout": np.asarray("csr_flat_v1"),
        "sample_storage_note": np.asarray(
            "sample_radii_flat/sample_areas_flat are CSR-style rows indexed by sample_indptr[v]:sample_indptr[v+1]."
        ),
        "sample_radii_flat": np.asarray(analysis.sample_radii_flat, dtype=np.float32),
        "sample_areas_flat": np.asarray(analysis.sample_areas_flat, dtype=np.float32),
        "sample_indptr": np.asarray(analysis.sample_indptr, dtype=np.int64),
        "sample_scales_solved": np.asarray(analysis.active_scales, dtype=np.float64),
        "n_samples_between_scales": np.asarray(int(m), dtype=np.int32),
        "boundary_cap_fraction": np.asarray(np.nan if cap is None else float(cap), dtype=np.float64),
        "cortex_mask": np.asarray(analysis.cortex_mask_full, dtype=bool),
        "sub_to_orig": np.asarray(analysis.sub_to_orig, dtype=np.int32),
        "field_health_flag": np.asarray(analysis.field_flag, dtype=np.uint8),
        "provenance_json": np.asarray(json.dumps(analysis.provenance(), sort_keys=True)),
    })
    np.savez_compressed(path, **payload)
    return path
