"""Batch runner: many subjects through the serving loop, one analysis NPZ per subject.

run_pipeline.py fans subjects out as one fastcw.py process per host core
(run_pipeline.py:102-131, 326-342). Here every subject is a job of one
serving.Server: the jobs' factors and source blocks stay resident on one GPU
under an HBM budget and their blocks overlap on the device. Each subject's
results are the arrays of WiringAnalysis.compute_all_wiring_costs over all its
cortical sources, written with save_analysis_npz (the reference's schema v3,
io_utils.py:436-477), as the per-subject command line writes them.

A subject is a mesh in an .npz file with `vertices` (n x 3), `faces` (m x 3)
and `cortex_mask` (n, bool); reading FreeSurfer or GIFTI surfaces stays with
the reference's io_utils.

    python -m fastcorticalwiring_b200.runner --out results/ lh_01.npz lh_02.npz ...
    python -m fastcorticalwiring_b200.runner --out results/ --manifest subjects.json

A manifest is a JSON list of {"name": ..., "mesh": path} (paths relative to the
manifest's folder). A subject whose mesh cannot be read or prepared is reported
and skipped, as run_pipeline.py:124-131 logs failed subjects and continues.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

from . import analysis as A
from . import engine as E
from . import mesh as M
from . import serving as S


class SubjectAnalysis(A.WiringAnalysis):
    """WiringAnalysis results filled from a serving job's records (no engine of its own)."""

    def __init__(self, pm: M.PreparedMesh, engine_info: dict, diffusion_length_mm: float, eps=1e-6,
                 precision="mixed", metadata=None, allow_interior_nonmanifold=False):
        self.mesh = pm
        self.distance_engine = None
        self.engine_type = "b200"
        self.metadata = dict(metadata or {})
        self.allow_interior_nonmanifold = bool(allow_interior_nonmanifold)
        self.n_interior_nonmanifold = A.check_interior_nonmanifold(pm, self.engine_type,
                                                                   self.allow_interior_nonmanifold)
        self._engine_info = dict(engine_info or {})
        self._diffusion_length_mm = float(diffusion_length_mm)
        self.eps = float(eps)
        self.precision = precision
        self.cortex_mask_full = np.asarray(pm.cortex_mask_full, dtype=bool)
        self.sub_to_orig = np.asarray(pm.sub_to_orig, dtype=np.int32)
        self.orig_to_sub = np.asarray(pm.orig_to_sub)
        self.n_vertices_full = int(self.cortex_mask_full.shape[0])
        self.vertex_areas_sub = pm.vertex_area
        self.n_flagged_fields = 0
        self.active_scales = ()
        self.n_samples_between_scales = 0
        self.boundary_cap_fraction = None
        self.sample_radii_flat = self.sample_areas_flat = self.sample_indptr = None

    def provenance(self):
        """core_analysis.py:1674-1687, with the job's engine parameters."""
        return {
            "geometry_method": A.GEOMETRY_METHOD,
            "engine": "b200",
            "use_robust": False,
            "diffusion_length_mm": self._diffusion_length_mm,
            "t_coef": self._engine_info.get("t_coef"),
            "mean_edge_length_mm": self._engine_info.get("mean_edge_length"),
            "n_flagged_fields": int(self.n_flagged_fields),
            "health_neg_frac_tol": 1e-3,
            "health_chord_frac_tol": 1e-3,
        }


def load_mesh(path):
    """(vertices, faces, cortex_mask) from an .npz subject file."""
    with np.load(path) as z:
        missing = {"vertices", "faces", "cortex_mask"} - set(z.files)
        if missing:
            raise ValueError(f"{path}: missing arrays {sorted(missing)}")
        return (np.asarray(z["vertices"], dtype=np.float64), np.asarray(z["faces"], dtype=np.int32),
                np.asarray(z["cortex_mask"], dtype=bool))


def load_manifest(path):
    """[(name, mesh path)] from a JSON list of {"name", "mesh"}; paths relative to the manifest."""
    with open(path) as f:
        items = json.load(f)
    if not isinstance(items, list):
        raise ValueError("the manifest must be a JSON list of {\"name\": ..., \"mesh\": ...}")
    base = os.path.dirname(os.path.abspath(path))
    out, seen = [], set()
    for it in items:
        if not isinstance(it, dict) or "mesh" not in it:
            raise ValueError(f"manifest entry without a mesh: {it!r}")
        mesh = it["mesh"] if os.path.isabs(it["mesh"]) else os.path.join(base, it["mesh"])
        name = str(it.get("name") or os.path.splitext(os.path.basename(mesh))[0])
        if name in seen:
            raise ValueError(f"duplicate subject name {name!r}")
        seen.add(name)
        out.append((name, mesh))
    return out


def run_subjects(subjects, output_dir, scale=None, n_samples_between_scales=3, boundary_cap_fraction=None,
                 precision="mixed", hbm_budget_gb=150.0, device=0, engine_params=None, log=None):
    """Run [(name, mesh path or (vertices, faces, cortex_mask))] and write `<name>.npz` per subject.

    Returns {"written": {name: path}, "failed": {name: message}, "sources_per_s": ..., "jobs": [...]}.
    """
    scales, m, cap = A.WiringAnalysis.run_arguments(scale, n_samples_between_scales, boundary_cap_fraction)
    names = [name for name, _ in subjects]
    if len(set(names)) != len(names):
        raise ValueError("subject names must be unique")
    log = log or (lambda msg: None)
    prepared, failed = {}, {}
    jobs = []
    for name, src in subjects:
        try:
            V, F, mask = load_mesh(src) if isinstance(src, (str, os.PathLike)) else src
            pm = M.prepare(V, F, mask)
        except Exception as exc:  # a subject that cannot be read is skipped (run_pipeline.py:124-131)
            failed[name] = f"{type(exc).__name__}: {exc}"
            log(f"[skip] {name}: {failed[name]}")
            continue
        prepared[name] = pm
        jobs.append((0.0, S.Job(name, pm.V, pm.F, np.ones(pm.n_vertices, dtype=bool), scales=scales, n_between=m,
                                precision=precision, prepared=pm)))
    written = {}
    report = []
    if jobs:
        server = S.Server(hbm_budget_bytes=float(hbm_budget_gb) * 1e9, device=device, engine_params=engine_params)
        t0 = time.perf_counter()
        try:
            results = server.run(jobs)
        finally:
            server.close()
        span = time.perf_counter() - t0
        params = E.ENGINE_DEFAULTS.copy()
        params.update(engine_params or {})
        diffusion = float(params.get("diffusion_length_mm", E.DEFAULT_DIFFUSION_LENGTH_MM))
        for name, pm in prepared.items():
            res = results[name]
            sa = SubjectAnalysis(pm, res.engine_info, diffusion, precision=precision, metadata={"subject": name})
            targets = sa._reset(scales, m, cap)
            sa._absorb(res.sources, res.records,
                       E.assemble_samples_device(res.records, targets, m, cap, device=device))
            sa._finish(res.sources.size)
            written[name] = A.save_analysis_npz(output_dir, f"{name}.npz", sa, m)
            report.append({"name": name, "sources": int(res.sources.size), "latency_s": res.latency_s,
                           "flagged": int(sa.n_flagged_fields)})
            log(f"[done] {name}: {res.sources.size} sources in {res.latency_s:.2f} s -> {written[name]}")
        total = sum(r["sources"] for r in report)
        rate = total / span if span > 0 else 0.0
    else:
        rate = 0.0
    return {"written": written, "failed": failed, "sources_per_s": rate, "jobs": report}


def main(argv=None):
    ap = argparse.ArgumentParser(description="All-sources wiring metrics for many subjects on one GPU.")
    ap.add_argument("meshes", nargs="*", help=".npz subject meshes (vertices, faces, cortex_mask)")
    ap.add_argument("--manifest", help="JSON list of {\"name\", \"mesh\"}")
    ap.add_argument("--out", required=True, help="output folder (one <name>.npz per subject)")
    ap.add_argument("--scales", default=None,
                    help="comma-separated area fractions (default: the analysis default scales)")
    ap.add_argument("--n-samples-between-scales", type=int, default=3)
    ap.add_argument("--boundary-cap-fraction", type=float, default=None)
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    subjects = load_manifest(args.manifest) if args.manifest else []
    subjects += [(os.path.splitext(os.path.basename(p))[0], p) for p in args.meshes]
    if not subjects:
        ap.error("no subjects: give .npz meshes or --manifest")
    names = [n for n, _ in subjects]
    if len(set(names)) != len(names):
        ap.error("subject names must be unique")
    scales = None if args.scales is None else [float(x) for x in args.scales.split(",") if x.strip()]
    out = run_subjects(subjects, args.out, scale=scales, n_samples_between_scales=args.n_samples_between_scales,
                       boundary_cap_fraction=args.boundary_cap_fraction, precision=args.precision,
                       hbm_budget_gb=args.hbm_budget_gb, device=args.device,
                       log=lambda msg: print(msg, file=sys.stderr, flush=True))
    print(json.dumps({"written": out["written"], "failed": out["failed"], "sources_per_s": out["sources_per_s"]}))
    return 1 if out["failed"] and not out["written"] else 0


if __name__ == "__main__":
    sys.exit(main())
