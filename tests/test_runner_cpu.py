"""Batch runner host logic (no GPU): subject manifests, mesh files and skipped subjects."""
import json
import os

import numpy as np
import pytest

from fastcorticalwiring_b200 import runner


def test_manifest_paths_names_and_duplicates(tmp_path):
    (tmp_path / "sub").mkdir()
    man = tmp_path / "subjects.json"
    man.write_text(json.dumps([{"name": "a", "mesh": "sub/a.npz"}, {"mesh": "/abs/b.npz"}]))
    got = runner.load_manifest(str(man))
    assert got == [("a", os.path.join(str(tmp_path), "sub/a.npz")), ("b", "/abs/b.npz")]
    man.write_text(json.dumps([{"name": "a", "mesh": "x.npz"}, {"name": "a", "mesh": "y.npz"}]))
    with pytest.raises(ValueError, match="duplicate"):
        runner.load_manifest(str(man))
    man.write_text(json.dumps({"name": "a"}))
    with pytest.raises(ValueError, match="JSON list"):
        runner.load_manifest(str(man))
    man.write_text(json.dumps([{"name": "a"}]))
    with pytest.raises(ValueError, match="without a mesh"):
        runner.load_manifest(str(man))


def test_mesh_file_arrays(tmp_path):
    p = tmp_path / "m.npz"
    np.savez(p, vertices=np.zeros((3, 3)), faces=np.array([[0, 1, 2]]), cortex_mask=np.ones(3, bool))
    V, F, mask = runner.load_mesh(str(p))
    assert V.dtype == np.float64 and F.dtype == np.int32 and mask.dtype == bool
    np.savez(p, vertices=np.zeros((3, 3)), faces=np.array([[0, 1, 2]]))
    with pytest.raises(ValueError, match="cortex_mask"):
        runner.load_mesh(str(p))


def test_unreadable_subjects_are_skipped_without_a_device(tmp_path):
    out = runner.run_subjects([("gone", str(tmp_path / "missing.npz"))], str(tmp_path / "out"))
    assert out["written"] == {} and "gone" in out["failed"]


def test_duplicate_subject_names_are_rejected(tmp_path):
    with pytest.raises(ValueError, match="unique"):
        runner.run_subjects([("a", "x.npz"), ("a", "y.npz")], str(tmp_path))


def test_run_arguments_follow_the_analysis_rules(tmp_path):
    with pytest.raises(ValueError, match="boundary_cap_fraction"):
        runner.run_subjects([], str(tmp_path), boundary_cap_fraction=0.5)
    with pytest.raises(ValueError, match="n_samples_between_scales"):
        runner.run_subjects([], str(tmp_path), n_samples_between_scales=-1)
    with pytest.raises(SystemExit):
        runner.main(["--out", str(tmp_path)])  # no subjects


def test_subject_analysis_from_records_writes_schema_v3(tmp_path):
    """The runner's glue on the host: records and samples into the analysis arrays and the NPZ."""
    from fastcorticalwiring_b200 import _lib, analysis, mesh as M
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    mesh = folded_icosphere(3, seed=4)
    pm = M.prepare(mesh.vertices, mesh.faces, mesh.cortex_mask)
    sa = runner.SubjectAnalysis(pm, {"t_coef": 2.0, "mean_edge_length": 0.5}, 0.7, metadata={"subject": "s"})
    scales, m, cap = analysis.WiringAnalysis.run_arguments(None, 1, None)
    targets = sa._reset(scales, m, cap)
    assert np.allclose(targets, pm.targets(scales))
    src = pm.bfs[:5].astype(np.int32)
    nt = len(scales)
    rec = np.zeros((src.size, _lib.metrics_stride(nt, m)))
    rec[:, 0], rec[:, 1], rec[:, 2] = 10.0, 11.0, 3.0
    rec[2, 5] = 1.0  # one flagged field
    rec[:, 7:7 + nt] = np.arange(1, nt + 1)
    cap_n = _lib.samples_capacity(nt, m)
    radii = np.tile(np.arange(cap_n, dtype=np.float32), (src.size, 1))
    counts = np.array([3, 0, 0, 1, 2], np.int32)
    with pytest.warns(RuntimeWarning, match="1 of 5 source vertices"):
        sa._absorb(src, rec, (radii, radii * 2, counts))
        sa._finish(src.size)
    orig = pm.sub_to_orig[src]
    assert sa.field_flag[orig[2]] == 1 and np.isnan(sa.msd_weighted[orig[2]])
    assert sa.msd_weighted[orig[0]] == np.float32(11.0)
    assert sa.radius_function[scales[-1]][orig[1]] == np.float32(nt)
    assert int(sa.sample_indptr[-1]) == int(counts.sum())
    r, a = sa.get_vertex_samples(orig[0])
    assert list(r) == [0.0, 1.0, 2.0] and list(a) == [0.0, 2.0, 4.0]
    path = analysis.save_analysis_npz(str(tmp_path), "s.npz", sa)
    z = np.load(path)
    assert int(z["fastcw_output_schema_version"]) == 3 and int(z["n_samples_between_scales"]) == 1
    prov = json.loads(str(z["provenance_json"]))
    assert prov["engine"] == "b200" and prov["t_coef"] == 2.0 and prov["n_flagged_fields"] == 1
    assert sa.metadata == {"subject": "s"}


def test_subject_analysis_warns_on_interior_nonmanifold_submesh():
    """Batch subjects get the same interior non-manifold warning as a single-subject analysis
    (core_analysis.py:628-635), and the count is kept on the subject."""
    from fastcorticalwiring_b200 import mesh as M
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    mesh = folded_icosphere(3, seed=1)
    V, F = mesh.vertices, mesh.faces
    a, b = F[0, 0], F[0, 1]
    V2 = np.vstack([V, V[a] + 1.0])
    F2 = np.vstack([F, [a, b, len(V)], [b, a, len(V)]])
    pm = M.prepare(V2, F2, np.ones(len(V2), bool))
    with pytest.warns(RuntimeWarning, match="Interior non-manifold vertices"):
        sa = runner.SubjectAnalysis(pm, {}, 0.7)
    assert sa.n_interior_nonmanifold == 2
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        quiet = runner.SubjectAnalysis(pm, {}, 0.7, allow_interior_nonmanifold=True)
    assert quiet.n_interior_nonmanifold == 2
