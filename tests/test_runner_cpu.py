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
