"""The batch runner (needs a B200): subjects run together through the serving loop give the
same analysis NPZ as WiringAnalysis on each subject alone.

Two order-4 hemispheres with their own folding seeds are written as subject files and run
in one batch; each output (schema v3: metric arrays, health flags and the sample CSR) must
match WiringAnalysis.compute_all_wiring_costs + save_analysis_npz on the same mesh: the
CSR row pointers exactly and every float32 value to 1e-6 relative (the same kernels on the
same inputs; only the order of atomically appended faces inside a bin differs).
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import analysis, runner  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402


def _close(a, b):
    assert a.shape == b.shape and a.dtype == b.dtype
    if a.dtype.kind != "f":
        assert np.array_equal(a, b)
        return
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    d = np.abs(a[~na].astype(np.float64) - b[~nb].astype(np.float64))
    assert np.all(d <= 1e-6 * np.maximum(np.abs(b[~nb].astype(np.float64)), 1e-30))


def test_batch_matches_single_subject_analysis(tmp_path):
    subjects = []
    for seed in (5, 6):
        m = folded_icosphere(4, seed=seed, jitter=0.2)
        p = tmp_path / f"lh_{seed}.npz"
        np.savez(p, vertices=m.vertices, faces=m.faces, cortex_mask=m.cortex_mask)
        subjects.append((f"lh_{seed}", str(p)))
    out = runner.run_subjects(subjects, str(tmp_path / "batch"), n_samples_between_scales=3,
                              boundary_cap_fraction=0.05)
    assert out["failed"] == {} and set(out["written"]) == {"lh_5", "lh_6"}
    for name, path in subjects:
        V, F, mask = runner.load_mesh(path)
        wa = analysis.WiringAnalysis(V, F, mask)
        wa.compute_all_wiring_costs(n_samples_between_scales=3, boundary_cap_fraction=0.05)
        ref = dict(np.load(analysis.save_analysis_npz(str(tmp_path / "single"), f"{name}.npz", wa)))
        got = dict(np.load(out["written"][name]))
        assert set(got) == set(ref)
        for k in ref:
            if k == "provenance_json":
                pg, pr = json.loads(str(got[k])), json.loads(str(ref[k]))
                for key in ("engine", "use_robust", "diffusion_length_mm", "geometry_method", "n_flagged_fields"):
                    assert pg[key] == pr[key], key
                assert abs(pg["t_coef"] - pr["t_coef"]) <= 1e-12 * pr["t_coef"]
            elif ref[k].dtype.kind in "US":
                assert str(got[k]) == str(ref[k]), k
            else:
                _close(got[k], ref[k])
    assert os.path.exists(out["written"]["lh_5"])
