"""Sample assembly and the batched analysis on the device (needs a B200).

The device assembly works on metric records; given the reference's own FP64
geometry records it must reproduce the reference's sample CSR exactly
(golden_samples_L5.npz: boundary cap 0.05; golden_metrics_L5.npz: no cap). The
full WiringAnalysis run is compared with the reference's float32 outputs at the
FP64 bar (1e-6 relative) and its NPZ with the keys and dtypes the reference's
writer produces.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import oracle  # noqa: E402
from fastcorticalwiring_b200 import _lib, analysis, engine, mesh as M  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402
from tests.conftest import GOLDEN  # noqa: E402


def _records(radii, extra_r, extra_a, dist_b, bad=None):
    """Metric records (fcw_compute_metrics layout) holding the given geometry."""
    n, nt = radii.shape
    ne = extra_r.shape[1]
    nb = ne // max(1, nt - 1)
    rec = np.zeros((n, _lib.metrics_stride(nt, nb)))
    rec[:, 2] = dist_b
    if bad is not None:
        rec[:, 5] = bad
    rec[:, 7:7 + nt] = radii
    rec[:, 7 + nt:7 + 2 * nt] = 1.0
    rec[:, 7 + 2 * nt:7 + 2 * nt + ne] = extra_r
    rec[:, 7 + 2 * nt + ne:7 + 2 * nt + 2 * ne] = extra_a
    return rec, nb


def _csr(r, a, c):
    indptr = np.concatenate([[0], np.cumsum(c)]).astype(np.int64)
    keep = np.arange(r.shape[1])[None, :] < c[:, None]
    return indptr, r[keep], a[keep]


@pytest.fixture(scope="module")
def eng():
    z = np.load(os.path.join(GOLDEN, "golden_metrics_L5.npz"))
    pm = M.prepare(z["V"], z["F"], z["mask"])
    e = engine.HeatEngine(pm.V, pm.F, block_k=64)
    yield e
    e.close()


@pytest.mark.parametrize("name,cap", [("golden_samples_L5.npz", "fixture"), ("golden_metrics_L5.npz", None)])
def test_device_assembly_reproduces_reference_csr(eng, name, cap):
    z = np.load(os.path.join(GOLDEN, name))
    c = float(z["cap"]) if cap == "fixture" else None
    rec, nb = _records(z["radii"], z["extra_r"], z["extra_a"], z["f32_dist_to_boundary"])
    for _ in range(2):  # a second call reuses the staging buffers
        r, a, cnt = eng.assemble_samples(rec, z["targets"], n_between=nb, boundary_cap=c)
        indptr, rr, aa = _csr(r, a, cnt)
        assert np.array_equal(indptr, z["sample_indptr"])
        assert np.array_equal(rr, z["sample_r"])
        assert np.array_equal(aa, z["sample_a"])


def test_device_assembly_edge_cases(eng):
    """Flagged fields, NaN radii, near-duplicates, caps of 0 and none, a single scale, no extras."""
    rng = np.random.default_rng(7)
    radii = np.sort(rng.uniform(1.0, 30.0, (6, 4)), axis=1)
    radii[1, 2] = np.nan
    radii[2, 1] = radii[2, 0] * (1 + 1e-12)  # a near-duplicate of its predecessor
    extra_r = np.sqrt(radii[:, :-1] * radii[:, 1:])
    extra_r = np.repeat(extra_r, 2, axis=1)
    extra_a = 1000.0 + extra_r
    extra_a[3, 0] = np.inf
    dist_b = np.array([10.0, 0.0, np.inf, np.nan, 5.0, 25.0], np.float32)
    bad = np.array([0, 0, 0, 0, 1, 0], float)
    targets = np.array([1.0, 2.0, 3.0, 4.0])
    rec, nb = _records(radii, extra_r, extra_a, dist_b, bad)
    for cap in (None, 0.0, 0.2):
        r, a, cnt = eng.assemble_samples(rec, targets, n_between=nb, boundary_cap=cap)
        for k in range(rec.shape[0]):
            want = [] if bad[k] else oracle.vertex_samples(radii[k], targets, extra_r[k], extra_a[k], dist_b[k], cap)
            got = list(zip(r[k, :cnt[k]].tolist(), a[k, :cnt[k]].tolist()))
            want = [(float(np.float32(x)), float(np.float32(y))) for x, y in want]
            assert got == want, (cap, k)
    one, _ = _records(radii[:, :1], np.zeros((6, 0)), np.zeros((6, 0)), dist_b)
    r, a, cnt = eng.assemble_samples(one, targets[:1], n_between=0, boundary_cap=0.1)
    assert list(cnt) == [1, 1, 1, 1, 1, 1]
    with pytest.raises(_lib.FCWError):
        eng.assemble_samples(rec, targets, n_between=nb, boundary_cap=0.5)


@pytest.fixture(scope="module")
def l5_metrics():
    z = np.load(os.path.join(GOLDEN, "golden_metrics_L5.npz"))
    an = analysis.WiringAnalysis(z["V"], z["F"], z["mask"], precision="fp64")
    an.compute_all_wiring_costs(scale=z["scales"], vertex_subset=z["sources_orig"], n_samples_between_scales=3)
    return z, an


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-30)


def test_analysis_matches_reference_outputs(l5_metrics):
    z, an = l5_metrics
    o = z["sources_orig"]
    assert np.array_equal(an.field_flag[o], z["field_flag"])
    for k, v in an.get_metric_arrays().items():
        assert v.dtype == np.float32 and v.shape == (an.n_vertices_full,)
        assert np.max(_rel(v[o], z["f32_" + k])) <= 1e-6, k
    rest = np.setdiff1d(np.arange(an.n_vertices_full), o)
    assert np.all(np.isnan(an.msd_unweighted[rest]))
    for j, v in enumerate(o):
        r, a = an.get_vertex_samples(v)
        lo, hi = z["sample_indptr"][j], z["sample_indptr"][j + 1]
        assert r.size == hi - lo
        assert np.max(_rel(r, z["sample_r"][lo:hi])) <= 1e-6
        assert np.max(_rel(a, z["sample_a"][lo:hi])) <= 1e-6
    assert an.sample_indptr[-1] == z["sample_indptr"][-1]


def test_analysis_with_boundary_cap_matches_reference():
    z = np.load(os.path.join(GOLDEN, "golden_samples_L5.npz"))
    mesh = folded_icosphere(int(z["level"]), seed=int(z["seed"]), jitter=float(z["jitter"]))
    an = analysis.WiringAnalysis(mesh.vertices, mesh.faces, mesh.cortex_mask, precision="fp64")
    an.compute_all_wiring_costs(scale=z["scales"], vertex_subset=z["sources_orig"], n_samples_between_scales=3,
                                boundary_cap_fraction=float(z["cap"]))
    o = z["sources_orig"]
    assert np.max(_rel(an.dist_to_boundary[o], z["f32_dist_to_boundary"])) <= 1e-6
    for j, v in enumerate(o):
        r, a = an.get_vertex_samples(v)
        lo, hi = z["sample_indptr"][j], z["sample_indptr"][j + 1]
        assert r.size == hi - lo, j
        assert np.max(_rel(r, z["sample_r"][lo:hi]), initial=0.0) <= 1e-6
        assert np.max(_rel(a, z["sample_a"][lo:hi]), initial=0.0) <= 1e-6


@pytest.mark.parametrize("precision, tol, tol_msd", [("fp64", 1e-6, 1e-6), ("mixed", 1e-4, 1e-5)])
def test_analysis_with_other_settings_matches_reference(precision, tol, tol_msd):
    """Diffusion length 1.0 mm, the default six scales and one sample between them: the FP64 form
    to the float32 outputs' precision, the mixed form within its bar."""
    z = np.load(os.path.join(GOLDEN, "golden_params_L4.npz"))
    an = analysis.WiringAnalysis(z["V"], z["F"], z["mask"], precision=precision,
                                 engine_kwargs={"diffusion_length_mm": float(z["diffusion_length_mm"])})
    an.compute_all_wiring_costs(scale=None, vertex_subset=z["sources_orig"],
                                n_samples_between_scales=int(z["n_between"]))
    o = z["sources_orig"]
    assert np.array_equal(an.field_flag[o], z["field_flag"])
    assert an.active_scales == tuple(float(s) for s in z["scales"])
    for k, v in an.get_metric_arrays().items():
        assert np.max(_rel(v[o], z["f32_" + k])) <= (tol_msd if k.startswith("msd") else tol), k
    for j, v in enumerate(o):
        r, a = an.get_vertex_samples(v)
        lo, hi = z["sample_indptr"][j], z["sample_indptr"][j + 1]
        assert r.size == hi - lo
        assert np.max(_rel(r, z["sample_r"][lo:hi])) <= tol
        assert np.max(_rel(a, z["sample_a"][lo:hi])) <= tol


def test_analysis_validation_matches_reference(l5_metrics):
    _, an = l5_metrics
    for bad in (-0.1, 0.5, 0.7, 1.0, np.nan):
        with pytest.raises(ValueError, match="boundary_cap_fraction must be in"):
            an.compute_all_wiring_costs(scale=[0.01, 0.02], vertex_subset=[0], boundary_cap_fraction=bad)
    with pytest.raises(ValueError, match="n_samples_between_scales must be >= 0"):
        an.compute_all_wiring_costs(scale=[0.01], vertex_subset=[0], n_samples_between_scales=-1)


def test_npz_matches_reference_schema(l5_metrics, tmp_path):
    _, an = l5_metrics
    ref = np.load(os.path.join(GOLDEN, "golden_samples_L5.npz"))
    path = analysis.save_analysis_npz(str(tmp_path), "out.npz", an, n_samples_between_scales=3)
    got = np.load(path)
    keys = sorted(got.files)
    assert keys == ref["npz_keys"].tolist()
    for k, dt, nd in zip(ref["npz_keys"], ref["npz_dtypes"], ref["npz_ndims"]):
        assert got[k].ndim == nd, k
        if not str(dt).startswith("<U"):
            assert str(got[k].dtype) == str(dt), k
    assert int(got["fastcw_output_schema_version"]) == int(ref["npz_schema"]) == 3
    import json
    prov = json.loads(str(got["provenance_json"]))
    assert prov["engine"] == "b200" and prov["use_robust"] is False
