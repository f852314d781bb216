"""Pin the CPU oracle (and the host mesh preparation) to the reference's own outputs.

The fixtures were produced by the reference code (tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

import oracle
from fastcorticalwiring_b200 import mesh as M
from tests.conftest import GOLDEN


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@pytest.fixture(scope="module", params=["golden_heat_L4.npz", "golden_metrics_L5.npz"])
def fx(request):
    z = _load(request.param)
    z["pm"] = M.prepare(z["V"], z["F"], z["mask"])
    return z


def test_mesh_prep_matches_reference(fx):
    pm = fx["pm"]
    assert np.array_equal(pm.vertex_area, fx["vertex_area"])          # bit-exact summation order
    assert np.array_equal(pm.boundary, fx["boundary"])
    assert np.array_equal(pm.bfs, fx["bfs_order"])
    assert pm.health_h == float(fx["health_h"])
    assert pm.bin_width == float(fx["bin_width"])
    assert np.array_equal(pm.targets(fx["scales"]), fx["targets"])


def test_heat_time_step(fx):
    pm = fx["pm"]
    h = oracle.mean_edge_length(pm.V, pm.F)
    t = ((0.7 / h) ** 2) * h * h
    assert t == float(fx["t"])


def test_oracle_geometry_bit_exact_on_reference_fields():
    z = _load("golden_heat_L4.npz")
    pm = M.prepare(z["V"], z["F"], z["mask"])
    fr = np.array([0.25, 0.5, 0.75])
    for j in range(z["phi"].shape[0]):
        r, p, er, ea, n = oracle.source_geometry(z["phi"][j], pm.F, pm.lean_area, pm.g11, pm.g12, pm.g22,
                                                 pm.bin_width, z["targets"], fr)
        assert np.array_equal(r, z["radii"][j])
        assert np.array_equal(p, z["perim"][j])
        assert np.array_equal(er, z["extra_r"][j], equal_nan=True)
        assert np.array_equal(ea, z["extra_a"][j], equal_nan=True)
        assert n == z["n_eval"][j]
        neg, viol, bad = oracle.field_health(z["phi"][j], pm.V, z["sources_sub"][j], pm.health_h)
        assert [neg, viol, float(bad)] == list(z["health"][j])


def test_oracle_heat_stages_match_reference():
    z = _load("golden_heat_L4.npz")
    pm = M.prepare(z["V"], z["F"], z["mask"])
    ho = oracle.HeatOracle(pm.V, pm.F)
    assert ho.t == float(z["t"])
    u = ho.heat(z["stage_sources"])
    assert np.max(np.abs(u - z["stage_u"])) <= 1e-13 * np.max(np.abs(z["stage_u"]))
    # the divergence is bit-exact given the same u
    assert np.array_equal(ho.divergence(z["stage_u"]), z["stage_div"])
    phi = ho.distances(z["sources_sub"])
    ref = z["phi"]
    assert np.max(np.abs(phi - ref)) <= 1e-11 * np.max(np.abs(ref))


def test_oracle_analysis_outputs_match_reference_float32(fx):
    """The float32 arrays core_analysis writes, recomputed by the oracle from its own fields."""
    pm = fx["pm"]
    ho = oracle.HeatOracle(pm.V, pm.F)
    phi = ho.distances(fx["sources_sub"])
    scales = [float(s) for s in fx["scales"]]
    for j, s in enumerate(fx["sources_sub"]):
        out = oracle.source_metrics(phi[j], int(s), pm, fx["targets"])
        assert not out["bad"] and fx["field_flag"][j] == 0
        assert np.float32(out["msd_u"]) == fx["f32_msd_unweighted"][j]
        assert np.float32(out["msd_w"]) == fx["f32_msd_weighted"][j]
        assert np.float32(out["dist_b"]) == fx["f32_dist_to_boundary"][j]
        for i, sc in enumerate(scales):
            tok = format(sc, "g")
            # FP64 fields from two factorisations differ at 1e-15: allow one float32 ulp
            np.testing.assert_allclose(np.float32(out["radii"][i]), fx["f32_radius_" + tok][j], rtol=2.4e-7)
            np.testing.assert_allclose(np.float32(out["perim"][i]), fx["f32_perimeter_" + tok][j], rtol=2.4e-7)


def test_oracle_matches_reference_with_other_settings():
    """Diffusion length 1.0 mm, the analysis' default six scales and one sample between scales."""
    z = _load("golden_params_L4.npz")
    pm = M.prepare(z["V"], z["F"], z["mask"])
    ho = oracle.HeatOracle(pm.V, pm.F, diffusion_length_mm=float(z["diffusion_length_mm"]))
    assert ho.t == float(z["t"])
    sub = pm.orig_to_sub[z["sources_orig"]]
    phi = ho.distances(sub)
    targets = pm.targets(z["scales"])
    nb = int(z["n_between"])
    for j, s in enumerate(sub):
        out = oracle.source_metrics(phi[j], int(s), pm, targets, n_between=nb)
        assert out["bad"] == bool(z["field_flag"][j])
        for i, sc in enumerate(z["scales"]):
            tok = format(float(sc), "g")
            # FP64 fields from two factorisations differ at 1e-15: allow one float32 ulp
            np.testing.assert_allclose(np.float32(out["radii"][i]), z[f"f32_radius_{tok}"][j], rtol=2.4e-7)
            np.testing.assert_allclose(np.float32(out["perim"][i]), z[f"f32_perimeter_{tok}"][j], rtol=2.4e-7)
        np.testing.assert_allclose(np.float32(out["msd_w"]), z["f32_msd_weighted"][j], rtol=2.4e-7)
        lo, hi = z["sample_indptr"][j], z["sample_indptr"][j + 1]
        assert hi - lo == len(z["scales"]) + (len(z["scales"]) - 1) * nb


def test_oracle_matches_reference_on_two_components():
    """A submesh of two connected components: the reference puts every vertex of the other
    component at one level, the M-weighted mean distance over the source's component, which
    carries the rounding of 1^T div X / shift (1e-9 of the field between two factorisations)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    z = _load("golden_components_L4.npz")
    pm = M.prepare(z["V"], z["F"], z["mask"])
    assert np.array_equal(pm.bfs, z["bfs_order"])
    n = pm.n_vertices
    G = coo_matrix((np.ones(pm.F.size), (pm.F.ravel(), pm.F[:, [1, 2, 0]].ravel())), shape=(n, n))
    ncomp, label = connected_components(G, directed=False)
    assert ncomp == 2 and len(set(label[z["sources_sub"]])) == 2
    ho = oracle.HeatOracle(pm.V, pm.F)
    phi = ho.distances(z["sources_sub"])
    mass = np.asarray(ho.mass).ravel()
    for j, s in enumerate(z["sources_sub"]):
        on = label == label[s]
        ref = z["phi"][j]
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(phi[j][on] - ref[on])) <= 1e-12 * scale
        assert np.max(np.abs(phi[j][~on] - ref[~on])) <= 1e-8 * scale
        assert np.ptp(ref[~on]) == 0.0
        level = np.sum(mass[on] * ref[on]) / np.sum(mass[on])
        assert abs(ref[~on][0] - level) <= 1e-8 * level
        out = oracle.source_metrics(phi[j], int(s), pm, z["targets"])
        assert out["bad"] == bool(z["field_flag"][j])
        if out["bad"]:
            assert np.isnan(z["f32_msd_weighted"][j])
            continue
        np.testing.assert_allclose(np.float32(out["msd_w"]), z["f32_msd_weighted"][j], rtol=2.4e-7)
        np.testing.assert_allclose(np.float32(out["msd_u"]), z["f32_msd_unweighted"][j], rtol=2.4e-7)
        for i, sc in enumerate(z["scales"]):
            tok = format(float(sc), "g")
            np.testing.assert_allclose(np.float32(out["radii"][i]), z["f32_radius_" + tok][j], rtol=2.4e-7)
            np.testing.assert_allclose(np.float32(out["perim"][i]), z["f32_perimeter_" + tok][j], rtol=2.4e-7)


def test_geometry_kat():
    z = _load("golden_geometry_kat.npz")
    V, F = z["V"], z["F"].astype(np.int32)
    area, g11, g12, g22 = M.lean_face_metric(V, F)
    w = float(z["bin_width"])
    assert M.lean_bin_width(V, F) == w
    for i, f in enumerate(z["fields"]):
        for j, r in enumerate(z["radii_eval"][i]):
            a, nl = oracle.field_eval("area", r, f, F, area, g11, g12, g22, w)
            da, _ = oracle.field_eval("darea", r, f, F, area, g11, g12, g22, w)
            p, _ = oracle.field_eval("perimeter", r, f, F, area, g11, g12, g22, w)
            assert a == z["area_eval"][i][j] and da == z["darea_eval"][i][j] and p == z["perim_eval"][i][j]
            assert nl == z["n_long"][i]
    assert z["n_long"][3] > 0            # the non-Lipschitz field exercises the long-face list
    for g, f in enumerate((z["fields"][0], z["fields"][3])):
        r, p, er, ea, n = oracle.source_geometry(f, F, area, g11, g12, g22, w, z["targets"], z["fracs"], 1e-12, 60)
        assert np.array_equal(r, z["geo_radii"][g]) and np.array_equal(p, z["geo_perim"][g])
        assert np.array_equal(er, z["geo_extra_r"][g]) and np.array_equal(ea, z["geo_extra_a"][g])
        assert n == z["geo_n_eval"][g]
    f = z["fields"][3]
    assert oracle.field_eval("area", np.nan, f, F, area, g11, g12, g22, w)[0] == z["nan_area"] == 0.0
    assert np.isnan(oracle.field_eval("radius", np.nan, f, F, area, g11, g12, g22, w, 1e-12)[0])
    assert np.isnan(oracle.field_eval("radius", 2 * float(z["total_area"]), f, F, area, g11, g12, g22, w, 1e-12)[0])
    assert oracle.field_eval("radius", 0.0, f, F, area, g11, g12, g22, w, 1e-12)[0] == 0.0 == z["zero_radius"]
