"""The sample-assembly oracle against the reference's own outputs (CPU).

golden_samples_L5.npz was written by the reference (tests/golden/make_golden.py):
compute_all_wiring_costs with boundary_cap_fraction=0.05 on sources 0..40 mm from
the mesh boundary, boundary_area_loss_fraction on an (r, d) grid including the
non-finite cases, and _clean_vertex_samples on crafted pair lists.
"""

import math
import os

import numpy as np
import pytest

import oracle
from tests.conftest import GOLDEN


@pytest.fixture(scope="module")
def z():
    return np.load(os.path.join(GOLDEN, "golden_samples_L5.npz"))


def test_boundary_loss_kats():
    """test_vertex_subsetting.py:52-58."""
    f = oracle.boundary_area_loss_fraction
    assert f(10.0, 10.0) == pytest.approx(0.0, abs=1e-12)
    assert f(10.0, 5.0) == pytest.approx(0.19550110947788538, abs=1e-12)
    assert f(10.0, 0.0) == pytest.approx(0.5, abs=1e-12)
    assert f(10.0, 20.0) == pytest.approx(0.0, abs=1e-12)
    assert f(10.0, np.inf) == pytest.approx(0.0, abs=1e-12)


def test_boundary_loss_grid_matches_reference(z):
    got = np.vectorize(oracle.boundary_area_loss_fraction)(z["loss_r"], z["loss_d"])
    ref = z["loss"]
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    assert np.array_equal(got[~np.isnan(ref)], ref[~np.isnan(ref)])


def test_clean_vertex_samples_matches_reference(z):
    ii, oi = z["clean_in_indptr"], z["clean_out_indptr"]
    for c in range(ii.size - 1):
        pairs = [tuple(p) for p in z["clean_in"][ii[c]:ii[c + 1]]]
        got = np.asarray(oracle.clean_vertex_samples(pairs), np.float64).reshape(-1, 2)
        assert np.array_equal(got, z["clean_out"][oi[c]:oi[c + 1]])
    assert oracle.clean_vertex_samples([]) == []


@pytest.mark.parametrize("radii,cap,kept,dropped", [
    ([9.98, 10.0, 10.02], 0.0, [math.sqrt(9.98 * 10.0)], [math.sqrt(10.0 * 10.02)]),
    ([14.4, 14.6, 15.1, 15.3], 0.1, [math.sqrt(14.4 * 14.6)], [math.sqrt(15.1 * 15.3)]),
    ([9990.0, 10010.0], None, [math.sqrt(9990.0 * 10010.0)], []),
])
def test_boundary_cap_cases(radii, cap, kept, dropped):
    """The boundary-cap cases of test_vertex_subsetting.py:83-116 (boundary at distance 10)."""
    radii = np.asarray(radii)
    extra_r = np.sqrt(radii[:-1] * radii[1:])
    rows = oracle.vertex_samples(radii, np.ones_like(radii), extra_r, 1000.0 + extra_r, np.float32(10.0), cap)
    extras = np.asarray([r for r, a in rows if a > 900.0])
    for k in kept:
        assert np.any(np.isclose(extras, k, rtol=1e-5))
    for d in dropped:
        assert not np.any(np.isclose(extras, d, rtol=1e-5))


def test_samples_match_reference_with_cap(z):
    cap = float(z["cap"])
    rows = {}
    for j in range(z["sources_sub"].size):
        assert z["field_flag"][j] == 0
        rows[j] = oracle.vertex_samples(z["radii"][j], z["targets"], z["extra_r"][j], z["extra_a"][j],
                                        z["f32_dist_to_boundary"][j], cap)
    indptr, r, a = oracle.csr(rows, z["sources_sub"].size)
    assert np.array_equal(indptr, z["sample_indptr"])
    assert np.array_equal(r, z["sample_r"])
    assert np.array_equal(a, z["sample_a"])


def test_samples_match_reference_without_cap():
    z = np.load(os.path.join(GOLDEN, "golden_metrics_L5.npz"))
    rows = {j: oracle.vertex_samples(z["radii"][j], z["targets"], z["extra_r"][j], z["extra_a"][j],
                                     z["f32_dist_to_boundary"][j], None)
            for j in range(z["sources_sub"].size)}
    indptr, r, a = oracle.csr(rows, z["sources_sub"].size)
    assert np.array_equal(indptr, z["sample_indptr"])
    assert np.array_equal(r, z["sample_r"])
    assert np.array_equal(a, z["sample_a"])
