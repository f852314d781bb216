"""Cortical submeshes of several connected components (needs a B200).

The reference runs every source over the whole submesh whatever its connectivity
(core_analysis.py:1349-1381 only reports the components). L is then singular once per
component: the FP64 form's L + shift*M leaves phi with zero M-weighted mean on the
source's component and zero on the others, so every vertex of another component sits at
the M-weighted mean distance over the source's component (that level carries the
rounding of 1^T div X / shift, about 1e-8 of it, hence the looser bound off the source's
component). The mixed form grounds one
vertex per component and sets the other components to that level; both forms and the
drop-in must agree with the oracle there as on the source's component.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import engine, mesh as M  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402

SCALES = M.RUNNER_SCALES


@pytest.fixture(scope="module")
def two():
    import oracle
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components

    a = folded_icosphere(4, seed=3, jitter=0.2)
    b = folded_icosphere(3, seed=5, jitter=0.1)
    V = np.vstack([a.vertices, 0.5 * b.vertices])  # a smaller surface inside the first one
    F = np.vstack([a.faces, b.faces + len(a.vertices)])
    pm = M.prepare(V, F, np.concatenate([a.cortex_mask, b.cortex_mask]))
    n = pm.n_vertices
    G = sp.coo_matrix((np.ones(3 * len(pm.F)), (pm.F.ravel(), pm.F[:, [1, 2, 0]].ravel())), shape=(n, n))
    ncomp, label = connected_components(G, directed=False)
    assert ncomp == 2
    first = np.flatnonzero(label == label[0])
    second = np.flatnonzero(label != label[0])
    src = np.concatenate([first[np.linspace(0, first.size - 1, 5).astype(int)],
                          second[np.linspace(0, second.size - 1, 3).astype(int)]]).astype(np.int32)
    orc = oracle.HeatOracle(pm.V, pm.F)
    eng = engine.HeatEngine(pm.V, pm.F, block_k=64)
    yield dict(pm=pm, label=label, src=src, orc=orc, ref=orc.distances(src), mass=np.asarray(orc.mass).ravel(),
               eng=eng)
    eng.close()


def _check_against(d, ref, label, src, on_tol, off_tol):
    for j, s in enumerate(src):
        on = label == label[s]
        scale = np.max(np.abs(ref[j]))
        assert np.max(np.abs(d[j][on] - ref[j][on])) <= on_tol * scale, (j, "on")
        assert np.max(np.abs(d[j][~on] - ref[j][~on])) <= off_tol * scale, (j, "off")


def test_engine_counts_the_components(two):
    assert two["eng"].info()["n_components"] == 2


def test_oracle_puts_other_components_at_the_mean_distance(two):
    for j, s in enumerate(two["src"]):
        on = two["label"] == two["label"][s]
        d = two["ref"][j]
        level = np.sum(two["mass"][on] * d[on]) / np.sum(two["mass"][on])
        assert np.ptp(d[~on]) == 0.0
        assert abs(d[~on][0] - level) <= 1e-6 * level


def test_fp64_and_dropin_match_oracle(two):
    eng = two["eng"]
    d = eng.compute_distances(two["src"], precision="fp64")
    assert np.all(np.isfinite(d))
    _check_against(d, two["ref"], two["label"], two["src"], 1e-9, 1e-6)
    one = np.stack([eng.compute_distance(int(s)) for s in two["src"]])
    _check_against(one, two["ref"], two["label"], two["src"], 1e-9, 1e-6)


def test_mixed_matches_oracle(two):
    d = two["eng"].compute_distances(two["src"], precision="mixed")
    assert np.all(np.isfinite(d))
    _check_against(d, two["ref"], two["label"], two["src"], 1e-4, 1e-4)
    for j, s in enumerate(two["src"]):
        assert d[j][s] == 0.0


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 1e-4)])
def test_metrics_match_oracle(two, precision, tol):
    import oracle

    pm = two["pm"]
    targets = pm.targets(SCALES)
    rec = two["eng"].compute_metrics(two["src"], targets, n_between=3, precision=precision)
    r = engine.split_records(rec, len(SCALES), 3)
    for j, s in enumerate(two["src"]):
        ref = oracle.source_metrics(two["ref"][j], int(s), pm, targets)
        assert bool(r["bad"][j]) == ref["bad"]
        if ref["bad"]:
            continue
        rel = lambda a, b: np.max(np.abs(np.asarray(a) - b) / np.maximum(np.abs(b), 1e-300))  # noqa: E731
        assert rel(r["radii"][j], ref["radii"]) <= tol
        assert rel(r["perim"][j], ref["perim"]) <= tol
        assert rel(r["msd_w"][j], ref["msd_w"]) <= tol


@pytest.mark.parametrize("refine,robust", [(1, 0), (0, 1), (2, 1)])
def test_refined_and_robust_mixed_match_fp64(two, refine, robust):
    """The refinement residual and the intrinsic-Delaunay operators ground every component too."""
    pm, src = two["pm"], two["src"]
    eng = engine.HeatEngine(pm.V, pm.F, block_k=64, refine=refine, robust=robust)
    try:
        assert eng.info()["n_components"] == 2
        d64 = eng.compute_distances(src, precision="fp64")
        d32 = eng.compute_distances(src, precision="mixed")
    finally:
        eng.close()
    assert np.all(np.isfinite(d32))
    _check_against(d32, d64, two["label"], src, 1e-4, 1e-4)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 1e-4)])
def test_engine_matches_reference_outputs_on_two_components(precision, tol):
    """The float32 arrays the reference's analysis wrote on a two-component submesh
    (tests/golden/golden_components_L4.npz, made by the reference's own code)."""
    import os

    from tests.conftest import GOLDEN

    z = dict(np.load(os.path.join(GOLDEN, "golden_components_L4.npz")))
    pm = M.prepare(z["V"], z["F"], z["mask"])
    eng = engine.HeatEngine(pm.V, pm.F, block_k=64)
    try:
        r = engine.split_records(eng.compute_metrics(z["sources_sub"].astype(np.int32), z["targets"], n_between=3,
                                                     precision=precision), len(SCALES), 3)
    finally:
        eng.close()
    rel = lambda a, b: np.abs(np.asarray(a, float) - b) / np.abs(b)  # noqa: E731
    for j in range(z["sources_sub"].size):
        assert bool(r["bad"][j]) == bool(z["field_flag"][j])
        if r["bad"][j]:
            continue
        assert rel(r["msd_w"][j], z["f32_msd_weighted"][j]) <= max(tol, 2.4e-7)
        for i, sc in enumerate(z["scales"]):
            tok = format(float(sc), "g")
            assert rel(r["radii"][j, i], z["f32_radius_" + tok][j]) <= max(tol, 2.4e-7)
            assert rel(r["perim"][j, i], z["f32_perimeter_" + tok][j]) <= max(tol, 2.4e-7)
