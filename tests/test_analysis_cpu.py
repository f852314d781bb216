"""WiringAnalysis host logic without a device.

Scales, run arguments and source subsets follow core_analysis.py: normalize_scales
(:727-752), scale_token (:754-757), the run validation (:1441-1500) and the subset
handling of compute_all_wiring_costs (:1519-1533: unparsable, out-of-range and
medial-wall ids are skipped; the survivors run in BFS order, once each).
"""
import numpy as np
import pytest

from fastcorticalwiring_b200 import analysis as A
from fastcorticalwiring_b200 import mesh as M
from fastcorticalwiring_b200.meshgen import folded_icosphere


def test_normalize_scales_and_tokens():
    assert A.WiringAnalysis.normalize_scales(None) == A.WiringAnalysis.DEFAULT_SCALES
    assert A.WiringAnalysis.normalize_scales(0.01) == (0.01,)
    assert A.WiringAnalysis.normalize_scales([0.05, 0.01, 0.05, np.float32(0.02)]) == (0.01, float(np.float32(0.02)),
                                                                                       0.05)
    for bad, msg in (([], "At least one scale"), ([0.0], "expected 0 < scale <= 1"), ([1.5], "expected 0"),
                     ([np.nan], "must be finite"), ([np.inf], "must be finite")):
        with pytest.raises(ValueError, match=msg):
            A.WiringAnalysis.normalize_scales(bad)
    assert A.WiringAnalysis.scale_token(0.00267988) == "0.00267988"
    assert A.WiringAnalysis.scale_token(0.05) == "0.05"


def test_run_arguments():
    scales, m, cap = A.WiringAnalysis.run_arguments([0.02, 0.01], 2, None)
    assert scales == (0.01, 0.02) and m == 2 and cap is None
    assert A.WiringAnalysis.run_arguments(None, 0, 0.0)[2] == 0.0
    for cap in (-0.1, 0.5, 1.0, np.nan):
        with pytest.raises(ValueError, match="boundary_cap_fraction must be in"):
            A.WiringAnalysis.run_arguments(None, 3, cap)
    with pytest.raises(ValueError, match="n_samples_between_scales must be >= 0"):
        A.WiringAnalysis.run_arguments(None, -1, None)
    with pytest.raises(ValueError, match="at most 32 scales"):
        A.WiringAnalysis.run_arguments(np.linspace(0.001, 0.1, 33), 3, None)
    with pytest.raises(ValueError, match="must be <= 8"):
        A.WiringAnalysis.run_arguments(None, 9, None)


def test_vertex_subset_filtering_and_order():
    mesh = folded_icosphere(3, seed=1)
    pm = M.prepare(mesh.vertices, mesh.faces, mesh.cortex_mask)
    wa = object.__new__(A.WiringAnalysis)  # the subset logic needs the mesh only, not an engine
    wa.mesh = pm
    wa.cortex_mask_full = np.asarray(pm.cortex_mask_full, dtype=bool)
    wa.orig_to_sub = np.asarray(pm.orig_to_sub)
    wa.n_vertices_full = int(wa.cortex_mask_full.shape[0])
    cortex = np.flatnonzero(mesh.cortex_mask)
    medial = np.flatnonzero(~mesh.cortex_mask)
    subset = [cortex[5], str(cortex[3]), cortex[5], medial[0], -1, 10 ** 9, "abc", float(cortex[7]), None]
    got = wa._sources(subset)
    want = {int(pm.orig_to_sub[c]) for c in (cortex[5], cortex[3], cortex[7])}
    assert set(got.tolist()) == want and got.size == 3
    bfs = list(pm.bfs)
    assert list(got) == sorted(got, key=bfs.index)  # BFS order
    assert np.array_equal(wa._sources(None), pm.bfs)
    assert wa._sources([]).size == 0


def test_nonmanifold_classification():
    """core_analysis.py:60-110 on crafted meshes: one face has three boundary edges; a fan of
    three faces on one edge makes both of its vertices non-manifold."""
    V = np.zeros((6, 3))
    r = A.classify_nonmanifold_vertices(V, np.array([[0, 1, 2]]))
    assert r["boundary_verts"] == {0, 1, 2} and r["non_manifold_verts"] == set()
    F = np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4]])
    r = A.classify_nonmanifold_vertices(V, F)
    assert r["non_manifold_verts"] == {0, 1}
    assert r["boundary_verts"] == {0, 1, 2, 3, 4} and r["also_boundary"] == {0, 1} and r["interior"] == set()
    assert A.classify_nonmanifold_vertices(V, np.zeros((0, 3), int))["interior"] == set()
    with pytest.raises(ValueError, match="expected \\(M, 3\\)"):
        A.classify_nonmanifold_vertices(V, np.zeros((2, 4), int))


def test_constructor_follows_the_reference():
    """engine_type must name this engine; an interior non-manifold cortical submesh warns as the
    reference does for engines without robust operators, before the engine is built."""
    import torch

    from fastcorticalwiring_b200 import _lib

    mesh = folded_icosphere(3, seed=1)
    with pytest.raises(ValueError, match="Unknown engine_type 'potpourri'"):
        A.WiringAnalysis(mesh.vertices, mesh.faces, mesh.cortex_mask, engine_type="potpourri")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible: the engine would be built")
    # a closed icosphere with a two-sided fin on an existing edge: an interior non-manifold edge
    V, F = mesh.vertices, mesh.faces
    a, b = F[0, 0], F[0, 1]
    V2 = np.vstack([V, V[a] + 1.0])
    F2 = np.vstack([F, [a, b, len(V)], [b, a, len(V)]])
    assert A.classify_nonmanifold_vertices(V2, F2)["interior"] == {int(a), int(b)}
    with pytest.warns(RuntimeWarning, match="Interior non-manifold vertices"):
        with pytest.raises(_lib.FCWError):
            A.WiringAnalysis(V2, F2, np.ones(len(V2), bool), metadata={"subject": "x"})
