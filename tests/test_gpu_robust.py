"""Robust (intrinsic Delaunay) operators on the device (needs a B200).

use_robust=True builds the heat and Poisson operators from the intrinsic Delaunay
triangulation of the mesh's tufted cover, as the reference's production engine does
(distance_engines.py:119-125); the divergence stays on the mesh's faces. The oracle
(oracle.HeatOracle(robust=True)) restates the same operators independently. Checks:
the engine against that oracle in FP64 and in the mixed form (the bars of the
extrinsic engine); the sphere's closed forms; and the reason the reference uses these
operators (LEAN_MODE_IMPLEMENTATION.md:15): on jittered meshes the extrinsic operators'
fields fail the health screen more often than the robust ones.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import engine, mesh as M  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere, unit_icosphere  # noqa: E402

SCALES = M.RUNNER_SCALES


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@pytest.fixture(scope="module")
def l4j():
    import oracle

    m = folded_icosphere(4, seed=0, jitter=0.2)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    src = pm.bfs[np.linspace(0, pm.n_vertices - 1, 48).astype(int)]
    ho = oracle.HeatOracle(pm.V, pm.F, robust=True)
    assert ho.n_flips > 0
    phi = ho.distances(src)
    targets = pm.targets(SCALES)
    ref = [oracle.source_metrics(phi[j], int(s), pm, targets) for j, s in enumerate(src)]
    eng = engine.HeatEngine(pm.V, pm.F, robust=1, block_k=64)
    yield dict(pm=pm, src=src, phi=phi, ref=ref, targets=targets, eng=eng, flips=ho.n_flips)
    eng.close()


def test_robust_engine_reports_its_flips(l4j):
    assert l4j["eng"].info()["n_flips"] == l4j["flips"]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-4)])
def test_robust_distances_match_oracle(l4j, precision, tol):
    d = l4j["eng"].compute_distances(l4j["src"], precision=precision)
    err = np.max(np.abs(d - l4j["phi"]), axis=1) / np.max(np.abs(l4j["phi"]), axis=1)
    print(f"\nROBUST L4j {precision} phi err {err.max():.2e}")
    assert err.max() <= tol


@pytest.mark.parametrize("precision,tol,msd_tol", [("fp64", 1e-9, 1e-9), ("mixed", 1e-4, 1e-5)])
def test_robust_metrics_match_oracle(l4j, precision, tol, msd_tol):
    r = engine.split_records(l4j["eng"].compute_metrics(l4j["src"], l4j["targets"], 3, precision=precision),
                             len(SCALES), 3)
    for j, o in enumerate(l4j["ref"]):
        if precision == "fp64":
            assert bool(r["bad"][j]) == o["bad"]
        if r["bad"][j] or o["bad"]:
            continue
        assert np.max(_rel(r["radii"][j], o["radii"])) <= tol
        assert np.max(_rel(r["perim"][j], o["perim"])) <= tol
        assert _rel(r["msd_w"][j], o["msd_w"]) <= msd_tol


def test_robust_sphere_closed_forms():
    R = 70.0
    V, F = unit_icosphere(6)
    pm = M.prepare(V * R, F, np.ones(len(V), bool))
    scales = np.array([0.002, 0.01, 0.05, 0.2])
    targets = pm.targets(scales)
    src = pm.bfs[np.linspace(0, pm.n_vertices - 1, 8).astype(int)]
    eng = engine.HeatEngine(pm.V, pm.F, robust=1)
    try:
        r = engine.split_records(eng.compute_metrics(src, targets, 3, precision="fp64"), scales.size, 3)
    finally:
        eng.close()
    frac = targets / (4.0 * np.pi * R * R)
    r_cf = R * np.arccos(1.0 - 2.0 * frac)
    p_cf = 2.0 * np.pi * R * np.sin(r_cf / R)
    assert not r["bad"].any()
    assert np.max(np.abs(r["radii"] - r_cf) / r_cf) <= 0.04
    assert np.max(np.abs(r["perim"] - p_cf) / p_cf) <= 0.02


@pytest.mark.parametrize("level,n", [(4, None), (6, 4096)])
def test_robust_operators_flag_fewer_fields_on_jittered_meshes(level, n):
    m = folded_icosphere(level, seed=0, jitter=0.2)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    src = pm.bfs if n is None else pm.bfs[np.linspace(0, pm.n_vertices - 1, n).astype(int)]
    flagged = {}
    for robust in (0, 1):
        eng = engine.HeatEngine(pm.V, pm.F, robust=robust)
        try:
            r = engine.split_records(eng.compute_metrics(src, pm.targets(SCALES), 3, precision="fp64"),
                                     len(SCALES), 3)
        finally:
            eng.close()
        flagged[robust] = int(r["bad"].sum())
    print(f"\nROBUST L{level}j flagged fields: extrinsic {flagged[0]} robust {flagged[1]} of {src.size}")
    assert flagged[1] <= flagged[0]
    if flagged[0] > 0:
        assert flagged[1] < flagged[0]
