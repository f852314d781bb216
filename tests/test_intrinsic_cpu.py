"""Robust (intrinsic Delaunay) operators on the host, against the oracle's restatement.

The production engine of the reference builds its heat-method operators on the
intrinsic Delaunay triangulation (potpourri3d, use_robust=True,
distance_engines.py:119-125). potpourri3d is absent, so what can be pinned is pinned
here: the engine's C++ flips agree with the oracle's independent restatement; every
interior edge of the result satisfies the Delaunay criterion (so every cotan weight is
nonnegative and L is an M-matrix); flips preserve the intrinsic metric (total area);
a mesh that is already Delaunay keeps the extrinsic operators bit for bit.
"""
import numpy as np
import pytest

import oracle
from fastcorticalwiring_b200 import _lib, mesh as M
from fastcorticalwiring_b200.meshgen import folded_icosphere, unit_icosphere


def _cot(opp, s1, s2):
    a, b, c = sorted((opp, s1, s2), reverse=True)
    A = 0.25 * np.sqrt(max((a + (b + c)) * (c - (a - b)) * (c + (a - b)) * (a + (b - c)), 0.0))
    return (s1 * s1 + s2 * s2 - opp * opp) / (4.0 * A)


@pytest.mark.parametrize("level,jitter,seed", [(4, 0.2, 0), (5, 0.2, 1), (4, 0.0, 2)])
def test_flips_match_the_oracle_and_reach_a_delaunay_triangulation(level, jitter, seed):
    m = folded_icosphere(level, seed=seed, jitter=jitter)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    r = _lib.intrinsic_operators(pm.V, pm.F)
    L_ref, mass_ref, nfl = oracle.robust_operators(pm.V, pm.F)
    assert r["nflips"] == nfl and nfl > 0
    assert abs(r["L"] - L_ref).max() <= 1e-13 * abs(L_ref).max()
    assert np.max(np.abs(r["mass"] - mass_ref)) <= 1e-13 * mass_ref.max()
    L = r["L"].tocoo()
    off = L.row != L.col
    assert np.all(L.data[off] <= 0.0)                     # all cotan weights nonnegative
    assert abs(r["L"] - r["L"].T).max() <= 1e-15 * abs(r["L"]).max()  # symmetric (to summation order)
    assert np.max(np.abs(np.asarray(r["L"].sum(axis=1)).ravel())) <= 1e-12
    # total area unchanged by the flips
    area = oracle.gradient_basis(pm.V, pm.F)[0]
    assert abs(r["mass"].sum() - area.sum()) <= 1e-10 * area.sum()
    # every interior edge of the intrinsic triangulation is Delaunay
    tri, ln, tw = r["tri"], r["len"].ravel(), r["twin"].ravel()
    nxt = lambda h: 3 * (h // 3) + (h % 3 + 1) % 3  # noqa: E731
    for h in np.flatnonzero(tw >= 0):
        t = tw[h]
        h1, t1 = nxt(h), nxt(t)
        w = _cot(ln[h], ln[h1], ln[nxt(h1)]) + _cot(ln[h], ln[t1], ln[nxt(t1)])
        assert w >= -1e-9, (h, w)
    # the extrinsic operator of the same mesh has negative weights (that is why it flips)
    Le = oracle.operators(pm.V, pm.F)[0].tocoo()
    assert np.any(Le.data[Le.row != Le.col] > 0.0)


def test_delaunay_mesh_keeps_the_extrinsic_operators():
    """No flip on a Delaunay mesh: the engine keeps the operators of prepare_mesh (returned
    untouched), which are the extrinsic ones (here against the oracle's assembly)."""
    V, F = unit_icosphere(3)
    V = V * 70.0
    r = _lib.intrinsic_operators(V, F)
    assert r["nflips"] == 0 and r["tri"] is None
    L, mass = oracle.operators(V, F)[:2]
    assert abs(r["L"] - L).max() <= 1e-15 * abs(L).max()
    assert np.max(np.abs(r["mass"] - mass)) <= 1e-15 * mass.max()
