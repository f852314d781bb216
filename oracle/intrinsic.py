"""Intrinsic Delaunay operators on the CPU, restated independently of the engine's C++.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). The robust operators of the
reference's production engine (potpourri3d MeshHeatMethodDistanceSolver with
use_robust=True, distance_engines.py:119-125, rationale LEAN_MODE_IMPLEMENTATION.md:15)
are the cotan Laplacian and lumped mass of the intrinsic Delaunay triangulation
of the mesh. potpourri3d is not installed here (its source is not in the reference
either), so this restates the published algorithm: Bobenko & Springborn's edge
flips on intrinsic lengths, on Sharp & Crane's tufted cover of the mesh (every face
doubled; a boundary edge glues a face's front to its own back) with their
mollification (lengths + eps so every triangle inequality holds with margin 1e-6 x
mean length); L and M are half those of the flipped cover. Non-manifold edges are
not glued. Faces no flip touched keep the extrinsic G^T A G block
(oracle.heat.operators), so a Delaunay mesh gets the extrinsic operators unchanged.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .heat import gradient_basis


def _area(a, b, c):
    s = sorted((a, b, c), reverse=True)
    a, b, c = s
    p = (a + (b + c)) * (c - (a - b)) * (c + (a - b)) * (a + (b - c))
    return 0.25 * np.sqrt(max(p, 0.0))


def _cot(opp, s1, s2):
    return (s1 * s1 + s2 * s2 - opp * opp) / (4.0 * _area(opp, s1, s2))


def intrinsic_delaunay(V, F, mollify_factor=1e-6, tol=1e-10):
    """(tri, length, twin, touched, nflips): the intrinsic Delaunay triangulation of the
    tufted cover of the mesh.

    The cover has 2 nf faces: the fronts (the mesh's faces) then the backs (corners in the
    order 0, 2, 1). Across a manifold interior edge fronts meet fronts and backs meet
    backs; across a boundary edge a face's front meets its own back. tri[f] = corner
    vertices of cover face f; length[f, c] / twin[f, c] belong to the halfedge from corner
    c to corner c+1 (twin as a flat index 3 f + c, -1 on non-manifold edges).
    """
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F, dtype=np.int64)
    nf = F.shape[0]
    tri = np.concatenate([F, F[:, [0, 2, 1]]], axis=0)
    length = np.linalg.norm(V[np.roll(tri, -1, axis=1)] - V[tri], axis=2)
    twin = -np.ones((2 * nf, 3), dtype=np.int64)
    back_slot = (2, 1, 0)  # the back copy of front halfedge (f, c)
    edges = {}
    for f in range(nf):
        for c in range(3):
            a, b = int(F[f, c]), int(F[f, (c + 1) % 3])
            edges.setdefault((min(a, b), max(a, b)), []).append((f, c, a))

    def glue(x, y):
        twin.flat[x] = y
        twin.flat[y] = x

    for hs in edges.values():
        if len(hs) == 1:
            f, c, _ = hs[0]
            glue(3 * f + c, 3 * (nf + f) + back_slot[c])
        elif len(hs) == 2:
            (f0, c0, a0), (f1, c1, a1) = hs
            if a0 != a1:
                glue(3 * f0 + c0, 3 * f1 + c1)
                glue(3 * (nf + f0) + back_slot[c0], 3 * (nf + f1) + back_slot[c1])
            else:
                glue(3 * f0 + c0, 3 * (nf + f1) + back_slot[c1])
                glue(3 * f1 + c1, 3 * (nf + f0) + back_slot[c0])
    delta = mollify_factor * float(length.mean())
    margin = length[:nf] + np.roll(length[:nf], -1, axis=1) - np.roll(length[:nf], -2, axis=1)
    eps = max(0.0, float(np.max(delta - margin)))
    if eps > 0.0:
        length = length + eps
    touched = np.zeros(2 * nf, dtype=bool)
    stack = [h for h in range(6 * nf) if twin.flat[h] > h]
    nflips = 0

    def nxt(h):
        return 3 * (h // 3) + (h % 3 + 1) % 3

    while stack:
        h = stack.pop()
        t = int(twin.flat[h])
        if t < 0:
            continue
        h1, t1 = nxt(h), nxt(t)
        h2, t2 = nxt(h1), nxt(t1)
        lab, lbc, lca, lad, ldb = (length.flat[h], length.flat[h1], length.flat[h2], length.flat[t1],
                                   length.flat[t2])
        if not (_cot(lab, lbc, lca) + _cot(lab, lad, ldb) < -tol):
            continue
        xc = (lab * lab + lca * lca - lbc * lbc) / (2.0 * lab)
        yc = np.sqrt(max(0.0, lca * lca - xc * xc))
        xd = (lab * lab + lad * lad - ldb * ldb) / (2.0 * lab)
        yd = -np.sqrt(max(0.0, lad * lad - xd * xd))
        lcd = float(np.hypot(xc - xd, yc - yd))
        va, vb = tri.flat[h], tri.flat[t]
        vc, vd = tri.flat[h2], tri.flat[t2]
        f0, f1 = h // 3, t // 3
        # the quad (a, d, b, c) split by c-d into (a, d, c) and (d, b, c)
        old = {t1: 3 * f0, h2: 3 * f0 + 2, t2: 3 * f1, h1: 3 * f1 + 1}
        outer = {s: int(twin.flat[s]) for s in old}
        lens = {s: float(length.flat[s]) for s in old}
        tri[f0] = (va, vd, vc)
        tri[f1] = (vd, vb, vc)
        for s, n in old.items():
            length.flat[n] = lens[s]
        length.flat[3 * f0 + 1] = length.flat[3 * f1 + 2] = lcd
        for s, n in old.items():
            o = outer[s]
            o = old.get(o, o) if o >= 0 else -1
            twin.flat[n] = o
            if o >= 0:
                twin.flat[o] = n
        twin.flat[3 * f0 + 1] = 3 * f1 + 2
        twin.flat[3 * f1 + 2] = 3 * f0 + 1
        touched[f0] = touched[f1] = True
        nflips += 1
        for n in old.values():
            if twin.flat[n] >= 0:
                stack.append(min(n, int(twin.flat[n])))
    return tri, length, twin, touched, nflips


def robust_operators(V, F, mollify_factor=1e-6):
    """(L, mass, nflips): half the cotan Laplacian and lumped mass of the flipped cover (a face
    whose two copies are both untouched adds its extrinsic block once); L as CSC."""
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F, dtype=np.int64)
    nv, nf = V.shape[0], F.shape[0]
    tri, length, twin, touched, nflips = intrinsic_delaunay(V, F, mollify_factor)
    area, g0, g1, g2 = gradient_basis(V, F)
    g = (g0, g1, g2)
    rows, cols, vals = [], [], []
    mass = np.zeros(nv)

    def add(cf, w):
        f = cf if cf < nf else cf - nf
        if not touched[cf]:
            v = F[f]
            blk = np.array([[area[f] * np.dot(g[i][f], g[j][f]) for j in range(3)] for i in range(3)])
            a = area[f]
        else:
            v = tri[cf]
            o = (length[cf, 1], length[cf, 2], length[cf, 0])  # side opposite corner i
            ct = [_cot(o[0], o[1], o[2]), _cot(o[1], o[2], o[0]), _cot(o[2], o[0], o[1])]
            blk = np.empty((3, 3))
            for i in range(3):
                for j in range(3):
                    blk[i, j] = 0.5 * (ct[(i + 1) % 3] + ct[(i + 2) % 3]) if i == j else -0.5 * ct[3 - i - j]
            a = _area(*o)
        for i in range(3):
            mass[v[i]] += w * (a / 3.0)
            for j in range(3):
                rows.append(v[i])
                cols.append(v[j])
                vals.append(w * blk[i, j])

    for f in range(nf):
        if not touched[f] and not touched[nf + f]:
            add(f, 1.0)
        else:
            add(f, 0.5)
            add(nf + f, 0.5)
    L = sp.csc_matrix((np.array(vals), (np.array(rows), np.array(cols))), shape=(nv, nv))
    L.sum_duplicates()
    return L, mass, nflips
