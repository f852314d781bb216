"""CPU restatement of the heat-method distance path and its per-source metrics.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). Functions cite the
reference code they restate:

* mean_edge_length        distance_engines.py:17-21
* gradient_basis          fastcw_lean.py:375-391
* operators               fastcw_lean.py:394-413
* normalized_divergence   fastcw_lean.py:416-442   (C, lean_oracle.c)
* HeatOracle              fastcw_lean.py:467-531   (factor of M + tL and L + shift*M,
                                                    delta RHS, shift phi(s) = 0); robust=True
                                                    takes L and M from oracle.intrinsic
                                                    (distance_engines.py:119-125)
* field_health            lean_geometry.py:343-357
* msd_and_boundary        core_analysis.py:1566-1581
* source_geometry         lean_geometry.py:302-340 (C, lean_oracle.c)

Factorisation: the reference uses CHOLMOD when scikit-sparse is installed and
SciPy SuperLU otherwise (fastcw_lean.py:445-464, 490-497). Neither CHOLMOD nor
the production potpourri3d solver is installed here; the oracle factors with
SciPy SuperLU in symmetric mode with no pivoting (the same matrix, an LDL-like
factor) after a coordinate nested-dissection reordering, which agrees with the
reference's pivoting SuperLU to FP64 rounding and factors large meshes in
seconds instead of minutes.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build_oracle_library(force: bool = False) -> str:
    """Compile lean_oracle.c into oracle/_build/liboracle.so (no FMA contraction)."""
    src = os.path.join(_HERE, "lean_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                               "-o", _LIB_PATH, src, "-lm"])
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build_oracle_library())
        P = ctypes.c_void_p
        I = ctypes.c_int64
        D = ctypes.c_double
        lib.oracle_source_geometry.restype = I
        lib.oracle_source_geometry.argtypes = [P, P, I, P, P, P, P, D, P, I, P, I, D, I, P, P, P, P, P, P, P]
        lib.oracle_field_eval.restype = D
        lib.oracle_field_eval.argtypes = [ctypes.c_int, D, P, P, I, P, P, P, P, D, D, I, P, P, P, P]
        lib.oracle_normalized_divergence.restype = None
        lib.oracle_normalized_divergence.argtypes = [P, I, I, P, I, P, P, P, P, P]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def mean_edge_length(V, F):
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0).astype(np.int64)
    e.sort(axis=1)
    e = np.unique(e, axis=0)
    return float(np.mean(np.linalg.norm(V[e[:, 1]] - V[e[:, 0]], axis=1)))


def gradient_basis(V, F):
    """Per-face area and the gradients of the three hat functions (3-vectors)."""
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F, dtype=np.int64)
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    ab, ac = b - a, c - a
    n = np.cross(ab, ac)
    twice = np.linalg.norm(n, axis=1)
    if np.any(twice <= 0.0):
        raise ValueError("Zero-area faces must be removed before building the heat engine.")
    area = 0.5 * twice
    unit = n / twice[:, None]
    scale = 1.0 / (2.0 * area)
    g1 = np.cross(ac, unit) * scale[:, None]
    g2 = np.cross(unit, ab) * scale[:, None]
    g0 = -g1 - g2
    return area, np.ascontiguousarray(g0), np.ascontiguousarray(g1), np.ascontiguousarray(g2)


def operators(V, F):
    """Stiffness L = G^T diag(area) G (CSC, duplicates summed) and lumped mass diag(area/3)."""
    F = np.asarray(F, dtype=np.int64)
    nv = int(np.asarray(V).shape[0])
    area, g0, g1, g2 = gradient_basis(V, F)
    g = (g0, g1, g2)
    r, c, v = [], [], []
    for i in range(3):
        for j in range(3):
            r.append(F[:, i])
            c.append(F[:, j])
            v.append(area * np.einsum("ij,ij->i", g[i], g[j]))
    L = sp.csc_matrix((np.concatenate(v), (np.concatenate(r), np.concatenate(c))), shape=(nv, nv))
    L.sum_duplicates()
    mass = np.zeros(nv)
    for i in range(3):
        np.add.at(mass, F[:, i], area / 3.0)
    return L, mass, area, g0, g1, g2


def normalized_divergence(u, F, area, g0, g1, g2):
    """Fused grad -> normalise -> divergence for u of shape (nv, k)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    if u.ndim == 1:
        u = u[:, None]
    Fi = np.ascontiguousarray(F, dtype=np.int32)
    out = np.empty_like(u)
    _load().oracle_normalized_divergence(_p(u), u.shape[0], u.shape[1], _p(Fi), Fi.shape[0],
                                         _p(np.ascontiguousarray(area)), _p(g0), _p(g1), _p(g2), _p(out))
    return out


def coordinate_dissection(V, A, leaf=128):
    """Fill-reducing order by recursive coordinate bisection of the vertex graph.

    Each part is split at the median of its widest coordinate; the vertices of
    the first half that touch the second half form the separator, numbered
    last. Only the factorisation's speed depends on this order, never its result.
    """
    A = sp.csr_matrix(A, copy=True)
    A.data = np.ones_like(A.data)  # pattern only (the stiffness has negative off-diagonals)
    n = A.shape[0]
    order = np.empty(n, dtype=np.int64)
    side = np.zeros(n, dtype=np.int8)
    stack = [(np.arange(n), 0, n)]
    while stack:
        verts, lo, hi = stack.pop()
        if verts.size <= leaf:
            order[lo:hi] = verts
            continue
        X = V[verts]
        ax = int(np.argmax(X.max(axis=0) - X.min(axis=0)))
        cut = np.median(X[:, ax])
        first = X[:, ax] < cut
        if first.all() or not first.any():
            order[lo:hi] = verts
            continue
        side[verts] = 2
        side[verts[first]] = 0
        side[verts[~first]] = 1
        touches = (A[verts[first]] @ (side == 1).astype(np.float64)) > 0
        sep = verts[first][touches]
        a = verts[first][~touches]
        b = verts[~first]
        side[verts] = 0
        order[hi - sep.size:hi] = sep
        stack.append((a, lo, lo + a.size))
        stack.append((b, lo + a.size, lo + a.size + b.size))
    return order


class _SymmetricFactor:
    """Sparse LU in SuperLU's symmetric mode (diagonal pivots) on a dissection-ordered matrix."""

    def __init__(self, A, order=None):
        from scipy.sparse.linalg import splu

        A = sp.csc_matrix(A)
        if order is None:
            self._p = None
            self._lu = splu(A, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0, options=dict(SymmetricMode=True))
        else:
            self._p = np.asarray(order)
            Ap = A[self._p][:, self._p].tocsc()
            self._lu = splu(Ap, permc_spec="NATURAL", diag_pivot_thresh=0.0, options=dict(SymmetricMode=True))

    def solve(self, B):
        B = np.asarray(B)
        if self._p is None:
            return self._lu.solve(np.asfortranarray(B))
        x = self._lu.solve(np.asfortranarray(B[self._p]))
        out = np.empty_like(x)
        out[self._p] = x
        return out


class HeatOracle:
    """Heat-method distances with the consistent extrinsic operators.

    t = t_coef * h^2 with h the mean unique-edge length and t_coef = (L/h)^2
    for a diffusion length L (distance_engines.py:119-122, fastcw_lean.py:485-489);
    Poisson operator L + shift * M (fastcw_lean.py:500).
    """

    def __init__(self, V, F, diffusion_length_mm=0.7, poisson_shift=1e-10, t_coef=None, ordering="dissection",
                 robust=False):
        V = np.ascontiguousarray(V, dtype=np.float64)
        F = np.ascontiguousarray(F, dtype=np.int32)
        L, mass, area, g0, g1, g2 = operators(V, F)
        self.n_flips = 0
        if robust:  # intrinsic Delaunay L and M; the divergence stays on the mesh's faces
            from .intrinsic import robust_operators

            L, mass, self.n_flips = robust_operators(V, F)
        h = mean_edge_length(V, F)
        if t_coef is None:
            t_coef = (float(diffusion_length_mm) / h) ** 2
        self.t_coef = float(t_coef)
        self.t = float(t_coef) * h * h
        M = sp.diags(mass, format="csc")
        self.L, self.mass = L, mass
        self.heat_matrix = (M + self.t * L).tocsc()
        self.poisson_matrix = (L + poisson_shift * M).tocsc()
        order = coordinate_dissection(V, L) if ordering == "dissection" else None
        self._heat = _SymmetricFactor(self.heat_matrix, order)
        self._poisson = _SymmetricFactor(self.poisson_matrix, order)
        self.F, self.area, self.g0, self.g1, self.g2 = F, area, g0, g1, g2
        self.n_vertices = V.shape[0]

    def heat(self, sources):
        src = np.asarray(sources, dtype=np.int64).reshape(-1)
        rhs = np.zeros((self.n_vertices, src.size))
        rhs[src, np.arange(src.size)] = 1.0
        return np.ascontiguousarray(self._heat.solve(rhs))

    def divergence(self, u):
        return normalized_divergence(u, self.F, self.area, self.g0, self.g1, self.g2)

    def poisson(self, div, sources):
        src = np.asarray(sources, dtype=np.int64).reshape(-1)
        phi = np.asarray(self._poisson.solve(div))
        return phi - phi[src, np.arange(src.size)][None, :]

    def distances(self, sources):
        """(k, nv) array, row j = distances from sources[j] (fastcw_lean.py:504-531)."""
        u = self.heat(sources)
        phi = self.poisson(self.divergence(u), sources)
        return np.ascontiguousarray(phi.T)


def field_health(d, V, src, h, neg_frac_tol=1e-3, chord_frac_tol=1e-3):
    """(negative fraction, chord-violation fraction, bad) for one field."""
    d = np.asarray(d, dtype=np.float64)
    if not np.isfinite(d).all():
        return float("nan"), float("nan"), True
    chord = np.linalg.norm(V - V[int(src)], axis=1)
    neg = float(np.mean(d < -h))
    viol = float(np.mean(d < 0.9 * chord - h))
    return neg, viol, bool(neg > neg_frac_tol or viol > chord_frac_tol)


def msd_and_boundary(d, vertex_area, boundary, eps=1e-6):
    """(msd_unweighted, msd_weighted, dist_to_boundary) in float64, NaN where undefined."""
    if boundary.size:
        bd = d[boundary]
        bd = bd[np.isfinite(bd)]
        dist_b = float(np.min(bd)) if bd.size else float("nan")
    else:
        dist_b = float("inf")
    valid = (d > eps) & np.isfinite(d)
    msd_u = msd_w = float("nan")
    if np.any(valid):
        dv = d[valid]
        w = vertex_area[valid]
        wsum = float(np.sum(w))
        msd_u = float(np.mean(dv))
        msd_w = float((dv * w).sum() / wsum) if np.isfinite(wsum) and wsum > 0.0 else float("nan")
    return msd_u, msd_w, dist_b


def source_geometry(d, F, area, g11, g12, g22, width, targets, fracs, rtol=1e-10, max_iter=60):
    """(radii, perimeters, extra_r, extra_a, n_eval) for one distance field."""
    lib = _load()
    d = np.ascontiguousarray(d, dtype=np.float64)
    Fi = np.ascontiguousarray(F, dtype=np.int32)
    nf = Fi.shape[0]
    t = np.ascontiguousarray(targets, dtype=np.float64)
    fr = np.ascontiguousarray(fracs, dtype=np.float64)
    nt, m = t.size, fr.size
    dmax, order, lng = np.empty(nf), np.empty(nf, np.int32), np.empty(nf, np.int32)
    radii, perim = np.empty(nt), np.empty(nt)
    ne = max(0, nt - 1) * m
    er, ea = np.empty(ne), np.empty(ne)
    n = lib.oracle_source_geometry(_p(d), _p(Fi), nf, _p(area), _p(g11), _p(g12), _p(g22), float(width),
                                   _p(t), nt, _p(fr), m, float(rtol), int(max_iter), _p(dmax), _p(order),
                                   _p(lng), _p(radii), _p(perim), _p(er), _p(ea))
    if n < 0:
        raise MemoryError("oracle geometry allocation failed")
    return radii, perim, er, ea, int(n)


def field_eval(mode, r, d, F, area, g11, g12, g22, width, rtol=1e-10, max_iter=60):
    """One evaluation: mode 'area', 'darea', 'perimeter' or 'radius' (r is then the target)."""
    lib = _load()
    code = {"area": 0, "darea": 1, "perimeter": 2, "radius": 3}[mode]
    d = np.ascontiguousarray(d, dtype=np.float64)
    Fi = np.ascontiguousarray(F, dtype=np.int32)
    nf = Fi.shape[0]
    dmax, order, lng = np.empty(nf), np.empty(nf, np.int32), np.empty(nf, np.int32)
    nl = ctypes.c_int64(0)
    v = lib.oracle_field_eval(code, float(r), _p(d), _p(Fi), nf, _p(area), _p(g11), _p(g12), _p(g22),
                              float(width), float(rtol), int(max_iter), _p(dmax), _p(order), _p(lng),
                              ctypes.byref(nl))
    return float(v), int(nl.value)


def source_metrics(d, src, pm, targets, n_between=3, eps=1e-6, rtol=1e-10, max_iter=60):
    """All per-source outputs for one field, following core_analysis.py:1550-1611.

    Returns a dict with health (neg, viol, bad), msd_u, msd_w, dist_b, radii,
    perim, extra_r, extra_a. A flagged field keeps its raw numbers here; the
    caller writes NaN for it, as the reference loop does.
    """
    fracs = np.arange(1, n_between + 1, dtype=np.float64) / (n_between + 1.0)
    neg, viol, bad = field_health(d, pm.V, src, pm.health_h)
    msd_u, msd_w, dist_b = msd_and_boundary(d, pm.vertex_area, pm.boundary, eps)
    radii, perim, er, ea, n_eval = source_geometry(d, pm.F, pm.lean_area, pm.g11, pm.g12, pm.g22,
                                                   pm.bin_width, targets, fracs, rtol, max_iter)
    return dict(neg=neg, viol=viol, bad=bad, msd_u=msd_u, msd_w=msd_w, dist_b=dist_b, radii=radii,
                perim=perim, extra_r=er, extra_a=ea, n_eval=n_eval)
