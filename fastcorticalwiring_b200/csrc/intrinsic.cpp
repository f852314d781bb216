// Intrinsic Delaunay ("robust") operators: the cotan Laplacian and lumped mass of the
// intrinsic Delaunay triangulation of the mesh's tufted cover, reached by edge flips
// on intrinsic edge lengths (Bobenko & Springborn's flip algorithm on the cover and
// mollified lengths of Sharp & Crane, "A Laplacian for Nonmanifold Triangle Meshes",
// 2020).
//
// The reference's production engine builds its heat-method operators this way
// (potpourri3d's MeshHeatMethodDistanceSolver with use_robust=True,
// distance_engines.py:119-125; the reason is LEAN_MODE_IMPLEMENTATION.md:15: on
// real cortical meshes the extrinsic cotan operators corrupt a large share of the
// fields). Only the operators change: the heat operator M + tL and the Poisson
// operator L + shift*M use the intrinsic L and M, while the normalised gradient
// and its divergence stay on the mesh's own faces.
//
// The tufted cover doubles every face (a front and a back side sharing the
// vertices). Across a manifold interior edge fronts meet fronts and backs meet
// backs; across a boundary edge a face's front meets its own back, so an obtuse
// angle opposite a boundary edge is flipped too (the new edge joins the opposite
// vertex to itself). L and M are half those of the flipped cover. Non-manifold
// edges are kept as they are (the cover's cyclic gluing around them is not built).
// Faces no flip touched keep the extrinsic stiffness block and area of
// prepare_mesh, and a mesh that is already Delaunay gets the extrinsic operators
// bit for bit.
#include <algorithm>
#include <cmath>
#include <unordered_map>

#include "fcw_internal.h"

namespace fcw {

namespace {

inline int nxt(int h) { return 3 * (h / 3) + (h % 3 + 1) % 3; }

// Triangle area from its side lengths (Heron, in the stable form for sorted sides).
double tri_area(double a, double b, double c) {
    if (a < b) std::swap(a, b);
    if (a < c) std::swap(a, c);
    if (b < c) std::swap(b, c);
    const double p = (a + (b + c)) * (c - (a - b)) * (c + (a - b)) * (a + (b - c));
    return 0.25 * std::sqrt(p > 0.0 ? p : 0.0);
}

// Cotangent of the angle opposite side `opp` in the triangle with sides (opp, s1, s2).
double cot_opposite(double opp, double s1, double s2) {
    const double A = tri_area(opp, s1, s2);
    return (s1 * s1 + s2 * s2 - opp * opp) / (4.0 * A);
}

inline double dot3(const double* a, const double* b) { return (a[0] * b[0] + a[2] * b[2]) + a[1] * b[1]; }

}  // namespace

int intrinsic_delaunay(MeshPrep& m, double mollify_factor, int64_t& nflips, std::string& err) {
    const int64_t nf = m.nf, nv = m.nv, ncf = 2 * nf;  // cover faces: fronts, then backs
    const int32_t* F = m.F.data();
    const double* V = m.V.data();
    std::vector<int32_t> tail(3 * ncf), twin(3 * ncf, -1);
    std::vector<double> len(3 * ncf);
    // back of face f = (F0, F2, F1): slot 3 (nf + f) + c runs from corner c to c + 1 of that order
    static const int bc[3] = {0, 2, 1};
    for (int64_t f = 0; f < nf; ++f)
        for (int c = 0; c < 3; ++c) {
            tail[3 * f + c] = F[3 * f + c];
            tail[3 * (nf + f) + c] = F[3 * f + bc[c]];
        }
    for (int64_t h = 0; h < 3 * ncf; ++h) {
        const int64_t a = tail[h], b = tail[nxt((int)h)];
        double d[3] = {V[3 * b] - V[3 * a], V[3 * b + 1] - V[3 * a + 1], V[3 * b + 2] - V[3 * a + 2]};
        len[h] = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
    // gluing: per undirected edge, its front halfedges (one per incident face)
    {
        std::unordered_map<int64_t, std::vector<int32_t>> byedge;
        byedge.reserve((size_t)(3 * nf));
        for (int64_t h = 0; h < 3 * nf; ++h) {
            int64_t a = tail[h], b = tail[nxt((int)h)];
            if (a > b) std::swap(a, b);
            byedge[a * nv + b].push_back((int32_t)h);
        }
        // the back copy of front halfedge 3 f + c (same edge, opposite direction)
        auto back_of = [&](int32_t h) {
            const int32_t f = h / 3, c = h % 3;
            // front corner c -> c + 1 is back corner order (0, 2, 1): the back halfedge from
            // F[c + 1] to F[c]
            static const int slot[3] = {2, 1, 0};  // front edge (0,1) -> back slot 2 (F1 -> F0), ...
            return (int32_t)(3 * (nf + f) + slot[c]);
        };
        auto glue = [&](int32_t x, int32_t y) {
            twin[x] = y;
            twin[y] = x;
        };
        for (auto& kv : byedge) {
            const auto& hs = kv.second;
            if (hs.size() == 1) {
                glue(hs[0], back_of(hs[0]));  // boundary: the face's front meets its own back
            } else if (hs.size() == 2) {
                const int32_t h0 = hs[0], h1 = hs[1];
                if (tail[h0] != tail[h1]) {  // consistently oriented: fronts together, backs together
                    glue(h0, h1);
                    glue(back_of(h0), back_of(h1));
                } else {  // opposite orientations: each front meets the other's back
                    glue(h0, back_of(h1));
                    glue(h1, back_of(h0));
                }
            }
        }
    }
    // mollification: every corner's triangle inequality holds with margin delta
    double mean = 0.0;
    for (double x : len) mean += x;
    mean /= (double)std::max<int64_t>(1, 3 * ncf);
    const double delta = mollify_factor * mean;
    double eps = 0.0;
    for (int64_t f = 0; f < nf; ++f)
        for (int c = 0; c < 3; ++c) {
            const double a = len[3 * f + c], b = len[3 * f + (c + 1) % 3], cc = len[3 * f + (c + 2) % 3];
            eps = std::max(eps, delta - (a + b - cc));
        }
    if (eps > 0.0)
        for (double& x : len) x += eps;

    std::vector<uint8_t> orig(ncf, 1), queued(3 * ncf, 0);
    std::vector<int32_t> stack;
    for (int32_t h = 0; h < 3 * ncf; ++h)
        if (twin[h] > h) {
            stack.push_back(h);
            queued[h] = 1;
        }
    const int64_t cap = 64 * (3 * ncf) + 1000;
    int64_t steps = 0;
    nflips = 0;
    while (!stack.empty()) {
        if (++steps > cap) {
            err = "intrinsic Delaunay flips did not terminate";
            return 1;
        }
        const int32_t h = stack.back();
        stack.pop_back();
        queued[h] = 0;
        const int32_t t = twin[h];
        if (t < 0) continue;
        const int32_t h1 = nxt(h), h2 = nxt(h1), t1 = nxt(t), t2 = nxt(t1);
        const double lab = len[h], lbc = len[h1], lca = len[h2], lad = len[t1], ldb = len[t2];
        const double w = cot_opposite(lab, lbc, lca) + cot_opposite(lab, lad, ldb);
        if (!(w < -1e-10)) continue;  // Delaunay (or degenerate: leave it)
        // unfold the two triangles: a = (0, 0), b = (lab, 0), c above, d below
        const double xc = (lab * lab + lca * lca - lbc * lbc) / (2.0 * lab);
        const double yc = std::sqrt(std::max(0.0, lca * lca - xc * xc));
        const double xd = (lab * lab + lad * lad - ldb * ldb) / (2.0 * lab);
        const double yd = -std::sqrt(std::max(0.0, lad * lad - xd * xd));
        const double lcd = std::hypot(xc - xd, yc - yd);
        const int32_t va = tail[h], vb = tail[t], vc = tail[h2], vd = tail[t2];
        const int32_t f0 = h / 3, f1 = t / 3;
        // new faces (a, d, c) and (d, b, c); slots: f0 <- a->d, d->c, c->a; f1 <- d->b, b->c, c->d
        const int32_t s_ad = 3 * f0, s_dc = 3 * f0 + 1, s_ca = 3 * f0 + 2;
        const int32_t s_db = 3 * f1, s_bc = 3 * f1 + 1, s_cd = 3 * f1 + 2;
        const int32_t old_slot[4] = {t1, h2, t2, h1};  // a->d, c->a, d->b, b->c before the flip
        const int32_t new_slot[4] = {s_ad, s_ca, s_db, s_bc};
        int32_t old_twin[4];
        for (int k = 0; k < 4; ++k) old_twin[k] = twin[old_slot[k]];
        auto remap = [&](int32_t s) {
            for (int k = 0; k < 4; ++k)
                if (old_slot[k] == s) return new_slot[k];
            return s;
        };
        const double l_new[4] = {lad, lca, ldb, lbc};
        tail[s_ad] = va; tail[s_dc] = vd; tail[s_ca] = vc;
        tail[s_db] = vd; tail[s_bc] = vb; tail[s_cd] = vc;
        for (int k = 0; k < 4; ++k) len[new_slot[k]] = l_new[k];
        len[s_dc] = len[s_cd] = lcd;
        for (int k = 0; k < 4; ++k) twin[new_slot[k]] = old_twin[k] < 0 ? -1 : remap(old_twin[k]);
        for (int k = 0; k < 4; ++k)
            if (twin[new_slot[k]] >= 0) twin[twin[new_slot[k]]] = new_slot[k];
        twin[s_dc] = s_cd;
        twin[s_cd] = s_dc;
        orig[f0] = orig[f1] = 0;
        ++nflips;
        for (int k = 0; k < 4; ++k) {
            const int32_t s = new_slot[k], tw = twin[s];
            if (tw < 0) continue;
            const int32_t key = std::min(s, tw);
            if (!queued[key]) {
                queued[key] = 1;
                stack.push_back(key);
            }
        }
    }
    if (nflips == 0) return 0;  // already Delaunay: the extrinsic operators stand

    // operators of the intrinsic triangulation: L and M are half those of the cover. A face
    // whose two copies no flip touched adds its extrinsic G^T A G block and area once;
    // otherwise each copy adds half of its block (cotangents of its intrinsic lengths, or the
    // extrinsic block if that copy is untouched) and half its area. Entries sum per
    // (row, column) in cover-face order.
    struct Trip {
        int32_t col, row;
        int64_t pos;
        double val;
    };
    std::vector<Trip> tr;
    tr.reserve((size_t)(18 * nf));
    m.mass.assign(nv, 0.0);
    auto add_face = [&](int64_t cf, double wgt) {
        double blk[3][3];
        double area;
        int32_t v[3];
        const int64_t f = cf < nf ? cf : cf - nf;
        if (orig[cf]) {  // untouched copy: the extrinsic block on the front face's corners
            const double* g = &m.gb[9 * f];
            for (int i = 0; i < 3; ++i) {
                v[i] = F[3 * f + i];
                for (int j = 0; j < 3; ++j) blk[i][j] = m.grad_area[f] * dot3(g + 3 * i, g + 3 * j);
            }
            area = m.grad_area[f];
        } else {
            // side opposite corner i: the halfedge from corner i+1 to corner i+2
            const double o0 = len[3 * cf + 1], o1 = len[3 * cf + 2], o2 = len[3 * cf];
            const double ct[3] = {cot_opposite(o0, o1, o2), cot_opposite(o1, o2, o0), cot_opposite(o2, o0, o1)};
            for (int i = 0; i < 3; ++i) {
                v[i] = tail[3 * cf + i];
                for (int j = 0; j < 3; ++j) {
                    if (i == j) blk[i][j] = 0.5 * (ct[(i + 1) % 3] + ct[(i + 2) % 3]);
                    else blk[i][j] = -0.5 * ct[3 - i - j];
                }
            }
            area = tri_area(o0, o1, o2);
        }
        for (int i = 0; i < 3; ++i) {
            m.mass[v[i]] += wgt * (area / 3.0);
            for (int j = 0; j < 3; ++j) tr.push_back({v[j], v[i], (int64_t)(3 * i + j) * ncf + cf, wgt * blk[i][j]});
        }
    };
    for (int64_t f = 0; f < nf; ++f) {
        if (orig[f] && orig[nf + f]) {
            add_face(f, 1.0);
        } else {
            add_face(f, 0.5);
            add_face(nf + f, 0.5);
        }
    }
    std::sort(tr.begin(), tr.end(), [](const Trip& a, const Trip& b) {
        if (a.col != b.col) return a.col < b.col;
        if (a.row != b.row) return a.row < b.row;
        return a.pos < b.pos;
    });
    m.Lp.assign(nv + 1, 0);
    m.Li.clear();
    m.Lx.clear();
    for (size_t k = 0; k < tr.size();) {
        size_t l = k;
        double sum = 0.0;
        while (l < tr.size() && tr[l].col == tr[k].col && tr[l].row == tr[k].row) sum += tr[l++].val;
        m.Li.push_back(tr[k].row);
        m.Lx.push_back(sum);
        m.Lp[tr[k].col + 1] = (int64_t)m.Li.size();
        k = l;
    }
    for (int64_t c = 0; c < nv; ++c) m.Lp[c + 1] = std::max(m.Lp[c + 1], m.Lp[c]);
    // the flipped cover for checks: faces as corner vertices, and per halfedge its length and twin
    m.itri.assign(tail.begin(), tail.end());
    m.ilen = len;
    m.itwin = twin;
    return 0;
}

}  // namespace fcw
