// Host-side per-mesh preparation: operators, face data, vertex areas.
//
// Each block restates the reference computation it cites, with the same
// operation order so that FP64 values agree bit for bit with the NumPy
// reference where NumPy itself sums sequentially (no FMA contraction: this
// file is compiled with -ffp-contract=off).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "fcw_internal.h"

namespace fcw {

namespace {

inline void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// numpy.einsum("ij,ij->i") over 3 columns accumulates as (a0 b0 + a2 b2) + a1 b1.
inline double einsum_dot3(const double* a, const double* b) { return (a[0] * b[0] + a[2] * b[2]) + a[1] * b[1]; }

inline double norm3(const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// numpy.quantile(x, q) with the default 'linear' method, including NumPy's
// two-sided lerp (a + (b-a)*t, or b - (b-a)*(1-t) when t >= 0.5).
double np_quantile(std::vector<double> x, double q) {
    const int64_t n = (int64_t)x.size();
    double vidx = (double)(n - 1) * q;
    double lo_f = std::floor(vidx);
    int64_t lo = (int64_t)lo_f, hi = std::min<int64_t>(lo + 1, n - 1);
    double t = vidx - lo_f;
    std::nth_element(x.begin(), x.begin() + lo, x.end());
    double a = x[lo];
    double b = a;
    if (hi != lo) b = *std::min_element(x.begin() + lo + 1, x.end());
    double diff = b - a;
    if (t >= 0.5) return b - diff * (1.0 - t);
    return a + diff * t;
}

// numpy.median: middle element, or the mean of the two middle elements.
double np_median(std::vector<double> x) {
    const int64_t n = (int64_t)x.size();
    int64_t k = n / 2;
    std::nth_element(x.begin(), x.begin() + k, x.end());
    double b = x[k];
    if (n % 2) return b;
    double a = *std::max_element(x.begin(), x.begin() + k);
    return (a + b) / 2.0;
}

}  // namespace

int prepare_mesh(const double* V, int64_t nv, const int32_t* F, int64_t nf, MeshPrep& m, std::string& err) {
    if (nv <= 0 || nf <= 0) { err = "mesh has no vertices or no faces"; return 1; }
    for (int64_t i = 0; i < 3 * nf; ++i) {
        if (F[i] < 0 || F[i] >= nv) { err = "face index out of range"; return 1; }
    }
    for (int64_t i = 0; i < 3 * nv; ++i) {
        if (!std::isfinite(V[i])) { err = "non-finite vertex coordinate"; return 1; }
    }
    m.nv = nv; m.nf = nf;
    m.V.assign(V, V + 3 * nv);
    m.F.assign(F, F + 3 * nf);

    // Unique undirected edges (a < b) in ascending (a, b) order, the order of the reference's
    // sorted unique edge list (distance_engines.py:17-21): bucketed by a, each bucket's b
    // sorted; the mean edge length sums them in that order. Free edges (one face) give the
    // boundary vertices (core_analysis.py:651-665).
    {
        std::vector<int64_t> eptr(nv + 1, 0);
        for (int64_t f = 0; f < nf; ++f)
            for (int c = 0; c < 3; ++c) eptr[std::min(F[3 * f + c], F[3 * f + (c + 1) % 3]) + 1]++;
        for (int64_t v = 0; v < nv; ++v) eptr[v + 1] += eptr[v];
        std::vector<int32_t> eb(3 * nf);
        {
            std::vector<int64_t> fill(eptr.begin(), eptr.end() - 1);
            for (int64_t f = 0; f < nf; ++f)
                for (int c = 0; c < 3; ++c) {
                    const int32_t a = F[3 * f + c], b = F[3 * f + (c + 1) % 3];
                    eb[fill[std::min(a, b)]++] = std::max(a, b);
                }
        }
        double sum = 0.0;
        int64_t cnt = 0;
        std::vector<int32_t> bverts;
        for (int64_t a = 0; a < nv; ++a) {
            int32_t* lo = eb.data() + eptr[a];
            int32_t* hi = eb.data() + eptr[a + 1];
            for (int32_t* p = lo + 1; p < hi; ++p)  // insertion sort: a handful of entries
                for (int32_t* q = p; q > lo && q[-1] > q[0]; --q) std::swap(q[-1], q[0]);
            for (int32_t* p = lo; p < hi;) {
                int32_t* r = p;
                while (r < hi && *r == *p) ++r;
                const int64_t b = *p;
                double d[3] = {V[3 * b] - V[3 * a], V[3 * b + 1] - V[3 * a + 1], V[3 * b + 2] - V[3 * a + 2]};
                sum += norm3(d);
                ++cnt;
                if (r - p == 1) { bverts.push_back((int32_t)a); bverts.push_back((int32_t)b); }  // free edge
                p = r;
            }
        }
        m.mean_edge = sum / (double)cnt;
        std::sort(bverts.begin(), bverts.end());
        bverts.erase(std::unique(bverts.begin(), bverts.end()), bverts.end());
        m.boundary = bverts;
    }

    // Face max edge, bucket width and health length (lean_geometry.py:99-114, core_analysis.py:705, 913-957).
    std::vector<double> Lmax(nf);
    m.lean_area.resize(nf); m.g11.resize(nf); m.g12.resize(nf); m.g22.resize(nf);
    m.grad_area.resize(nf); m.gb.resize(9 * nf);
    std::vector<double> ca_area(nf);
    for (int64_t f = 0; f < nf; ++f) {
        const double* p0 = V + 3 * (int64_t)F[3 * f];
        const double* p1 = V + 3 * (int64_t)F[3 * f + 1];
        const double* p2 = V + 3 * (int64_t)F[3 * f + 2];
        double e01[3], e12[3], e20[3], e02[3];
        for (int k = 0; k < 3; ++k) {
            e01[k] = p1[k] - p0[k]; e12[k] = p2[k] - p1[k]; e20[k] = p0[k] - p2[k]; e02[k] = p2[k] - p0[k];
        }
        double l01 = norm3(e01), l12 = norm3(e12), l20 = norm3(e20);
        Lmax[f] = std::max(std::max(l01, l12), l20);
        // core_analysis.py:929-955 face area with a scale-aware degeneracy threshold
        double nrm[3];
        cross3(e01, e02, nrm);
        double nn = norm3(nrm);
        double tiny = 2.220446049250313e-16 * (Lmax[f] * Lmax[f]) * 10.0;
        ca_area[f] = nn < tiny ? 0.0 : 0.5 * nn;
        // lean_geometry.py:44-63 inverse Gram metric
        double a11 = einsum_dot3(e01, e01), a22 = einsum_dot3(e02, e02), a12 = einsum_dot3(e01, e02);
        double det = a11 * a22 - a12 * a12;
        m.lean_area[f] = 0.5 * std::sqrt(det > 0.0 ? det : 0.0);
        double inv = det > 0.0 ? 1.0 / det : 0.0;
        m.g11[f] = a22 * inv; m.g12[f] = -a12 * inv; m.g22[f] = a11 * inv;
        // fastcw_lean.py:375-391 hat-function gradients
        if (!(nn > 0.0)) { err = "Zero-area faces must be removed before building the heat engine."; return 1; }
        double area = 0.5 * nn;
        double un[3] = {nrm[0] / nn, nrm[1] / nn, nrm[2] / nn};
        double inv2a = 1.0 / (2.0 * area);
        double c1[3], c2[3];
        cross3(e02, un, c1);
        cross3(un, e01, c2);
        double* g = &m.gb[9 * f];
        for (int k = 0; k < 3; ++k) { g[3 + k] = c1[k] * inv2a; g[6 + k] = c2[k] * inv2a; }
        for (int k = 0; k < 3; ++k) g[k] = -g[3 + k] - g[6 + k];
        m.grad_area[f] = area;
    }
    m.bin_width = np_quantile(Lmax, 0.999) * 1.05;
    m.health_h = np_median(Lmax);

    // Barycentric vertex areas, face by face (core_analysis.py:959-978).
    m.vertex_area.assign(nv, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
        double c = ca_area[f] / 3.0;
        for (int k = 0; k < 3; ++k) m.vertex_area[F[3 * f + k]] += c;
    }
    m.total_area = 0.0;
    for (int64_t v = 0; v < nv; ++v) m.total_area += m.vertex_area[v];

    // Lumped mass, corner by corner (fastcw_lean.py:410-412).
    m.mass.assign(nv, 0.0);
    for (int c = 0; c < 3; ++c)
        for (int64_t f = 0; f < nf; ++f) m.mass[F[3 * f + c]] += m.grad_area[f] / 3.0;

    // Stiffness L = G^T diag(A) G as full symmetric CSC; duplicates summed in the
    // order the reference concatenates its triplets (block (i,j), then face): the
    // triplet (i, j, f) lands in column F[f][j], row F[f][i], at position
    // (3i + j) nf + f of the reference's list. Column by column from the vertex's
    // incident faces, entries sorted by (row, that position), so each row's
    // duplicates add in the reference's order.
    {
        std::vector<int64_t> vptr(nv + 1, 0);
        for (int64_t q = 0; q < 3 * nf; ++q) vptr[F[q] + 1]++;
        for (int64_t v = 0; v < nv; ++v) vptr[v + 1] += vptr[v];
        std::vector<int64_t> vface(3 * nf);
        {
            std::vector<int64_t> fill(vptr.begin(), vptr.end() - 1);
            for (int64_t q = 0; q < 3 * nf; ++q) vface[fill[F[q]]++] = q;  // q = 3 f + corner, ascending f
        }
        struct Entry {
            int32_t row;
            int64_t pos;
            double val;
        };
        std::vector<Entry> ent;
        m.Lp.assign(nv + 1, 0);
        m.Li.clear(); m.Lx.clear();
        m.Li.reserve(7 * nv); m.Lx.reserve(7 * nv);
        for (int64_t c = 0; c < nv; ++c) {
            ent.clear();
            for (int64_t t = vptr[c]; t < vptr[c + 1]; ++t) {
                const int64_t f = vface[t] / 3;
                const int j = (int)(vface[t] - 3 * f);
                const double* g = &m.gb[9 * f];
                for (int i = 0; i < 3; ++i)
                    ent.push_back({F[3 * f + i], (int64_t)(3 * i + j) * nf + f,
                                   m.grad_area[f] * einsum_dot3(g + 3 * i, g + 3 * j)});
            }
            // (row, pos) keys are distinct, so this insertion sort (a few dozen entries) gives
            // the one sorted order
            for (size_t k = 1; k < ent.size(); ++k)
                for (size_t q = k; q > 0 && (ent[q - 1].row != ent[q].row ? ent[q - 1].row > ent[q].row
                                                                         : ent[q - 1].pos > ent[q].pos); --q)
                    std::swap(ent[q - 1], ent[q]);
            for (size_t k = 0; k < ent.size();) {
                size_t l = k;
                double sum = 0.0;
                while (l < ent.size() && ent[l].row == ent[k].row) { sum += ent[l].val; ++l; }
                m.Li.push_back(ent[k].row);
                m.Lx.push_back(sum);
                k = l;
            }
            m.Lp[c + 1] = (int64_t)m.Li.size();
        }
    }
    return 0;
}

}  // namespace fcw
