// Symbolic sparse Cholesky analysis on the host.
//
// Ordering: geometric nested dissection. Each set of vertices is split at the
// median of its projection on one of eight directions (its coordinates'
// principal axis, two directions orthogonal to it and their mixes), the one
// whose smaller one-sided boundary between the halves is smallest; that boundary
// becomes the vertex separator, numbered after both halves. Sets of at most `leaf_size` vertices are leaves.
// The halves of the top three splits are dissected on their own threads; the order is the serial one.
// The elimination tree is then postordered (same fill, contiguous subtrees),
// and columns are grouped into supernodes:
//   * relaxed supernodes: every maximal subtree of at most `relax` columns
//     becomes one supernode with a dense diagonal block;
//   * fundamental supernodes elsewhere: chains j -> j+1 with a single child and
//     colcount(j) = colcount(j+1) + 1, cut every `max_width` columns.
// For every supernode we record its row structure, the extend-add map into
// its parent, per-row segments for the forward pull, the supernodal etree
// levels, and where each lower entry of A lands in the panel storage.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <memory>
#include <numeric>
#include <system_error>
#include <thread>

#include "fcw_internal.h"

namespace fcw {

namespace {

struct Graph {
    int64_t n = 0;
    std::vector<int64_t> xadj;
    std::vector<int32_t> adj;  // no self loops
};

Graph pattern_graph(const MeshPrep& m) {
    Graph g;
    g.n = m.nv;
    g.xadj.assign(m.nv + 1, 0);
    for (int64_t c = 0; c < m.nv; ++c)
        for (int64_t k = m.Lp[c]; k < m.Lp[c + 1]; ++k)
            if (m.Li[k] != c) g.xadj[c + 1]++;
    for (int64_t c = 0; c < m.nv; ++c) g.xadj[c + 1] += g.xadj[c];
    g.adj.resize(g.xadj[m.nv]);
    std::vector<int64_t> fill(g.xadj.begin(), g.xadj.end() - 1);
    for (int64_t c = 0; c < m.nv; ++c)
        for (int64_t k = m.Lp[c]; k < m.Lp[c + 1]; ++k)
            if (m.Li[k] != c) g.adj[fill[c]++] = m.Li[k];
    return g;
}

void principal_axis(const double* X, const int32_t* v, int64_t n, double c[3], double axis[3]) {
    c[0] = c[1] = c[2] = 0.0;
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) c[k] += X[3 * (int64_t)v[i] + k];
    for (int k = 0; k < 3; ++k) c[k] /= (double)n;
    double C[3][3] = {{0}};
    for (int64_t i = 0; i < n; ++i) {
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = X[3 * (int64_t)v[i] + k] - c[k];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) C[a][b] += d[a] * d[b];
    }
    // start from the longest bounding-box axis, then power iteration
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            double x = X[3 * (int64_t)v[i] + k];
            lo[k] = std::min(lo[k], x);
            hi[k] = std::max(hi[k], x);
        }
    int best = 0;
    for (int k = 1; k < 3; ++k)
        if (hi[k] - lo[k] > hi[best] - lo[best]) best = k;
    double a[3] = {0, 0, 0};
    a[best] = 1.0;
    a[(best + 1) % 3] = 1e-3;  // break symmetric ties deterministically
    for (int it = 0; it < 60; ++it) {
        double b[3];
        for (int r = 0; r < 3; ++r) b[r] = C[r][0] * a[0] + C[r][1] * a[1] + C[r][2] * a[2];
        double nb = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        if (!(nb > 0.0)) break;
        for (int r = 0; r < 3; ++r) a[r] = b[r] / nb;
    }
    double na = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int r = 0; r < 3; ++r) axis[r] = a[r] / na;
}

constexpr int kCandidates = 8;

// The principal axis a, two unit directions orthogonal to it (p, q), and the mixes
// (a +- p)/sqrt2, (a +- q)/sqrt2, (p +- q)/sqrt2 (the last pair only if room): 8 directions.
void candidate_axes(const double a[3], double dirs[kCandidates][3]) {
    double p[3];
    // a vector not parallel to a, made orthogonal to it
    const double e[3] = {std::fabs(a[0]) < 0.9 ? 1.0 : 0.0, std::fabs(a[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    const double d = e[0] * a[0] + e[1] * a[1] + e[2] * a[2];
    for (int k = 0; k < 3; ++k) p[k] = e[k] - d * a[k];
    double np_ = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    for (int k = 0; k < 3; ++k) p[k] /= np_;
    const double q[3] = {a[1] * p[2] - a[2] * p[1], a[2] * p[0] - a[0] * p[2], a[0] * p[1] - a[1] * p[0]};
    const double r = 1.0 / std::sqrt(2.0);
    for (int k = 0; k < 3; ++k) {
        dirs[0][k] = a[k];
        dirs[1][k] = p[k];
        dirs[2][k] = q[k];
        dirs[3][k] = (a[k] + p[k]) * r;
        dirs[4][k] = (a[k] - p[k]) * r;
        dirs[5][k] = (a[k] + q[k]) * r;
        dirs[6][k] = (a[k] - q[k]) * r;
        dirs[7][k] = (p[k] + q[k]) * r;
    }
}

// The two halves of a split are dissected on separate threads down to kParallelDepth
// (disjoint vertex sets and output ranges). Each call marks its vertex set with a fresh
// id; a neighbour's mark is read across the cut while another thread may rewrite it, so
// the marks are relaxed atomics. A foreign mark never equals the reader's fresh id, and
// side[] is read only for vertices of the reader's own set, so the order is the same as
// a serial run's.
constexpr int kParallelDepth = 3;
constexpr int64_t kParallelMin = 4096;  // smaller sets stay on the calling thread

struct Dissector {
    const Graph& g;
    const double* X;
    int leaf;
    std::unique_ptr<std::atomic<int32_t>[]> stamp;
    std::vector<int8_t> side;
    std::atomic<int32_t> next_id{1};

    Dissector(const Graph& g_, const double* X_, int leaf_)
        : g(g_), X(X_), leaf(leaf_), stamp(new std::atomic<int32_t>[g_.n]), side(g_.n, 0) {
        for (int64_t i = 0; i < g_.n; ++i) stamp[i].store(0, std::memory_order_relaxed);
    }
    bool member(int32_t y, int32_t id) const { return stamp[y].load(std::memory_order_relaxed) == id; }

    // Size of the smaller one-sided boundary of the median split of proj (-1 if one side is empty).
    int64_t separator_size(const int32_t* v, int64_t n, const std::vector<double>& proj, double med, int32_t id) {
        int64_t n0 = 0;
        for (int64_t i = 0; i < n; ++i) {
            side[v[i]] = proj[i] < med ? 0 : 1;
            n0 += side[v[i]] == 0;
        }
        if (n0 == 0 || n0 == n) return -1;
        int64_t s0 = 0, s1 = 0;
        for (int64_t i = 0; i < n; ++i) {
            const int32_t x = v[i];
            for (int64_t k = g.xadj[x]; k < g.xadj[x + 1]; ++k) {
                const int32_t y = g.adj[k];
                if (member(y, id) && side[y] != side[x]) {
                    (side[x] == 0 ? s0 : s1)++;
                    break;
                }
            }
        }
        return std::min(s0, s1);
    }

    // Writes an elimination order of v[0..n) into out[0..n).
    void dissect(const int32_t* v, int64_t n, int32_t* out, int depth = 0) {
        if (n <= leaf) {
            std::copy(v, v + n, out);
            return;
        }
        const int32_t id = next_id.fetch_add(1, std::memory_order_relaxed);
        for (int64_t i = 0; i < n; ++i) stamp[v[i]].store(id, std::memory_order_relaxed);
        double c[3], ax[3];
        principal_axis(X, v, n, c, ax);
        // candidate cut directions: the principal axis, two directions orthogonal to it, and
        // their half-way mixes; each is split at its median and the smallest separator wins
        double dirs[kCandidates][3];
        candidate_axes(ax, dirs);
        std::vector<double> proj(n), tmp(n);
        int64_t best_size = -1;
        int best_dir = 0;
        double best_med = 0.0;
        for (int d = 0; d < kCandidates; ++d) {
            const double* a = dirs[d];
            for (int64_t i = 0; i < n; ++i) {
                const double* x = X + 3 * (int64_t)v[i];
                proj[i] = (x[0] - c[0]) * a[0] + (x[1] - c[1]) * a[1] + (x[2] - c[2]) * a[2];
            }
            tmp = proj;
            std::nth_element(tmp.begin(), tmp.begin() + n / 2, tmp.end());
            const double med = tmp[n / 2];
            const int64_t sz = separator_size(v, n, proj, med, id);
            if (sz >= 0 && (best_size < 0 || sz < best_size)) {
                best_size = sz;
                best_dir = d;
                best_med = med;
            }
        }
        if (best_size < 0) {
            std::copy(v, v + n, out);
            return;
        }
        for (int64_t i = 0; i < n; ++i) {
            const double* x = X + 3 * (int64_t)v[i];
            const double* a = dirs[best_dir];
            proj[i] = (x[0] - c[0]) * a[0] + (x[1] - c[1]) * a[1] + (x[2] - c[2]) * a[2];
        }
        const double med = best_med;
        int64_t n0 = 0;
        for (int64_t i = 0; i < n; ++i) {
            side[v[i]] = proj[i] < med ? 0 : 1;
            n0 += side[v[i]] == 0;
        }
        std::vector<int32_t> b0, b1;
        for (int64_t i = 0; i < n; ++i) {
            int32_t x = v[i];
            for (int64_t k = g.xadj[x]; k < g.xadj[x + 1]; ++k) {
                int32_t y = g.adj[k];
                if (member(y, id) && side[y] != side[x]) {
                    (side[x] == 0 ? b0 : b1).push_back(x);
                    break;
                }
            }
        }
        const std::vector<int32_t>& sep = b0.size() <= b1.size() ? b0 : b1;
        for (int32_t x : sep) side[x] = 2;
        std::vector<int32_t> A, B;
        A.reserve(n0);
        B.reserve(n - n0);
        for (int64_t i = 0; i < n; ++i) {
            if (side[v[i]] == 0) A.push_back(v[i]);
            else if (side[v[i]] == 1) B.push_back(v[i]);
        }
        std::vector<int32_t> S(sep);
        std::thread t;
        if (depth < kParallelDepth && (int64_t)std::min(A.size(), B.size()) >= kParallelMin) {
            try {
                t = std::thread([&] { dissect(A.data(), (int64_t)A.size(), out, depth + 1); });
            } catch (const std::system_error&) {  // no thread to be had: stay serial
            }
        }
        if (t.joinable()) {
            dissect(B.data(), (int64_t)B.size(), out + A.size(), depth + 1);
            t.join();
        } else {
            dissect(A.data(), (int64_t)A.size(), out, depth + 1);
            dissect(B.data(), (int64_t)B.size(), out + A.size(), depth + 1);
        }
        std::copy(S.begin(), S.end(), out + A.size() + B.size());
    }
};

// Elimination tree of the symmetric pattern in the order given by perm (Liu).
std::vector<int32_t> etree(const Graph& g, const std::vector<int32_t>& perm, const std::vector<int32_t>& iperm) {
    const int64_t n = g.n;
    std::vector<int32_t> parent(n, -1), anc(n, -1);
    for (int64_t j = 0; j < n; ++j) {
        int32_t old = perm[j];
        for (int64_t k = g.xadj[old]; k < g.xadj[old + 1]; ++k) {
            int32_t i = iperm[g.adj[k]];
            if (i >= j) continue;
            int32_t r = i;
            while (anc[r] != -1 && anc[r] != j) {
                int32_t t = anc[r];
                anc[r] = (int32_t)j;
                r = t;
            }
            if (anc[r] == -1) {
                anc[r] = (int32_t)j;
                parent[r] = (int32_t)j;
            }
        }
    }
    return parent;
}

}  // namespace

int build_symbolic(const MeshPrep& m, int leaf_size, int max_width, int relax, Symbolic& S, std::string& err) {
    const int64_t n = m.nv;
    if (leaf_size < 1 || max_width < 1 || max_width > 1024 || relax < 1 || relax > max_width) {
        err = "invalid symbolic parameters";
        return 1;
    }
    Graph g = pattern_graph(m);

    // 1. nested dissection
    std::vector<int32_t> all(n), nd(n);
    std::iota(all.begin(), all.end(), 0);
    Dissector dis(g, m.V.data(), leaf_size);
    dis.dissect(all.data(), n, nd.data());
    std::vector<int32_t> inv(n);
    for (int64_t i = 0; i < n; ++i) inv[nd[i]] = (int32_t)i;

    // 2. etree + postorder
    std::vector<int32_t> par = etree(g, nd, inv);
    std::vector<int32_t> head(n, -1), next(n, -1);
    for (int64_t j = n - 1; j >= 0; --j)
        if (par[j] != -1) { next[j] = head[par[j]]; head[par[j]] = (int32_t)j; }
    std::vector<int32_t> post(n), stack;
    int64_t k = 0;
    for (int64_t r = 0; r < n; ++r) {
        if (par[r] != -1) continue;
        stack.push_back((int32_t)r);
        while (!stack.empty()) {
            int32_t p = stack.back();
            int32_t c = head[p];
            if (c == -1) {
                stack.pop_back();
                post[p] = (int32_t)k++;
            } else {
                head[p] = next[c];
                stack.push_back(c);
            }
        }
    }
    S.n = n;
    S.perm.assign(n, 0);
    S.iperm.assign(n, 0);
    for (int64_t j = 0; j < n; ++j) S.perm[post[j]] = nd[j];
    for (int64_t j = 0; j < n; ++j) S.iperm[S.perm[j]] = (int32_t)j;
    std::vector<int32_t> parent(n, -1);
    for (int64_t j = 0; j < n; ++j) parent[post[j]] = par[j] == -1 ? -1 : post[par[j]];

    // adjacency in elimination order, sorted
    std::vector<int64_t> nx(n + 1, 0);
    std::vector<int32_t> na(g.adj.size());
    for (int64_t j = 0; j < n; ++j) nx[j + 1] = nx[j] + (g.xadj[S.perm[j] + 1] - g.xadj[S.perm[j]]);
    for (int64_t j = 0; j < n; ++j) {
        int32_t old = S.perm[j];
        int64_t o = nx[j];
        for (int64_t q = g.xadj[old]; q < g.xadj[old + 1]; ++q) na[o++] = S.iperm[g.adj[q]];
        std::sort(na.begin() + nx[j], na.begin() + nx[j + 1]);
    }

    // 3. column counts (row-subtree traversal)
    std::vector<int64_t> colcount(n, 1);
    {
        std::vector<int32_t> mark(n, -1);
        for (int64_t i = 0; i < n; ++i) {
            mark[i] = (int32_t)i;
            for (int64_t q = nx[i]; q < nx[i + 1]; ++q) {
                int32_t j = na[q];
                if (j >= i) break;
                while (mark[j] != i) {
                    colcount[j]++;
                    mark[j] = (int32_t)i;
                    j = parent[j];
                }
            }
        }
    }
    std::vector<int32_t> nchild(n, 0), desc(n, 0);
    for (int64_t j = 0; j < n; ++j)
        if (parent[j] != -1) { nchild[parent[j]]++; desc[parent[j]] += desc[j] + 1; }

    // 4. supernodes
    const int R = relax;
    std::vector<int8_t> in_relax(n, 0);
    std::vector<int32_t> relax_start(n, -1);
    for (int64_t r = 0; r < n; ++r) {
        bool small = desc[r] + 1 <= R;
        bool top = parent[r] == -1 || desc[parent[r]] + 1 > R;
        if (small && top) {
            int64_t s0 = r - desc[r];
            for (int64_t j = s0; j <= r; ++j) { in_relax[j] = 1; relax_start[j] = (int32_t)s0; }
        }
    }
    S.sn_c0.clear();
    S.col_sn.assign(n, -1);
    {
        int64_t j = 0;
        bool open_fund = false;
        while (j < n) {
            if (in_relax[j]) {
                int64_t s0 = j, e = j;
                while (e + 1 < n && in_relax[e + 1] && relax_start[e + 1] == s0) ++e;
                S.sn_c0.push_back((int32_t)s0);
                for (int64_t q = s0; q <= e; ++q) S.col_sn[q] = (int32_t)S.sn_c0.size() - 1;
                j = e + 1;
                open_fund = false;
                continue;
            }
            bool merge = open_fund && parent[j - 1] == j && nchild[j] == 1 && colcount[j - 1] == colcount[j] + 1 &&
                         (j - S.sn_c0.back()) < max_width;
            if (!merge) S.sn_c0.push_back((int32_t)j);
            S.col_sn[j] = (int32_t)S.sn_c0.size() - 1;
            open_fund = true;
            ++j;
        }
    }
    // 4b. amalgamation: merge a supernode into its parent when their columns are
    // contiguous and the explicit zeros stay moderate (fewer, wider supernodes and
    // fewer etree levels: on the order-7 mesh 27% more stored entries buy 2.4x fewer
    // supernodes, and the solves run faster on the wider tiles). For a supernode whose columns form an etree chain or
    // subtree, its row structure beyond its last column l has colcount[l]-1 rows.
    {
        const int32_t n0 = (int32_t)S.sn_c0.size();
        std::vector<int32_t> first(S.sn_c0.begin(), S.sn_c0.end());
        std::vector<int32_t> last(n0);
        for (int32_t s = 0; s < n0; ++s) last[s] = (s + 1 < n0 ? S.sn_c0[s + 1] : (int32_t)n) - 1;
        std::vector<double> truenz(n0, 0.0);
        for (int32_t s = 0; s < n0; ++s)
            for (int32_t j = first[s]; j <= last[s]; ++j) truenz[s] += (double)colcount[j];
        std::vector<int32_t> into(n0, -1);
        auto find = [&](int32_t s) {
            while (into[s] != -1) s = into[s];
            return s;
        };
        for (int pass = 0; pass < 8; ++pass) {
            bool changed = false;
            for (int32_t s = 0; s < n0; ++s) {
                if (into[s] != -1) continue;
                const int32_t pc = parent[last[s]];
                if (pc == -1) continue;
                const int32_t p = find(S.col_sn[pc]);
                if (last[s] + 1 != first[p]) continue;
                const double nsm = (double)(last[p] - first[s] + 1);
                if (nsm > max_width) continue;
                const double nrp = (double)(colcount[last[p]] - 1);
                const double stored = nsm * (nsm + 1.0) / 2.0 + nsm * nrp;
                const double zf = 1.0 - (truenz[s] + truenz[p]) / stored;
                const bool ok = nsm <= 16 || (nsm <= 32 && zf < 0.8) || (nsm <= 64 && zf < 0.4);
                if (!ok) continue;
                first[p] = first[s];
                truenz[p] += truenz[s];
                into[s] = p;
                changed = true;
            }
            if (!changed) break;
        }
        std::vector<int32_t> c0;
        for (int32_t s = 0; s < n0; ++s)
            if (into[s] == -1) c0.push_back(first[s]);
        std::sort(c0.begin(), c0.end());
        S.sn_c0 = c0;
        for (size_t s = 0; s < c0.size(); ++s) {
            const int32_t e = s + 1 < c0.size() ? c0[s + 1] : (int32_t)n;
            for (int32_t j = c0[s]; j < e; ++j) S.col_sn[j] = (int32_t)s;
        }
    }
    const int32_t ns_total = (int32_t)S.sn_c0.size();
    S.nsuper = ns_total;
    S.sn_c0.push_back((int32_t)n);
    S.sn_parent.assign(ns_total, -1);
    for (int32_t s = 0; s < ns_total; ++s) {
        int32_t l = S.sn_c0[s + 1] - 1;
        S.sn_parent[s] = parent[l] == -1 ? -1 : S.col_sn[parent[l]];
    }
    S.child_ptr.assign(ns_total + 1, 0);
    for (int32_t s = 0; s < ns_total; ++s)
        if (S.sn_parent[s] != -1) S.child_ptr[S.sn_parent[s] + 1]++;
    for (int32_t s = 0; s < ns_total; ++s) S.child_ptr[s + 1] += S.child_ptr[s];
    S.child_list.assign(S.child_ptr[ns_total], 0);
    {
        std::vector<int32_t> f(S.child_ptr.begin(), S.child_ptr.end() - 1);
        for (int32_t s = 0; s < ns_total; ++s)
            if (S.sn_parent[s] != -1) S.child_list[f[S.sn_parent[s]]++] = s;
    }

    // 5. row structures
    std::vector<std::vector<int32_t>> st(ns_total);
    {
        std::vector<int32_t> mark(n, -1);
        for (int32_t s = 0; s < ns_total; ++s) {
            int32_t f0 = S.sn_c0[s], l = S.sn_c0[s + 1] - 1;
            auto& lst = st[s];
            for (int32_t j = f0; j <= l; ++j)
                for (int64_t q = nx[j]; q < nx[j + 1]; ++q) {
                    int32_t i = na[q];
                    if (i > l && mark[i] != s) { mark[i] = s; lst.push_back(i); }
                }
            for (int32_t q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q)
                for (int32_t i : st[S.child_list[q]])
                    if (i > l && mark[i] != s) { mark[i] = s; lst.push_back(i); }
            std::sort(lst.begin(), lst.end());
        }
    }
    S.sn_m.assign(ns_total, 0);
    S.sn_rowptr.assign(ns_total + 1, 0);
    S.sn_valptr.assign(ns_total + 1, 0);
    S.sn_invptr.assign(ns_total + 1, 0);
    S.sn_updptr.assign(ns_total + 1, 0);
    S.max_ns = S.max_m = 0;
    S.nnz_l = 0;
    S.flops_factor = 0.0;
    for (int32_t s = 0; s < ns_total; ++s) {
        int64_t ns = S.sn_c0[s + 1] - S.sn_c0[s], nr = (int64_t)st[s].size(), mm = ns + nr;
        S.sn_m[s] = (int32_t)mm;
        S.sn_rowptr[s + 1] = S.sn_rowptr[s] + mm;
        S.sn_valptr[s + 1] = S.sn_valptr[s] + mm * ns;
        S.sn_invptr[s + 1] = S.sn_invptr[s] + ns * ns;
        S.sn_updptr[s + 1] = S.sn_updptr[s] + nr * nr;
        S.max_ns = std::max<int32_t>(S.max_ns, (int32_t)ns);
        S.max_m = std::max<int32_t>(S.max_m, (int32_t)mm);
        S.nnz_l += mm * ns - ns * (ns - 1) / 2;
        S.flops_factor += (double)ns * ns * ns / 3.0 + (double)ns * ns * nr + (double)nr * nr * ns;
    }
    S.nnz_factor = S.sn_valptr[ns_total];
    S.n_inv = S.sn_invptr[ns_total];
    S.n_upd = S.sn_updptr[ns_total];
    S.rows.assign(S.sn_rowptr[ns_total], 0);
    for (int32_t s = 0; s < ns_total; ++s) {
        int64_t o = S.sn_rowptr[s];
        for (int32_t j = S.sn_c0[s]; j < S.sn_c0[s + 1]; ++j) S.rows[o++] = j;
        for (int32_t i : st[s]) S.rows[o++] = i;
    }
    auto find_pos = [&](int32_t s, int32_t row) -> int64_t {
        int32_t c0 = S.sn_c0[s], ns = S.sn_c0[s + 1] - c0;
        if (row >= c0 && row < c0 + ns) return row - c0;
        const int32_t* b = S.rows.data() + S.sn_rowptr[s] + ns;
        const int32_t* e = S.rows.data() + S.sn_rowptr[s + 1];
        const int32_t* it = std::lower_bound(b, e, row);
        if (it == e || *it != row) return -1;
        return ns + (it - b);
    };
    // extend-add map into the parent
    S.relind.assign(S.rows.size(), -1);
    for (int32_t s = 0; s < ns_total; ++s) {
        int32_t p = S.sn_parent[s];
        int32_t ns = S.sn_c0[s + 1] - S.sn_c0[s];
        for (int64_t q = S.sn_rowptr[s] + ns; q < S.sn_rowptr[s + 1]; ++q) {
            if (p == -1) { err = "symbolic: root supernode has off-diagonal rows"; return 1; }
            int64_t pos = find_pos(p, S.rows[q]);
            if (pos < 0) { err = "symbolic: child structure not contained in parent"; return 1; }
            S.relind[q] = (int32_t)pos;
        }
    }
    // levels (height in the supernodal etree)
    S.sn_level.assign(ns_total, 0);
    for (int32_t s = 0; s < ns_total; ++s)
        if (S.sn_parent[s] != -1)
            S.sn_level[S.sn_parent[s]] = std::max(S.sn_level[S.sn_parent[s]], S.sn_level[s] + 1);
    S.nlevels = 0;
    for (int32_t s = 0; s < ns_total; ++s) S.nlevels = std::max(S.nlevels, S.sn_level[s] + 1);
    S.level_ptr.assign(S.nlevels + 1, 0);
    for (int32_t s = 0; s < ns_total; ++s) S.level_ptr[S.sn_level[s] + 1]++;
    for (int32_t l = 0; l < S.nlevels; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
    S.level_nodes.assign(ns_total, 0);
    {
        std::vector<int32_t> f(S.level_ptr.begin(), S.level_ptr.end() - 1);
        for (int32_t s = 0; s < ns_total; ++s) S.level_nodes[f[S.sn_level[s]]++] = s;
    }
    // forward-pull segments: for each row, the (supernode, position) pairs that update it
    S.seg_ptr.assign(n + 1, 0);
    for (int32_t s = 0; s < ns_total; ++s) {
        int32_t ns = S.sn_c0[s + 1] - S.sn_c0[s];
        for (int64_t q = S.sn_rowptr[s] + ns; q < S.sn_rowptr[s + 1]; ++q) S.seg_ptr[S.rows[q] + 1]++;
    }
    for (int64_t i = 0; i < n; ++i) S.seg_ptr[i + 1] += S.seg_ptr[i];
    S.seg_sn.assign(S.seg_ptr[n], 0);
    S.seg_pos.assign(S.seg_ptr[n], 0);
    {
        std::vector<int64_t> f(S.seg_ptr.begin(), S.seg_ptr.end() - 1);
        for (int32_t s = 0; s < ns_total; ++s) {
            int32_t ns = S.sn_c0[s + 1] - S.sn_c0[s];
            for (int64_t q = S.sn_rowptr[s] + ns; q < S.sn_rowptr[s + 1]; ++q) {
                int32_t row = S.rows[q];
                S.seg_sn[f[row]] = s;
                S.seg_pos[f[row]] = (int32_t)(q - S.sn_rowptr[s]);
                f[row]++;
            }
        }
    }
    // where each lower entry of A lands (A's pattern = L's pattern incl. diagonal)
    S.a_dst.clear();
    S.a_src.clear();
    S.a_col.clear();
    for (int64_t b = 0; b < n; ++b) {
        for (int64_t q = m.Lp[b]; q < m.Lp[b + 1]; ++q) {
            int32_t a = m.Li[q];
            int32_t i = S.iperm[a], j = S.iperm[b];
            if (i < j) continue;
            int32_t s = S.col_sn[j];
            int64_t pos = find_pos(s, i);
            if (pos < 0) { err = "symbolic: entry of A outside the factor structure"; return 1; }
            int32_t ns = S.sn_c0[s + 1] - S.sn_c0[s];
            S.a_dst.push_back(S.sn_valptr[s] + pos * ns + (j - S.sn_c0[s]));
            S.a_src.push_back(q);
            S.a_col.push_back((int32_t)b);
        }
    }
    S.nnz_lower_a = (int64_t)S.a_dst.size();
    return 0;
}

}  // namespace fcw
