// Per-source kernels: shift + transpose, then all per-source metrics.
//
// After the Poisson solve the fields sit in an n x K vertex-major block. The
// shift kernel subtracts each column's value at its source and transposes to
// K x n (one contiguous field per source). k_source_metrics then computes, one
// CTA per source, the health screen, MSD, distance to boundary, and the
// radius/perimeter geometry of lean_geometry.py restricted to the faces near
// the source (see its comment for why that restriction is exact).
#include <math.h>

#include "kernels.cuh"

namespace fcw {

namespace {

template <typename Tin, typename Tout>
__global__ void k_shift_transpose(int32_t n, int32_t K, const Tin* __restrict__ phi, const int32_t* __restrict__ src,
                                  Tout* __restrict__ dT) {
    __shared__ Tin tile[32][33];
    __shared__ Tin sh[32];
    const int v0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    if (ty == 0) {
        const int s = src[k0 + tx];
        sh[tx] = s >= 0 ? phi[(int64_t)s * K + k0 + tx] : Tin(0);
    }
    for (int r = ty; r < 32; r += 8) {
        const int v = v0 + r;
        tile[r][tx] = v < n ? phi[(int64_t)v * K + k0 + tx] : Tin(0);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int v = v0 + tx;
        if (v < n) dT[(int64_t)(k0 + r) * n + v] = (Tout)(tile[tx][r] - sh[r]);
    }
}


__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

// Per-(vertex tile, source) partial statistics written by k_shift_stats.
enum { P_SUM_D, P_SUM_DA, P_SUM_A, P_CNT, P_NEG, P_VIOL, P_NONFINITE, P_DMAX, P_N };

// One vertex's share of the health screen and MSD sums (lean_geometry.py:343-357,
// core_analysis.py:1573-1581) for the distance di at a vertex (vx, vy, vz) of area va from
// a source at (sx, sy, sz): counts of non-finite values, of d < -h and of d < 0.9 |x - x_s| - h,
// the valid-distance sums and the maximum. The chord test compares squares and takes the
// reference's sqrt form only within a 1e-10 band of the threshold, so the counts match the
// reference exactly. Returns whether the vertex is nearer than R0.
__device__ __forceinline__ bool vertex_stats(double di, double vx, double vy, double vz, double va, double sx,
                                             double sy, double sz, double h, double eps, double R0, double& sd,
                                             double& sda, double& sa, double& dm, int& cnt, int& ng, int& vi,
                                             int& nf) {
    if (!isfinite(di)) {
        ++nf;
        return false;
    }
    if (di < -h) ++ng;
    const double dx = vx - sx, dy = vy - sy, dz = vz - sz;
    const double c2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
    const double t = di + h;
    bool viol;
    if (t < 0.0) {
        viol = true;
    } else {
        const double lhs = t * t, rhs = 0.81 * c2;
        if (lhs < rhs * (1.0 - 1e-10)) viol = true;
        else if (lhs > rhs * (1.0 + 1e-10)) viol = false;
        else viol = di < __dsub_rn(dmul(0.9, __dsqrt_rn(c2)), h);
    }
    if (viol) ++vi;
    if (di > eps) {
        sd += di;
        sda += di * va;
        sa += va;
        ++cnt;
    }
    dm = fmax(dm, di);
    return di < R0;
}

// The shift + transpose of one kStatVTile-vertex x 32-source tile, fused with the per-vertex
// work of the health screen and MSD (lean_geometry.py:343-357, core_analysis.py:1573-1581):
// counts of d < -h and of d < 0.9 |x - x_s| - h, the valid-distance sums and the maximum.
// The chord test compares squares and takes the reference's sqrt form only within a
// 1e-10 band of the threshold, so the counts match the reference exactly. Vertices
// closer than the near radius are appended to their source's near list: per tile and
// source, one atomic reserves the run, written in vertex order (which keeps the
// per-source kernel's near-vertex walk local).
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256, 3) k_shift_stats(MetricArgs a, int32_t K, const Tin* __restrict__ phi,
                                                     Tout* __restrict__ dT) {
    __shared__ Tin tile[32][33];
    __shared__ Tin sh[32];
    __shared__ double sc[32][3];
    __shared__ int srcv[32];
    __shared__ unsigned nearmask[32][kStatVTile / 32];  // per source and sub-tile: lanes (vertices) near it
    const int n = a.n;
    const int k0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int vbase = blockIdx.x * kStatVTile;
    for (int q = ty; q < kStatVTile / 32; q += 8) nearmask[tx][q] = 0u;
    if (ty == 0) {
        const int sidx = a.src[k0 + tx];
        srcv[tx] = sidx;
        sh[tx] = sidx >= 0 ? phi[(int64_t)sidx * K + k0 + tx] : Tin(0);
        for (int c = 0; c < 3; ++c) sc[tx][c] = sidx >= 0 ? a.coords[3 * (int64_t)sidx + c] : 0.0;
    }
    double sd[4], sda[4], sa[4], dm[4];
    int cnt[4], ng[4], vi[4], nf[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) { sd[j] = sda[j] = sa[j] = 0.0; dm[j] = 0.0; cnt[j] = ng[j] = vi[j] = nf[j] = 0; }
    const double h = a.health_h, R0 = a.near_radius;
    const unsigned lanes_below = (1u << tx) - 1u;
    // the field values of the next 32-vertex sub-tile are loaded while this one is processed
    Tin nxt[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int v = vbase + ty + 8 * j;
        nxt[j] = v < n ? phi[(int64_t)v * K + k0 + tx] : Tin(0);
    }
    for (int sub = 0; sub < kStatVTile / 32; ++sub) {
        const int v0 = vbase + sub * 32;
        if (v0 >= n) break;
        __syncthreads();  // the previous sub-tile's reads of `tile` are done
#pragma unroll
        for (int j = 0; j < 4; ++j) tile[ty + 8 * j][tx] = nxt[j];
        if (sub + 1 < kStatVTile / 32) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int v = v0 + 32 + ty + 8 * j;
                nxt[j] = v < n ? phi[(int64_t)v * K + k0 + tx] : Tin(0);
            }
        }
        const int v = v0 + tx;
        const bool in = v < n;
        double vx = 0.0, vy = 0.0, vz = 0.0, va = 0.0;
        if (in) {
            vx = a.coords[3 * (int64_t)v];
            vy = a.coords[3 * (int64_t)v + 1];
            vz = a.coords[3 * (int64_t)v + 2];
            va = a.vertex_area[v];
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = ty + 8 * j, k = k0 + r;
            const Tout dv = (Tout)(tile[tx][r] - sh[r]);
            if (in) dT[(int64_t)k * n + v] = dv;
            if (srcv[r] < 0) continue;  // warp-uniform (one source per warp)
            const double di = (double)dv;
            const bool near = in && vertex_stats(di, vx, vy, vz, va, sc[r][0], sc[r][1], sc[r][2], h, a.eps, R0,
                                                 sd[j], sda[j], sa[j], dm[j], cnt[j], ng[j], vi[j], nf[j]);
            const unsigned mask = __ballot_sync(0xffffffffu, near);
            if (tx == 0) nearmask[r][sub] = mask;
        }
    }
    // reduce over the 32 vertices of each warp (lanes), one source per (warp, j)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        for (int off = 16; off > 0; off >>= 1) {
            sd[j] += __shfl_down_sync(0xffffffffu, sd[j], off);
            sda[j] += __shfl_down_sync(0xffffffffu, sda[j], off);
            sa[j] += __shfl_down_sync(0xffffffffu, sa[j], off);
            dm[j] = fmax(dm[j], __shfl_down_sync(0xffffffffu, dm[j], off));
            cnt[j] += __shfl_down_sync(0xffffffffu, cnt[j], off);
            ng[j] += __shfl_down_sync(0xffffffffu, ng[j], off);
            vi[j] += __shfl_down_sync(0xffffffffu, vi[j], off);
            nf[j] += __shfl_down_sync(0xffffffffu, nf[j], off);
        }
        if (tx == 0) {
            const int k = k0 + ty + 8 * j;
            double* q = a.partials + ((int64_t)blockIdx.x * K + k) * P_N;
            q[P_SUM_D] = sd[j]; q[P_SUM_DA] = sda[j]; q[P_SUM_A] = sa[j]; q[P_CNT] = (double)cnt[j];
            q[P_NEG] = (double)ng[j]; q[P_VIOL] = (double)vi[j]; q[P_NONFINITE] = (double)nf[j]; q[P_DMAX] = dm[j];
        }
    }
    // the tile's near vertices of each source, appended to its list with one atomic, in vertex order
    __syncthreads();
    constexpr int NS = kStatVTile / 32;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int r = ty + 8 * j, k = k0 + r;
        const unsigned m_l = tx < NS ? nearmask[r][tx] : 0u;
        int c = __popc(m_l), incl = c;
        for (int off = 1; off < NS; off <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, off);
            if (tx >= off) incl += t;
        }
        const int total = __shfl_sync(0xffffffffu, incl, NS - 1);
        if (total == 0) continue;  // warp-uniform
        int base = 0;
        if (tx == 0) base = atomicAdd(&a.near_count[k], total);
        base = __shfl_sync(0xffffffffu, base, 0);
        const int excl = incl - c;
#pragma unroll
        for (int sb = 0; sb < NS; ++sb) {
            const unsigned m = nearmask[r][sb];
            const int off = __shfl_sync(0xffffffffu, excl, sb);
            if (m & (1u << tx))
                a.near_list[(int64_t)k * n + base + off + __popc(m & lanes_below)] = vbase + sb * 32 + tx;
        }
    }
}

// One field (the single-source path): the same shift, statistics and near list for the one
// column of phi (n, elimination order) into d. A CTA takes kStatVTile vertices, a warp 32
// consecutive ones per step; the tile's near vertices are appended in vertex order with one
// atomic, as k_shift_stats appends them.
__global__ void __launch_bounds__(256) k_shift_stats_one(MetricArgs a, const double* __restrict__ phi,
                                                         double* __restrict__ d) {
    constexpr int NG = kStatVTile / 32;  // 32-vertex groups of a tile
    static_assert(NG == 32, "one lane per group in the near-list scan");
    __shared__ unsigned gmask[NG];
    __shared__ int gbase[NG];
    __shared__ double wred[8][4];
    __shared__ int wcnt[8][4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = a.n, vbase = blockIdx.x * kStatVTile;
    const int se = a.src[0];
    const double p0 = phi[se];
    const double sx = a.coords[3 * (int64_t)se], sy = a.coords[3 * (int64_t)se + 1], sz = a.coords[3 * (int64_t)se + 2];
    double sd = 0.0, sda = 0.0, sa = 0.0, dm = 0.0;
    int cnt = 0, ng = 0, vi = 0, nf = 0;
    for (int g = warp; g < NG; g += 8) {
        const int v = vbase + 32 * g + lane;
        bool near = false;
        if (v < n) {
            const double dv = phi[v] - p0;
            d[v] = dv;
            near = vertex_stats(dv, a.coords[3 * (int64_t)v], a.coords[3 * (int64_t)v + 1],
                                a.coords[3 * (int64_t)v + 2], a.vertex_area[v], sx, sy, sz, a.health_h, a.eps,
                                a.near_radius, sd, sda, sa, dm, cnt, ng, vi, nf);
        }
        const unsigned m = __ballot_sync(0xffffffffu, near);
        if (lane == 0) gmask[g] = m;
    }
    for (int off = 16; off > 0; off >>= 1) {
        sd += __shfl_down_sync(0xffffffffu, sd, off);
        sda += __shfl_down_sync(0xffffffffu, sda, off);
        sa += __shfl_down_sync(0xffffffffu, sa, off);
        dm = fmax(dm, __shfl_down_sync(0xffffffffu, dm, off));
        cnt += __shfl_down_sync(0xffffffffu, cnt, off);
        ng += __shfl_down_sync(0xffffffffu, ng, off);
        vi += __shfl_down_sync(0xffffffffu, vi, off);
        nf += __shfl_down_sync(0xffffffffu, nf, off);
    }
    if (lane == 0) {
        wred[warp][0] = sd; wred[warp][1] = sda; wred[warp][2] = sa; wred[warp][3] = dm;
        wcnt[warp][0] = cnt; wcnt[warp][1] = ng; wcnt[warp][2] = vi; wcnt[warp][3] = nf;
    }
    __syncthreads();
    if (warp == 0) {
        // the tile's partials, the warps' sums added in warp order
        if (lane == 0) {
            double q[P_N] = {0.0};
            for (int w = 0; w < 8; ++w) {
                q[P_SUM_D] += wred[w][0]; q[P_SUM_DA] += wred[w][1]; q[P_SUM_A] += wred[w][2];
                q[P_DMAX] = fmax(q[P_DMAX], wred[w][3]);
                q[P_CNT] += wcnt[w][0]; q[P_NEG] += wcnt[w][1]; q[P_VIOL] += wcnt[w][2]; q[P_NONFINITE] += wcnt[w][3];
            }
            double* o = a.partials + (int64_t)blockIdx.x * P_N;
            for (int i = 0; i < P_N; ++i) o[i] = q[i];
        }
        // group offsets of the near list, in vertex order (NG = 32 groups: one per lane)
        const int c = __popc(gmask[lane]);
        int incl = c;
        for (int off = 1; off < 32; off <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += t;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int b = 0;
        if (lane == 0 && total > 0) b = atomicAdd(a.near_count, total);
        b = __shfl_sync(0xffffffffu, b, 0);
        gbase[lane] = b + incl - c;
    }
    __syncthreads();
    const unsigned below = (1u << lane) - 1u;
    for (int g = warp; g < NG; g += 8) {
        const unsigned m = gmask[g];
        if (m & (1u << lane)) a.near_list[gbase[g] + __popc(m & below)] = vbase + 32 * g + lane;
    }
}

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------

// Area of {d <= r} in a linear face and its derivative (lean_geometry.py:66-88).
__device__ __forceinline__ void face_cdf(double d0, double d1, double d2, double A, double r, double& ar,
                                         double& da) {
    double lo = d0, mi = d1, hi = d2, t;
    if (lo > mi) { t = lo; lo = mi; mi = t; }
    if (mi > hi) { t = mi; mi = hi; hi = t; }
    if (lo > mi) { t = lo; lo = mi; mi = t; }
    // both partial cases in one branch-free form (one division): x = r - lo below the
    // middle corner, y = hi - r from it on
    const bool below = r < mi;
    const double z = below ? r - lo : hi - r;
    const double q = z / ((hi - lo) * (below ? mi - lo : hi - mi));
    const double zq = z * q;
    const double a_in = below ? A * zq : A * (1.0 - zq);
    const double d_in = 2.0 * A * q;
    const bool whole = r >= hi, none = r <= lo;
    ar = whole ? A : (none ? 0.0 : a_in);
    da = (whole || none) ? 0.0 : d_in;
}

// |grad d| on a face (lean_geometry.py:91-96).
__device__ __forceinline__ double grad_norm(double d0, double d1, double d2, double g11, double g12, double g22) {
    const double al = d1 - d0, be = d2 - d0;
    const double q = al * al * g11 + 2.0 * al * be * g12 + be * be * g22;
    return q > 0.0 ? sqrt(q) : 0.0;
}

// Sum over the warp; every lane returns lane 0's value, so callers' control
// flow (the Newton iteration) stays warp-uniform.
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Threads per source CTA: four CTAs share an SM, so one source's barrier waits
// (uneven near-vertex walks, idle warps in the last round of targets) overlap
// with the other sources' work.
constexpr int kMetricThreads = 256;

// Each distance bin of the complete range is split into up to kSubBins sub-bins by
// the same quotient hi / width that picks the bin, so that an evaluation at r can
// take the faces below r's sub-bin as whole areas and skip the sub-bins above r
// whose faces (and all later ones) lie beyond r.
constexpr int kSubBins = 16;
constexpr int kInfKey = 0x7f800000;  // lo_key(+inf)

// Order-preserving int key of a float (for atomicMin) and back.
__device__ __forceinline__ int lo_key(double lo) {
    const int b = __float_as_int(__double2float_rd(lo));  // rounded down: a lower bound of lo
    return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ double key_lo(int k) { return (double)__int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

struct SrcShared {
    union {
        unsigned long long hist[kMaxBins + 1];  // face areas per sub-bin, fixed point (order-free sums)
        double pre[kMaxBins + 1];               // then the exclusive prefix sums of the sub-bins' areas
    };
    int ptr[kMaxBins + 1];     // faces per sub-bin -> exclusive prefix -> (counting sort) inclusive prefix
    double red[32][4];         // per warp (up to 1024 threads)
    double dred[32][5];
    double radii[kMaxTargets];
    double total, dglob;
    int minlo[kMaxBins + 1];   // per sub-bin: a lower bound of its faces' lo (lo_key), then the suffix minima
    int nbins, rc, nlong, ntot, n_eval, bad, overflow;
    int sb;                    // sub-bins per bin
    int nstage;                // binned faces staged (unsorted) at the top of the band array
};

// Sub-bins per bin for nbb complete bins: as many as the shared arrays hold.
__device__ __forceinline__ int sub_bins(int nbb) {
    int sb = kSubBins;
    while (sb > 1 && nbb * sb > kMaxBins) sb >>= 1;
    return sb;
}

// Sub-bin of quotient q = hi / width within its bin kb = bin_of(hi). (q - kb) * sb is
// exact (Sterbenz, power-of-two scale), so sub-bin order follows q, and q follows hi.
__device__ __forceinline__ int sub_of(double q, int kb, int sb) {
    const int j = (int)((q - (double)kb) * sb);
    return j < 0 ? 0 : (j >= sb ? sb - 1 : j);
}

// A source's distance field with its near-face bins (lean_geometry.py:117-299 restated over
// the faces that can matter): bins [0, rc) are complete, larger bins are never queried.
template <typename T>
struct Field {
    const T* d;
    const MetricArgs* a;
    SrcShared* s;
    const int4* band;      // near faces (face, corners) sorted by sub-bin
    const int32_t* longf;  // near faces whose distance extent exceeds the bin width

    __device__ double dv(int v) const { return (double)d[v]; }
    __device__ int bin_of(double dmax) const {
        const int k = (int)(dmax / a->width);
        return k < 0 ? 0 : k;
    }
    __device__ double prefix_at(int k) const { return k <= s->rc && k < s->nbins ? s->pre[k * s->sb] : s->total; }

    __device__ void face_term(int f, double r, int mode, double& x1, double& x2) const {
        const int* fv = a->fv;
        const double d0 = dv(fv[3 * f]), d1 = dv(fv[3 * f + 1]), d2 = dv(fv[3 * f + 2]);
        double ar, da;
        face_cdf(d0, d1, d2, a->farea[f], r, ar, da);
        if (mode == 0) {
            x1 += ar;
            x2 += da;
        } else if (da > 0.0) {
            x1 += da * grad_norm(d0, d1, d2, a->g11[f], a->g12[f], a->g22[f]);
        }
    }

    // face_term of a band record (face, corners): no lookup of the face's corners
    __device__ void rec_term(const int4& q, double d0, double d1, double d2, double r, int mode, double& x1,
                             double& x2) const {
        double ar, da;
        face_cdf(d0, d1, d2, a->farea[q.x], r, ar, da);
        if (mode == 0) {
            x1 += ar;
            x2 += da;
        } else if (da > 0.0) {
            x1 += da * grad_norm(d0, d1, d2, a->g11[q.x], a->g12[q.x], a->g22[q.x]);
        }
    }

    // Faces with bin in [kr, kend) plus long faces with bin >= kend, summed by one warp;
    // `inside` + s1 is the area (mode 0). Within complete bins only the sub-bins
    // [j0, j1) are visited: every face of a lower sub-bin has hi < r (face_cdf would
    // return its whole area, summed into `inside` from the prefix), and every face
    // from sub-bin j1 on has lo >= r (both of its terms are exactly zero).
    __device__ void band_sum(int kr, int kend, double r, int mode, double& s1, double& s2, double& inside) const {
        const int lane = threadIdx.x & 31;
        double x1 = 0.0, x2 = 0.0;
        const int* fv = a->fv;
        if (kend <= s->rc) {
            const int sb = s->sb;
            const int j0 = kr * sb + sub_of(r / a->width, kr, sb);
            const int jend = kend * sb;  // at most j0 + 2 * kSubBins
            // j1: the first sub-bin above j0 from which on every binned face has lo >= r
            const int jc = j0 + 1 + lane;
            const unsigned far = __ballot_sync(0xffffffffu, jc < jend && key_lo(s->minlo[jc]) >= r);
            const int j1 = far ? j0 + __ffs(far) : jend;
            inside = s->pre[j0];
            // sub-bin j's faces are band[ptr[j-1], ptr[j]) after the counting sort
            int j = (j0 > 0 ? s->ptr[j0 - 1] : 0) + lane;
            const int je = s->ptr[j1 - 1];
            // two records per lane in flight
            for (; j + 32 < je; j += 64) {
                int4 q[2];
                double dd[2][3];
#pragma unroll
                for (int u = 0; u < 2; ++u) q[u] = band[j + 32 * u];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    dd[u][0] = dv(q[u].y);
                    dd[u][1] = dv(q[u].z);
                    dd[u][2] = dv(q[u].w);
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) rec_term(q[u], dd[u][0], dd[u][1], dd[u][2], r, mode, x1, x2);
            }
            for (; j < je; j += 32) {
                const int4 q0 = band[j];
                rec_term(q0, dv(q0.y), dv(q0.z), dv(q0.w), r, mode, x1, x2);
            }
        } else {  // beyond the complete bins: scan every face (not reached for healthy fields)
            inside = prefix_at(kr);
            for (int f = lane; f < a->nf; f += 32) {
                const double d0 = dv(fv[3 * f]), d1 = dv(fv[3 * f + 1]), d2 = dv(fv[3 * f + 2]);
                if (!(isfinite(d0) && isfinite(d1) && isfinite(d2))) continue;
                const int kb = bin_of(fmax(fmax(d0, d1), d2));
                if (kb >= kr && kb < kend) face_term(f, r, mode, x1, x2);
            }
        }
        for (int j = lane; j < s->nlong; j += 32) {
            const int f = longf[j];
            const double d0 = dv(fv[3 * f]), d1 = dv(fv[3 * f + 1]), d2 = dv(fv[3 * f + 2]);
            if (bin_of(fmax(fmax(d0, d1), d2)) >= kend) face_term(f, r, mode, x1, x2);
        }
        s1 = warp_sum(x1);
        s2 = warp_sum(x2);
    }

    // lean_geometry.py:183-212
    __device__ void area_at(double r, double& A, double& dA) const {
        if (!(r > 0.0)) { A = 0.0; dA = 0.0; return; }
        const int kr = (int)(r / a->width);
        if (kr >= s->nbins) { A = s->total; dA = 0.0; return; }
        const int kend = min(kr + 2, s->nbins);
        double b1, b2, inside;
        band_sum(kr, kend, r, 0, b1, b2, inside);
        A = inside + b1;
        dA = b2;
    }

    // lean_geometry.py:215-244
    __device__ double perimeter_at(double r) const {
        if (!(r > 0.0)) return 0.0;
        const int kr = (int)(r / a->width);
        if (kr >= s->nbins) return 0.0;
        const int kend = min(kr + 2, s->nbins);
        double b1, b2, inside;
        band_sum(kr, kend, r, 1, b1, b2, inside);
        return b1;
    }

    // lean_geometry.py:247-299
    __device__ double solve_radius(double target, int& n_eval) const {
        n_eval = 0;
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        if (target != target) return nan;
        if (target <= 0.0) return 0.0;
        if (target > s->total * (1.0 + 1e-12)) return nan;
        int lo_i = 0, hi_i = s->nbins;
        while (lo_i < hi_i) {
            const int mid = (lo_i + hi_i) / 2;
            if (prefix_at(mid) >= target) hi_i = mid; else lo_i = mid + 1;
        }
        const double w = a->width;
        double r_hi = lo_i * w;
        double r_lo = lo_i >= 2 ? (lo_i - 2) * w : 0.0;
        double A, dA;
        if (s->nlong > 0) {
            while (r_lo > 0.0) {
                area_at(r_lo, A, dA);
                ++n_eval;
                if (A < target) break;
                r_hi = r_lo;
                r_lo = r_lo - 2.0 * w;
                if (r_lo < 0.0) r_lo = 0.0;
            }
        }
        double r = 0.5 * (r_lo + r_hi);
        for (int it = 0; it < a->max_iter; ++it) {
            area_at(r, A, dA);
            ++n_eval;
            const double err = A - target;
            if (fabs(err) <= a->rtol * target) return r;
            if (err > 0.0) r_hi = r; else r_lo = r;
            double rn = 0.5 * (r_lo + r_hi);
            if (dA > 0.0) {
                const double cand = r - err / dA;
                if (r_lo < cand && cand < r_hi) rn = cand;
            }
            if (r_hi - r_lo <= 1e-13 * (1.0 + r_hi)) return rn;
            r = rn;
        }
        return r;
    }
};


// Everything computed from one source's field, one CTA per source:
//   1. the health screen, MSD and global max from the shift kernel's partial sums,
//      and the distance to boundary;
//   2. the faces that have a corner closer than rc*w (rc starts at a first cut inside
//      the radius of the shift kernel's near lists), each emitted once by its first
//      near corner through the vertex->face incidence lists: their area histogram,
//      counting sort by sub-bin and the long-face list (lean_geometry.py:117-180 on
//      these faces). Bins below rc are complete. If the largest target is not enclosed
//      two bins below rc, rc grows (to the near lists' radius, then up to every bin,
//      scanning all vertices) and step 2 repeats;
//   3. one warp per target: bracket + safeguarded Newton + perimeter; then the samples.
template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_source_metrics(MetricArgs a, const T* __restrict__ dT) {
    __shared__ SrcShared S;
    const int k = blockIdx.x;
    const int src = a.src[k];
    if (src < 0) return;
    const int tid = threadIdx.x, bs = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = bs >> 5;
    const int nt = a.n_targets, m = a.n_between;
    const int ne = nt > 0 ? (nt - 1) * m : 0;
    double* o = (a.desc ? a.desc->out : a.out) + (int64_t)k * a.stride;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    const T* d = dT + (int64_t)k * a.n;
    int4* band = a.band + (int64_t)k * a.nf;
    int32_t* longf = a.longf + (int64_t)k * a.nf;
    const double w = a.width;

    // 1. reduce the shift kernel's partial statistics (fixed order: deterministic)
    double sum_d = 0.0, sum_da = 0.0, sum_a = 0.0, dmax = 0.0;
    double cnt = 0.0, neg = 0.0, viol = 0.0, nonfinite = 0.0;
    for (int tI = tid; tI < a.ntiles; tI += bs) {
        const double* q = a.partials + ((int64_t)tI * a.K + k) * P_N;
        sum_d += q[P_SUM_D]; sum_da += q[P_SUM_DA]; sum_a += q[P_SUM_A]; cnt += q[P_CNT];
        neg += q[P_NEG]; viol += q[P_VIOL]; nonfinite += q[P_NONFINITE]; dmax = fmax(dmax, q[P_DMAX]);
    }
    double bmin = INFINITY;
    double bcnt = 0.0;
    for (int i = tid; i < a.n_boundary; i += bs) {
        const double di = (double)d[a.boundary[i]];
        if (isfinite(di)) { bmin = fmin(bmin, di); bcnt += 1.0; }
    }
    for (int off = 16; off > 0; off >>= 1) {
        sum_d += __shfl_down_sync(0xffffffffu, sum_d, off);
        sum_da += __shfl_down_sync(0xffffffffu, sum_da, off);
        sum_a += __shfl_down_sync(0xffffffffu, sum_a, off);
        bmin = fmin(bmin, __shfl_down_sync(0xffffffffu, bmin, off));
        dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, off));
        cnt += __shfl_down_sync(0xffffffffu, cnt, off);
        neg += __shfl_down_sync(0xffffffffu, neg, off);
        viol += __shfl_down_sync(0xffffffffu, viol, off);
        nonfinite += __shfl_down_sync(0xffffffffu, nonfinite, off);
        bcnt += __shfl_down_sync(0xffffffffu, bcnt, off);
    }
    if (lane == 0) {
        S.red[warp][0] = sum_d; S.red[warp][1] = sum_da; S.red[warp][2] = sum_a; S.red[warp][3] = bmin;
        S.dred[warp][0] = cnt; S.dred[warp][1] = neg; S.dred[warp][2] = viol; S.dred[warp][3] = nonfinite;
        S.dred[warp][4] = bcnt;
        S.radii[warp] = dmax;  // scratch for the block max
    }
    __syncthreads();
    if (tid == 0) {
        double Sd = 0, Sda = 0, Sa = 0, Bm = INFINITY, Dm = 0.0, C = 0, NG = 0, VI = 0, NF = 0, BC = 0;
        for (int q = 0; q < nwarps; ++q) {
            Sd += S.red[q][0]; Sda += S.red[q][1]; Sa += S.red[q][2]; Bm = fmin(Bm, S.red[q][3]);
            Dm = fmax(Dm, S.radii[q]);
            C += S.dred[q][0]; NG += S.dred[q][1]; VI += S.dred[q][2]; NF += S.dred[q][3]; BC += S.dred[q][4];
        }
        o[0] = C > 0 ? Sd / C : nan;
        o[1] = (C > 0 && isfinite(Sa) && Sa > 0.0) ? Sda / Sa : nan;
        o[2] = a.n_boundary > 0 ? (BC > 0 ? Bm : nan) : INFINITY;
        const double negf = NF > 0 ? nan : NG / (double)a.n;
        const double violf = NF > 0 ? nan : VI / (double)a.n;
        o[3] = negf;
        o[4] = violf;
        S.bad = (NF > 0 || negf > 1e-3 || violf > 1e-3) ? 1 : 0;
        o[5] = S.bad ? 1.0 : 0.0;
        S.dglob = Dm;
        const double nb = Dm / w;
        S.nbins = nb < (double)(kMaxBins - 2) ? (int)nb + 2 : kMaxBins + 1;
        S.total = a.total_area;
        S.n_eval = 0;
        S.rc = a.first_bins;
    }
    __syncthreads();
    // A flagged field gets no geometry (core_analysis.py:1558-1564).
    if (S.bad || S.nbins > kMaxBins) {
        if (!S.bad && tid == 0) atomicOr(a.err, KERR_HIST_OVERFLOW);
        for (int i = tid; i < 2 * nt + 2 * ne; i += bs) o[7 + i] = nan;
        if (tid == 0) o[6] = 0.0;
        return;
    }
    const int nbins = S.nbins;
    double tmax = 0.0;
    for (int t = 0; t < nt; ++t)
        if (a.targets[t] > tmax && a.targets[t] <= S.total * (1.0 + 1e-12)) tmax = a.targets[t];

    // 2. near faces, with a growing cut if the margin was not enough
    Field<T> F{d, &a, &S, band, longf};
    for (int attempt = 0; attempt < 32; ++attempt) {
        const int rc = S.rc;
        const int nbb = min(rc + 1, nbins);  // complete bins [0, nbb)
        const int sb = sub_bins(nbb);
        const int nsub = nbb * sb;
        for (int i = tid; i <= nsub; i += bs) {
            S.hist[i] = 0ull;
            S.ptr[i] = 0;
            S.minlo[i] = kInfKey;
        }
        if (tid == 0) { S.nlong = 0; S.overflow = 0; S.sb = sb; S.nstage = 0; }
        __syncthreads();
        const double R = rc >= nbins ? INFINITY : rc * w;
        // vertices closer than R: from the shift kernel's near list while R is within its radius
        const bool listed = rc <= a.near_bins && rc < nbins;
        const int nv_scan = listed ? a.near_count[k] : a.n;
        const int32_t* nl = a.near_list + (int64_t)k * a.n;
        for (int pass = 0; pass < 2; ++pass) {  // 0: histogram + long faces, 1: counting sort
            // pass 0 also stages each binned face at the top of the band array; while the
            // staged list and the sorted one (both ntot long) cannot overlap, pass 1 sorts
            // the staged list instead of walking the incidences again
            if (pass == 1 && 2 * S.ntot <= a.nf) {
                const int ntot = S.ntot;
                for (int p = tid; p < ntot; p += bs) {
                    const int4 rq = band[a.nf - 1 - p];
                    const double d0 = (double)d[rq.y], d1 = (double)d[rq.z], d2 = (double)d[rq.w];
                    double hi = d0;  // as in pass 0
                    if (d1 > hi) hi = d1;
                    if (d2 > hi) hi = d2;
                    const double q = hi / w;
                    const int kb = q < 1.0 ? 0 : (int)q;
                    band[atomicAdd(&S.ptr[kb * sb + sub_of(q, kb, sb)], 1)] = rq;
                }
                __syncthreads();
                continue;
            }
            for (int ii = tid; ii < nv_scan; ii += bs) {
                const int i = listed ? nl[ii] : ii;
                const double di = (double)d[i];
                if (!(di < R)) continue;
                const int q1 = a.inc_ptr[i + 1];
                constexpr int QB = sizeof(T) == 4 ? 4 : 2;
                // the vertex's incidences in groups of QB: the records, then their corner
                // distances, are loaded together before any is used
                for (int qb = a.inc_ptr[i]; qb < q1; qb += QB) {
                    int4 rec[QB];
                    int cc[QB];
                    T dd[QB][3];
                    long long fx[QB];
#pragma unroll
                    for (int u = 0; u < QB; ++u)
                        if (qb + u < q1) {
                            rec[u] = a.inc_rec[qb + u];
                            cc[u] = a.inc_corner[qb + u];
                        }
#pragma unroll
                    for (int u = 0; u < QB; ++u)
                        if (qb + u < q1) {
                            dd[u][0] = d[rec[u].y];
                            dd[u][1] = d[rec[u].z];
                            dd[u][2] = d[rec[u].w];
                            if (pass == 0) fx[u] = a.farea_fx[rec[u].x];
                        }
#pragma unroll
                    for (int u = 0; u < QB; ++u) {
                        if (qb + u >= q1) continue;
                        const int f = rec[u].x;
                        const int c = cc[u];
                        const double d0 = (double)dd[u][0], d1 = (double)dd[u][1], d2 = (double)dd[u][2];
                        if (c >= 1 && d0 < R) continue;   // an earlier corner emits it
                        if (c == 2 && d1 < R) continue;
                        // (every value is finite here: a field with a non-finite value is flagged above)
                        double lo = d0, hi = d0;
                        if (d1 < lo) lo = d1;
                        if (d1 > hi) hi = d1;
                        if (d2 < lo) lo = d2;
                        if (d2 > hi) hi = d2;
                        const double q = hi / w;  // F.bin_of's quotient
                        const int kb = q < 1.0 ? 0 : (int)q;
                        const int jb = kb * sb + sub_of(q, kb, sb);
                        if (pass == 0) {
                            if (hi - lo > w) longf[atomicAdd(&S.nlong, 1)] = f;
                            if (kb < nbb) {
                                atomicAdd(&S.hist[jb], (unsigned long long)fx[u]);
                                atomicAdd(&S.ptr[jb], 1);
                                atomicMin(&S.minlo[jb], lo_key(lo));
                                band[a.nf - 1 - atomicAdd(&S.nstage, 1)] = rec[u];
                            }
                        } else if (kb < nbb) {
                            band[atomicAdd(&S.ptr[jb], 1)] = rec[u];  // ptr[jb] ends at the next sub-bin's start
                        }
                    }
                }
            }
            __syncthreads();
            if (pass == 0) {
                // exclusive prefix sums over the sub-bins [0, nsub) by warp 0, exact in
                // fixed point, each rounded once to an area
                if (warp == 0) {
                    const int chunk = (nsub + 31) / 32;
                    const int b0 = min(lane * chunk, nsub), b1 = min(b0 + chunk, nsub);
                    unsigned long long sa = 0ull;
                    int sc = 0;
                    for (int b = b0; b < b1; ++b) { sa += S.hist[b]; sc += S.ptr[b]; }
                    unsigned long long ea = sa;
                    int ec = sc;
                    for (int off = 1; off < 32; off <<= 1) {
                        const unsigned long long ta = __shfl_up_sync(0xffffffffu, ea, off);
                        const int tc = __shfl_up_sync(0xffffffffu, ec, off);
                        if (lane >= off) { ea += ta; ec += tc; }
                    }
                    unsigned long long ra = ea - sa;
                    int rcn = ec - sc;
                    for (int b = b0; b < b1; ++b) {
                        const unsigned long long xa = S.hist[b];
                        const int xc = S.ptr[b];
                        S.pre[b] = (double)ra * a.area_unscale;
                        S.ptr[b] = rcn;
                        ra += xa;
                        rcn += xc;
                    }
                    if (lane == 31) {
                        S.ntot = ec;
                        S.pre[nsub] = (double)ea * a.area_unscale;
                        S.ptr[nsub] = ec;
                    }
                } else if (warp == 1) {
                    // suffix minima of the sub-bins' lower bounds of lo
                    const int chunk = (nsub + 31) / 32;
                    const int b0 = min(lane * chunk, nsub), b1 = min(b0 + chunk, nsub);
                    int mk = kInfKey;
                    for (int b = b0; b < b1; ++b) mk = min(mk, S.minlo[b]);
                    for (int off = 1; off < 32; off <<= 1) {
                        const int t = __shfl_down_sync(0xffffffffu, mk, off);
                        if (lane + off < 32) mk = min(mk, t);
                    }
                    int after = __shfl_down_sync(0xffffffffu, mk, 1);
                    if (lane == 31) after = kInfKey;
                    for (int b = b1 - 1; b >= b0; --b) {
                        after = min(after, S.minlo[b]);
                        S.minlo[b] = after;
                    }
                }
                __syncthreads();
            }
        }
        // enough? the largest target must be enclosed two bins below the cut
        bool ok = rc >= nbins || (rc >= 2 && S.pre[(rc - 2) * sb] >= tmax);
        if (ok) break;
        __syncthreads();
        if (tid == 0) S.rc = rc < a.near_bins ? a.near_bins : min(nbins, 2 * rc + 4);
        __syncthreads();
    }
    if (S.rc >= nbins) {
        // every bin is complete: the prefix array covers [0, nbins]
        if (tid == 0) S.rc = nbins;
    }
    __syncthreads();

    // 3. radii + perimeters, one warp per target (lean_geometry.py:315-324)
    for (int t = warp; t < nt; t += nwarps) {
        int ev = 0;
        const double r = F.solve_radius(a.targets[t], ev);
        double p = nan;
        if (r == r) p = F.perimeter_at(r);
        if (lane == 0) {
            S.radii[t] = r;
            o[7 + t] = r;
            o[7 + nt + t] = p;
            atomicAdd(&S.n_eval, ev);
        }
    }
    __syncthreads();
    // supplementary samples between consecutive radii (lean_geometry.py:325-339)
    for (int idx = warp; idx < ne; idx += nwarps) {
        const int si = idx / m, j = idx - si * m;
        const double r0 = S.radii[si], r1 = S.radii[si + 1];
        double rr = nan, ar = nan;
        if (r0 == r0 && r1 == r1 && r0 > 0.0 && r1 > r0) {
            rr = exp(log(r0) + a.fracs[j] * (log(r1) - log(r0)));
            double dA;
            F.area_at(rr, ar, dA);
            if (lane == 0) atomicAdd(&S.n_eval, 1);
        }
        if (lane == 0) {
            o[7 + 2 * nt + idx] = rr;
            o[7 + 2 * nt + ne + idx] = ar;
        }
    }
    __syncthreads();
    if (tid == 0) o[6] = (double)S.n_eval;
}

__global__ void k_permute_rows(int32_t n, int32_t cols, const double* __restrict__ in, int32_t in_ld,
                               const int32_t* __restrict__ in_idx, double* __restrict__ out, int32_t out_ld,
                               const int32_t* __restrict__ out_idx) {
    const int64_t total = (int64_t)n * cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / cols), c = (int)(e - (int64_t)i * cols);
        const int ri = in_idx ? in_idx[i] : i;
        const int ro = out_idx ? out_idx[i] : i;
        out[(int64_t)ro * out_ld + c] = in[(int64_t)ri * in_ld + c];
    }
}

}  // namespace

template <typename Tin, typename Tout>
void launch_shift_transpose(int32_t n, int32_t K, const Tin* phi, const int32_t* src, Tout* dT, cudaStream_t st) {
    if (n <= 0 || K <= 0) return;
    k_shift_transpose<Tin, Tout><<<dim3((n + 31) / 32, K / 32), dim3(32, 8), 0, st>>>(n, K, phi, src, dT);
}

void launch_permute_rows(int32_t n, int32_t cols, const double* in, int32_t in_ld, const int32_t* in_idx,
                         double* out, int32_t out_ld, const int32_t* out_idx, cudaStream_t st) {
    if (n <= 0 || cols <= 0) return;
    int64_t total = (int64_t)n * cols;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_permute_rows<<<blocks, 256, 0, st>>>(n, cols, in, in_ld, in_idx, out, out_ld, out_idx);
}

template <typename Tin, typename Tout>
void launch_shift_stats(const MetricArgs& a, int32_t K, const Tin* phi, Tout* dT, cudaStream_t st) {
    if (a.n <= 0 || K <= 0) return;
    cudaMemsetAsync(a.near_count, 0, (size_t)K * sizeof(int), st);
    k_shift_stats<Tin, Tout><<<dim3(a.ntiles, K / 32), dim3(32, 8), 0, st>>>(a, K, phi, dT);
}

void launch_shift_stats_one(const MetricArgs& a, const double* phi, double* d, cudaStream_t st) {
    if (a.n <= 0) return;
    cudaMemsetAsync(a.near_count, 0, sizeof(int), st);
    k_shift_stats_one<<<a.ntiles, 256, 0, st>>>(a, phi, d);
}

template <typename T>
void launch_source_metrics(const MetricArgs& a, const T* dT, cudaStream_t st) {
    if (a.nsrc <= 0) return;
    // a lone source (the single-source path) gets a CTA of 1024 threads: its binning, sort and
    // targets spread over 32 warps instead of waiting on one CTA's 8
    if (a.nsrc == 1) k_source_metrics<T, 1024><<<1, 1024, 0, st>>>(a, dT);
    else k_source_metrics<T, kMetricThreads><<<a.nsrc, kMetricThreads, 0, st>>>(a, dT);
}

template void launch_shift_transpose<double, double>(int32_t, int32_t, const double*, const int32_t*, double*,
                                                     cudaStream_t);
template void launch_shift_transpose<float, float>(int32_t, int32_t, const float*, const int32_t*, float*,
                                                   cudaStream_t);
template void launch_shift_stats<double, double>(const MetricArgs&, int32_t, const double*, double*, cudaStream_t);
template void launch_shift_stats<float, float>(const MetricArgs&, int32_t, const float*, float*, cudaStream_t);
template void launch_source_metrics<double>(const MetricArgs&, const double*, cudaStream_t);
template void launch_source_metrics<float>(const MetricArgs&, const float*, cudaStream_t);

}  // namespace fcw
