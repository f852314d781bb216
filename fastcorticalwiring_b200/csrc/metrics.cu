// Per-source kernels: shift + transpose, vertex statistics, radius/perimeter geometry.
//
// After the Poisson solve the fields sit in an n x K vertex-major block. The
// shift kernel subtracts each column's value at its source and transposes to
// K x n (one contiguous field per source), which the per-source kernels read:
//
//  * vertex statistics, one CTA per source: health screen (lean_geometry.py:343-357),
//    MSD unweighted/area-weighted and distance to boundary (core_analysis.py:1566-1581);
//  * geometry, one CTA per source (lean_geometry.py:117-340): faces are binned by
//    their largest distance into bins of fixed width; the area histogram's
//    prefix sums bracket every target area, faces in the bracketing bins are
//    compacted once (counting sort by bin), and one warp per target runs the
//    reference's safeguarded Newton iteration on A(r) with the exact
//    piecewise-quadratic face areas, then the coarea perimeter; the
//    supplementary log-spaced samples follow, one warp per sample.
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

template <typename T>
__global__ void __launch_bounds__(256) k_vertex_stats(MetricArgs a, const T* __restrict__ dT) {
    const int k = blockIdx.x;
    const int s = a.src[k];
    if (s < 0) return;
    const T* d = dT + (int64_t)k * a.n;
    const double xs0 = a.coords[3 * (int64_t)s], xs1 = a.coords[3 * (int64_t)s + 1], xs2 = a.coords[3 * (int64_t)s + 2];
    const double h = a.health_h;
    double sum_d = 0.0, sum_da = 0.0, sum_a = 0.0;
    int cnt = 0, neg = 0, viol = 0, nonfinite = 0;
    for (int i = threadIdx.x; i < a.n; i += blockDim.x) {
        const double di = (double)d[i];
        if (!isfinite(di)) { ++nonfinite; continue; }
        if (di < -h) ++neg;
        const double dx = a.coords[3 * (int64_t)i] - xs0;
        const double dy = a.coords[3 * (int64_t)i + 1] - xs1;
        const double dz = a.coords[3 * (int64_t)i + 2] - xs2;
        const double chord = __dsqrt_rn(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)));
        if (di < __dsub_rn(dmul(0.9, chord), h)) ++viol;
        if (di > a.eps) {
            const double w = a.vertex_area[i];
            sum_d += di;
            sum_da += di * w;
            sum_a += w;
            ++cnt;
        }
    }
    double bmin = INFINITY;
    int bcnt = 0;
    for (int i = threadIdx.x; i < a.n_boundary; i += blockDim.x) {
        const double di = (double)d[a.boundary[i]];
        if (isfinite(di)) { bmin = fmin(bmin, di); ++bcnt; }
    }
    // block reduction
    __shared__ double rd[4][8];
    __shared__ int ri[5][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        sum_d += __shfl_down_sync(0xffffffffu, sum_d, o);
        sum_da += __shfl_down_sync(0xffffffffu, sum_da, o);
        sum_a += __shfl_down_sync(0xffffffffu, sum_a, o);
        bmin = fmin(bmin, __shfl_down_sync(0xffffffffu, bmin, o));
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        neg += __shfl_down_sync(0xffffffffu, neg, o);
        viol += __shfl_down_sync(0xffffffffu, viol, o);
        nonfinite += __shfl_down_sync(0xffffffffu, nonfinite, o);
        bcnt += __shfl_down_sync(0xffffffffu, bcnt, o);
    }
    if (lane == 0) {
        rd[0][warp] = sum_d; rd[1][warp] = sum_da; rd[2][warp] = sum_a; rd[3][warp] = bmin;
        ri[0][warp] = cnt; ri[1][warp] = neg; ri[2][warp] = viol; ri[3][warp] = nonfinite; ri[4][warp] = bcnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        double Sd = 0, Sda = 0, Sa = 0, Bm = INFINITY;
        int C = 0, NG = 0, VI = 0, NF = 0, BC = 0;
        for (int w = 0; w < nw; ++w) {
            Sd += rd[0][w]; Sda += rd[1][w]; Sa += rd[2][w]; Bm = fmin(Bm, rd[3][w]);
            C += ri[0][w]; NG += ri[1][w]; VI += ri[2][w]; NF += ri[3][w]; BC += ri[4][w];
        }
        double* o = a.out + (int64_t)k * a.stride;
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        o[0] = C > 0 ? Sd / (double)C : nan;
        o[1] = (C > 0 && isfinite(Sa) && Sa > 0.0) ? Sda / Sa : nan;
        o[2] = a.n_boundary > 0 ? (BC > 0 ? Bm : nan) : INFINITY;
        const double negf = NF ? nan : (double)NG / (double)a.n;
        const double violf = NF ? nan : (double)VI / (double)a.n;
        o[3] = negf;
        o[4] = violf;
        o[5] = (NF > 0 || negf > 1e-3 || violf > 1e-3) ? 1.0 : 0.0;
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
    if (r >= hi) { ar = A; da = 0.0; return; }
    if (r <= lo) { ar = 0.0; da = 0.0; return; }
    if (r < mi) {
        const double den = (mi - lo) * (hi - lo);
        const double x = r - lo;
        ar = A * x * x / den;
        da = 2.0 * A * x / den;
        return;
    }
    const double den = (hi - lo) * (hi - mi);
    const double y = hi - r;
    ar = A * (1.0 - y * y / den);
    da = 2.0 * A * y / den;
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

struct GeoShared {
    double pre[kMaxBins];   // exclusive prefix of face area per bin
    int ptr[kMaxBins];      // exclusive prefix of face count per bin
    int fill[kMaxBins];
    double red[32];
    double radii[kMaxTargets];
    double total;
    int nbins, nlong, ntot, b_lo, b_hi, base, n_eval, bad_scan;
};

template <typename T>
struct Field {
    const T* d;
    const MetricArgs* a;
    GeoShared* s;
    const int32_t* band;   // compacted faces of bins [b_lo, b_hi], sorted by bin
    const int32_t* longf;

    __device__ double dv(int v) const { return (double)d[v]; }
    __device__ int bin_of(double dmax) const {
        int k = (int)(dmax / a->width);
        return k < 0 ? 0 : k;
    }
    __device__ int ptr_at(int k) const { return k < s->nbins ? s->ptr[k] : s->ntot; }
    __device__ double prefix_at(int k) const { return k < s->nbins ? s->pre[k] : s->total; }

    // Band + long-face sums over faces with bin in [kr, kend), all lanes of a warp.
    // mode 0: (A, dA) contributions; mode 1: perimeter.
    __device__ void band_sum(int kr, int kend, double r, int mode, double& s1, double& s2) const {
        const int lane = threadIdx.x & 31;
        double x1 = 0.0, x2 = 0.0;
        const int* fv = a->fv;
        if (kr >= s->b_lo && kend - 1 <= s->b_hi) {
            const int j0 = ptr_at(kr) - s->base, j1 = ptr_at(kend) - s->base;
            for (int j = j0 + lane; j < j1; j += 32) face_term(band[j], r, mode, x1, x2);
        } else {  // outside the compacted range: scan every face (rare; long-face walk-down)
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

    // lean_geometry.py:183-212
    __device__ void area_at(double r, double& A, double& dA) const {
        if (!(r > 0.0)) { A = 0.0; dA = 0.0; return; }
        const int kr = (int)(r / a->width);
        if (kr >= s->nbins) { A = s->total; dA = 0.0; return; }
        const int kend = min(kr + 2, s->nbins);
        double b1, b2;
        band_sum(kr, kend, r, 0, b1, b2);
        A = prefix_at(kr) + b1;
        dA = b2;
    }

    // lean_geometry.py:215-244
    __device__ double perimeter_at(double r) const {
        if (!(r > 0.0)) return 0.0;
        const int kr = (int)(r / a->width);
        if (kr >= s->nbins) return 0.0;
        const int kend = min(kr + 2, s->nbins);
        double b1, b2;
        band_sum(kr, kend, r, 1, b1, b2);
        return b1;
    }

    // lean_geometry.py:247-299 (bracket already known: lo_i)
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

template <typename T>
__global__ void __launch_bounds__(512) k_geometry(MetricArgs a, const T* __restrict__ dT) {
    __shared__ GeoShared S;
    const int k = blockIdx.x;
    const int src = a.src[k];
    if (src < 0) return;
    const int tid = threadIdx.x, bs = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = bs >> 5;
    const int nt = a.n_targets, m = a.n_between;
    const int ne = nt > 0 ? (nt - 1) * m : 0;
    double* o = a.out + (int64_t)k * a.stride;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    const T* d = dT + (int64_t)k * a.n;
    int32_t* band = a.band + (int64_t)k * a.nf;
    int32_t* longf = a.longf + (int64_t)k * a.nf;

    // A flagged field gets no geometry (core_analysis.py:1558-1564).
    if (o[5] != 0.0) {
        for (int i = tid; i < 2 * nt + 2 * ne; i += bs) o[7 + i] = nan;
        if (tid == 0) o[6] = 0.0;
        return;
    }
    for (int i = tid; i < kMaxBins; i += bs) { S.pre[i] = 0.0; S.ptr[i] = 0; S.fill[i] = 0; }
    if (tid == 0) { S.nlong = 0; S.n_eval = 0; S.bad_scan = 0; }
    __syncthreads();

    // pass 1: per-face max distance -> bin histogram, long faces, global max (lean_geometry.py:125-164)
    const double w = a.width;
    double tmax = 0.0;
    for (int f = tid; f < a.nf; f += bs) {
        const double d0 = (double)d[a.fv[3 * f]], d1 = (double)d[a.fv[3 * f + 1]], d2 = (double)d[a.fv[3 * f + 2]];
        if (!(isfinite(d0) && isfinite(d1) && isfinite(d2))) continue;
        double lo = d0, hi = d0;
        if (d1 < lo) lo = d1;
        if (d1 > hi) hi = d1;
        if (d2 < lo) lo = d2;
        if (d2 > hi) hi = d2;
        if (hi - lo > w) {
            const int idx = atomicAdd(&S.nlong, 1);
            longf[idx] = f;
        }
        if (hi > tmax) tmax = hi;
        int kb = (int)(hi / w);
        if (kb < 0) kb = 0;
        if (kb < kMaxBins) {
            atomicAdd(&S.pre[kb], a.farea[f]);
            atomicAdd(&S.ptr[kb], 1);
        } else {
            S.bad_scan = 1;
        }
    }
    for (int o2 = 16; o2 > 0; o2 >>= 1) tmax = fmax(tmax, __shfl_xor_sync(0xffffffffu, tmax, o2));
    if (lane == 0) S.red[warp] = tmax;
    __syncthreads();
    if (tid == 0) {
        double g = 0.0;
        for (int i = 0; i < nwarps; ++i) g = fmax(g, S.red[i]);
        const double nb = g / w;
        S.nbins = nb < (double)(kMaxBins - 2) ? (int)nb + 2 : kMaxBins + 1;
    }
    __syncthreads();
    if (S.nbins > kMaxBins || S.bad_scan) {
        if (tid == 0) atomicOr(a.err, KERR_HIST_OVERFLOW);
        for (int i = tid; i < 2 * nt + 2 * ne; i += bs) o[7 + i] = nan;
        return;
    }
    // exclusive prefix sums over bins (warp 0: each lane scans a chunk)
    const int nbins = S.nbins;
    if (warp == 0) {
        const int chunk = (nbins + 31) / 32;
        const int b0 = min(lane * chunk, nbins), b1 = min(b0 + chunk, nbins);
        double sa = 0.0;
        int sc = 0;
        for (int b = b0; b < b1; ++b) { sa += S.pre[b]; sc += S.ptr[b]; }
        double ea = sa;
        int ec = sc;
        for (int o2 = 1; o2 < 32; o2 <<= 1) {
            const double ta = __shfl_up_sync(0xffffffffu, ea, o2);
            const int tc = __shfl_up_sync(0xffffffffu, ec, o2);
            if (lane >= o2) { ea += ta; ec += tc; }
        }
        double ra = ea - sa;  // exclusive
        int rc = ec - sc;
        for (int b = b0; b < b1; ++b) {
            const double xa = S.pre[b];
            const int xc = S.ptr[b];
            S.pre[b] = ra;
            S.ptr[b] = rc;
            ra += xa;
            rc += xc;
        }
        if (lane == 31) { S.total = ea; S.ntot = ec; }
    }
    __syncthreads();

    Field<T> F{d, &a, &S, band, longf};
    // bracket bins of every target -> compacted band range
    if (tid == 0) {
        int lo_min = 1 << 30, lo_max = -1;
        for (int t = 0; t < nt; ++t) {
            const double target = a.targets[t];
            if (!(target > 0.0) || target > S.total * (1.0 + 1e-12)) continue;
            int lo_i = 0, hi_i = nbins;
            while (lo_i < hi_i) {
                const int mid = (lo_i + hi_i) / 2;
                if (F.prefix_at(mid) >= target) hi_i = mid; else lo_i = mid + 1;
            }
            lo_min = min(lo_min, lo_i);
            lo_max = max(lo_max, lo_i);
        }
        if (lo_max < 0) { S.b_lo = 1; S.b_hi = 0; }
        else { S.b_lo = max(0, lo_min - 2); S.b_hi = min(nbins - 1, lo_max + 1); }
        S.base = S.b_lo <= S.b_hi ? S.ptr[S.b_lo] : 0;
    }
    __syncthreads();
    // pass 2: counting sort of the faces of bins [b_lo, b_hi] (lean_geometry.py:168-179)
    if (S.b_lo <= S.b_hi) {
        for (int f = tid; f < a.nf; f += bs) {
            const double d0 = (double)d[a.fv[3 * f]], d1 = (double)d[a.fv[3 * f + 1]], d2 = (double)d[a.fv[3 * f + 2]];
            if (!(isfinite(d0) && isfinite(d1) && isfinite(d2))) continue;
            const int kb = F.bin_of(fmax(fmax(d0, d1), d2));
            if (kb < S.b_lo || kb > S.b_hi) continue;
            const int slot = S.ptr[kb] - S.base + atomicAdd(&S.fill[kb], 1);
            band[slot] = f;
        }
    }
    __syncthreads();

    // radii + perimeters, one warp per target (lean_geometry.py:315-324)
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

template <typename T>
void launch_vertex_stats(const MetricArgs& a, const T* dT, cudaStream_t st) {
    if (a.nsrc <= 0) return;
    k_vertex_stats<T><<<a.nsrc, 256, 0, st>>>(a, dT);
}

template <typename T>
void launch_geometry(const MetricArgs& a, const T* dT, cudaStream_t st) {
    if (a.nsrc <= 0) return;
    k_geometry<T><<<a.nsrc, 512, 0, st>>>(a, dT);
}

template void launch_shift_transpose<double, double>(int32_t, int32_t, const double*, const int32_t*, double*,
                                                     cudaStream_t);
template void launch_shift_transpose<float, float>(int32_t, int32_t, const float*, const int32_t*, float*,
                                                   cudaStream_t);
template void launch_vertex_stats<double>(const MetricArgs&, const double*, cudaStream_t);
template void launch_vertex_stats<float>(const MetricArgs&, const float*, cudaStream_t);
template void launch_geometry<double>(const MetricArgs&, const double*, cudaStream_t);
template void launch_geometry<float>(const MetricArgs&, const float*, cudaStream_t);

}  // namespace fcw
