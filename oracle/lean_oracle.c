/*
 * CPU oracle for the per-source geometry and the fused divergence.
 *
 * TEST INFRASTRUCTURE ONLY. This file is a plain-C restatement of the
 * reference algorithm, the CUDA path's results are compared with: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it. The
 * product never links or calls it.
 *
 * Each function cites the reference code it restates (file:line within the
 * FastCorticalWiring project). Arithmetic is written in the same order as the
 * reference so that results agree to the last bit where the reference's JIT
 * does not reassociate (it does not: no fastmath). Build with
 * -ffp-contract=off so no fused multiply-adds are formed.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* lean_geometry.py:66-88 -- area of {d <= r} inside one linear face, and d/dr. */
static void face_cdf(double d0, double d1, double d2, double A, double r,
                     double *area, double *darea) {
    double lo = d0, mid = d1, hi = d2, t;
    if (lo > mid) { t = lo; lo = mid; mid = t; }
    if (mid > hi) { t = mid; mid = hi; hi = t; }
    if (lo > mid) { t = lo; lo = mid; mid = t; }
    if (r >= hi) { *area = A; *darea = 0.0; return; }
    if (r <= lo) { *area = 0.0; *darea = 0.0; return; }
    if (r < mid) {
        double den = (mid - lo) * (hi - lo);
        double x = r - lo;
        *area = A * x * x / den;
        *darea = 2.0 * A * x / den;
        return;
    }
    double den = (hi - lo) * (hi - mid);
    double y = hi - r;
    *area = A * (1.0 - y * y / den);
    *darea = 2.0 * A * y / den;
}

/* lean_geometry.py:91-96 -- |grad d| on a face from the inverse Gram matrix. */
static double grad_norm(double d0, double d1, double d2, double g11, double g12, double g22) {
    double al = d1 - d0, be = d2 - d0;
    double q = al * al * g11 + 2.0 * al * be * g12 + be * be * g22;
    return q > 0.0 ? sqrt(q) : 0.0;
}

typedef struct {
    int64_t nbins;
    int64_t *ptr;     /* nbins + 1 */
    double *prefix;   /* nbins + 1 */
    int64_t n_long;
} buckets_t;

static int finite3(double a, double b, double c) { return isfinite(a) && isfinite(b) && isfinite(c); }

/* lean_geometry.py:117-180 -- bucket faces by dmax into bins of fixed width. */
static int build_buckets(const double *d, const int32_t *F, int64_t nf, const double *area,
                         double width, double *dmax_buf, int32_t *order_buf, int32_t *long_buf,
                         buckets_t *b) {
    double dglob = 0.0;
    int64_t n_long = 0;
    for (int64_t f = 0; f < nf; ++f) {
        double a = d[F[3 * f]], c1 = d[F[3 * f + 1]], c2 = d[F[3 * f + 2]];
        if (!finite3(a, c1, c2)) { dmax_buf[f] = NAN; continue; }
        double lo = a, hi = a;
        if (c1 < lo) lo = c1;
        if (c1 > hi) hi = c1;
        if (c2 < lo) lo = c2;
        if (c2 > hi) hi = c2;
        dmax_buf[f] = hi;
        if (hi - lo > width) long_buf[n_long++] = (int32_t)f;
        if (hi > dglob) dglob = hi;
    }
    int64_t nbins = (int64_t)(dglob / width) + 2;
    int64_t *cnt = (int64_t *)calloc((size_t)(nbins + 1), sizeof(int64_t));
    double *pre = (double *)calloc((size_t)(nbins + 1), sizeof(double));
    int64_t *fill = (int64_t *)malloc((size_t)nbins * sizeof(int64_t));
    if (!cnt || !pre || !fill) { free(cnt); free(pre); free(fill); return -1; }
    for (int64_t f = 0; f < nf; ++f) {
        double h = dmax_buf[f];
        if (h != h) continue;
        int64_t k = (int64_t)(h / width);
        if (k < 0) k = 0; else if (k >= nbins) k = nbins - 1;
        cnt[k + 1] += 1;
        pre[k + 1] += area[f];
    }
    for (int64_t k = 0; k < nbins; ++k) { cnt[k + 1] += cnt[k]; pre[k + 1] += pre[k]; }
    memcpy(fill, cnt, (size_t)nbins * sizeof(int64_t));
    for (int64_t f = 0; f < nf; ++f) {
        double h = dmax_buf[f];
        if (h != h) continue;
        int64_t k = (int64_t)(h / width);
        if (k < 0) k = 0; else if (k >= nbins) k = nbins - 1;
        order_buf[fill[k]++] = (int32_t)f;
    }
    free(fill);
    b->nbins = nbins; b->ptr = cnt; b->prefix = pre; b->n_long = n_long;
    return 0;
}

typedef struct {
    const double *d; const int32_t *F; const double *area;
    const double *g11, *g12, *g22;
    double width; const double *dmax; const int32_t *order; const int32_t *lng;
    buckets_t b;
} field_t;

/* lean_geometry.py:183-212 -- exact A(r) and dA/dr from prefix + two-bin band + long faces. */
static void area_at(const field_t *s, double r, double *A_out, double *dA_out) {
    if (!(r > 0.0)) { *A_out = 0.0; *dA_out = 0.0; return; }
    int64_t kr = (int64_t)(r / s->width);
    if (kr >= s->b.nbins) { *A_out = s->b.prefix[s->b.nbins]; *dA_out = 0.0; return; }
    double A = s->b.prefix[kr], dA = 0.0, a, da;
    int64_t kend = kr + 2;
    if (kend > s->b.nbins) kend = s->b.nbins;
    for (int64_t j = s->b.ptr[kr]; j < s->b.ptr[kend]; ++j) {
        int64_t f = s->order[j];
        face_cdf(s->d[s->F[3 * f]], s->d[s->F[3 * f + 1]], s->d[s->F[3 * f + 2]], s->area[f], r, &a, &da);
        A += a; dA += da;
    }
    for (int64_t j = 0; j < s->b.n_long; ++j) {
        int64_t f = s->lng[j];
        if ((int64_t)(s->dmax[f] / s->width) >= kend) {
            face_cdf(s->d[s->F[3 * f]], s->d[s->F[3 * f + 1]], s->d[s->F[3 * f + 2]], s->area[f], r, &a, &da);
            A += a; dA += da;
        }
    }
    *A_out = A; *dA_out = dA;
}

/* lean_geometry.py:215-244 -- level-set length at r by the coarea formula. */
static double perimeter_at(const field_t *s, double r) {
    if (!(r > 0.0)) return 0.0;
    int64_t kr = (int64_t)(r / s->width);
    if (kr >= s->b.nbins) return 0.0;
    int64_t kend = kr + 2;
    if (kend > s->b.nbins) kend = s->b.nbins;
    double P = 0.0, a, da;
    for (int64_t j = s->b.ptr[kr]; j < s->b.ptr[kend]; ++j) {
        int64_t f = s->order[j];
        double d0 = s->d[s->F[3 * f]], d1 = s->d[s->F[3 * f + 1]], d2 = s->d[s->F[3 * f + 2]];
        face_cdf(d0, d1, d2, s->area[f], r, &a, &da);
        if (da > 0.0) P += da * grad_norm(d0, d1, d2, s->g11[f], s->g12[f], s->g22[f]);
    }
    for (int64_t j = 0; j < s->b.n_long; ++j) {
        int64_t f = s->lng[j];
        if ((int64_t)(s->dmax[f] / s->width) >= kend) {
            double d0 = s->d[s->F[3 * f]], d1 = s->d[s->F[3 * f + 1]], d2 = s->d[s->F[3 * f + 2]];
            face_cdf(d0, d1, d2, s->area[f], r, &a, &da);
            if (da > 0.0) P += da * grad_norm(d0, d1, d2, s->g11[f], s->g12[f], s->g22[f]);
        }
    }
    return P;
}

/* lean_geometry.py:247-299 -- bracket by prefix bisection, then safeguarded Newton. */
static double solve_radius(const field_t *s, double target, double rtol, int max_iter, int64_t *n_eval_out) {
    double total = s->b.prefix[s->b.nbins];
    *n_eval_out = 0;
    if (target != target) return NAN;
    if (target <= 0.0) return 0.0;
    if (target > total * (1.0 + 1e-12)) return NAN;
    int64_t lo_i = 0, hi_i = s->b.nbins;
    while (lo_i < hi_i) {
        int64_t mid = (lo_i + hi_i) / 2;
        if (s->b.prefix[mid] >= target) hi_i = mid; else lo_i = mid + 1;
    }
    double r_hi = (double)lo_i * s->width;
    double r_lo = lo_i >= 2 ? (double)(lo_i - 2) * s->width : 0.0;
    int64_t n_eval = 0;
    double A, dA;
    if (s->b.n_long > 0) {
        while (r_lo > 0.0) {
            area_at(s, r_lo, &A, &dA);
            n_eval++;
            if (A < target) break;
            r_hi = r_lo;
            r_lo = r_lo - 2.0 * s->width;
            if (r_lo < 0.0) r_lo = 0.0;
        }
    }
    double r = 0.5 * (r_lo + r_hi);
    for (int it = 0; it < max_iter; ++it) {
        area_at(s, r, &A, &dA);
        n_eval++;
        double err = A - target;
        if (fabs(err) <= rtol * target) { *n_eval_out = n_eval; return r; }
        if (err > 0.0) r_hi = r; else r_lo = r;
        double rn = 0.5 * (r_lo + r_hi);
        if (dA > 0.0) {
            double cand = r - err / dA;
            if (r_lo < cand && cand < r_hi) rn = cand;
        }
        if (r_hi - r_lo <= 1e-13 * (1.0 + r_hi)) { *n_eval_out = n_eval; return rn; }
        r = rn;
    }
    *n_eval_out = n_eval;
    return r;
}

static int field_init(field_t *s, const double *d, const int32_t *F, int64_t nf, const double *area,
                      const double *g11, const double *g12, const double *g22, double width,
                      double *dmax_buf, int32_t *order_buf, int32_t *long_buf) {
    s->d = d; s->F = F; s->area = area; s->g11 = g11; s->g12 = g12; s->g22 = g22;
    s->width = width; s->dmax = dmax_buf; s->order = order_buf; s->lng = long_buf;
    return build_buckets(d, F, nf, area, width, dmax_buf, order_buf, long_buf, &s->b);
}

static void field_free(field_t *s) { free(s->b.ptr); free(s->b.prefix); }

/* lean_geometry.py:302-340 -- radii + perimeters at sorted targets, then log-spaced samples. */
int64_t oracle_source_geometry(const double *d, const int32_t *F, int64_t nf, const double *area,
                               const double *g11, const double *g12, const double *g22, double width,
                               const double *targets, int64_t nt, const double *fracs, int64_t m,
                               double rtol, int64_t max_iter, double *dmax_buf, int32_t *order_buf,
                               int32_t *long_buf, double *radii, double *perim, double *extra_r,
                               double *extra_a) {
    field_t s;
    if (field_init(&s, d, F, nf, area, g11, g12, g22, width, dmax_buf, order_buf, long_buf)) return -1;
    int64_t n_eval = 0, k;
    for (int64_t i = 0; i < nt; ++i) {
        double r = solve_radius(&s, targets[i], rtol, (int)max_iter, &k);
        n_eval += k;
        radii[i] = r;
        perim[i] = (r == r) ? perimeter_at(&s, r) : NAN;
    }
    for (int64_t i = 0; i + 1 < nt; ++i) {
        double r0 = radii[i], r1 = radii[i + 1];
        for (int64_t j = 0; j < m; ++j) {
            int64_t idx = i * m + j;
            if (r0 == r0 && r1 == r1 && r0 > 0.0 && r1 > r0) {
                double rr = exp(log(r0) + fracs[j] * (log(r1) - log(r0)));
                double a, da;
                area_at(&s, rr, &a, &da);
                extra_r[idx] = rr; extra_a[idx] = a;
                n_eval++;
            } else {
                extra_r[idx] = NAN; extra_a[idx] = NAN;
            }
        }
    }
    field_free(&s);
    return n_eval;
}

/* Single evaluations for the unit tests (lean_geometry.py:183-299). mode: 0 area, 1 dA/dr,
 * 2 perimeter, 3 radius for target r. Returns NaN on allocation failure. */
double oracle_field_eval(int mode, double r, const double *d, const int32_t *F, int64_t nf,
                         const double *area, const double *g11, const double *g12, const double *g22,
                         double width, double rtol, int64_t max_iter, double *dmax_buf,
                         int32_t *order_buf, int32_t *long_buf, int64_t *n_long_out) {
    field_t s;
    if (field_init(&s, d, F, nf, area, g11, g12, g22, width, dmax_buf, order_buf, long_buf)) return NAN;
    double out = NAN, A, dA;
    int64_t k;
    if (mode == 0 || mode == 1) { area_at(&s, r, &A, &dA); out = mode == 0 ? A : dA; }
    else if (mode == 2) out = perimeter_at(&s, r);
    else if (mode == 3) out = solve_radius(&s, r, rtol, (int)max_iter, &k);
    if (n_long_out) *n_long_out = s.b.n_long;
    field_free(&s);
    return out;
}

/* fastcw_lean.py:416-442 -- out[v, j] = sum_f A_f (X_f . gradB_v), X_f = -grad u / |grad u|.
 * u and out are (nv, k) row-major; faces are visited in order, as in the reference. */
void oracle_normalized_divergence(const double *u, int64_t nv, int64_t k, const int32_t *F, int64_t nf,
                                  const double *area, const double *gb0, const double *gb1,
                                  const double *gb2, double *out) {
    memset(out, 0, (size_t)(nv * k) * sizeof(double));
    for (int64_t f = 0; f < nf; ++f) {
        int64_t i0 = F[3 * f], i1 = F[3 * f + 1], i2 = F[3 * f + 2];
        double A = area[f];
        const double *b0 = gb0 + 3 * f, *b1 = gb1 + 3 * f, *b2 = gb2 + 3 * f;
        for (int64_t j = 0; j < k; ++j) {
            double du1 = u[i1 * k + j] - u[i0 * k + j];
            double du2 = u[i2 * k + j] - u[i0 * k + j];
            double gx = du1 * b1[0] + du2 * b2[0];
            double gy = du1 * b1[1] + du2 * b2[1];
            double gz = du1 * b1[2] + du2 * b2[2];
            double nn = sqrt(gx * gx + gy * gy + gz * gz);
            if (!(nn > 1e-300)) continue;
            double s = -A / nn;
            out[i0 * k + j] += s * (gx * b0[0] + gy * b0[1] + gz * b0[2]);
            out[i1 * k + j] += s * (gx * b1[0] + gy * b1[1] + gz * b1[2]);
            out[i2 * k + j] += s * (gx * b2[0] + gy * b2[1] + gz * b2[2]);
        }
    }
}
