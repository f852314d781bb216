// Per-source (radius, area) sample assembly on the metric records.
//
// For each healthy source: the finite solved radii paired with their target
// areas, then the finite supplementary samples, less those whose disc would
// lose more than `cap` of its area to a straight boundary at the source's
// float32 distance to boundary; stably sorted by radius, with radii within
// max(1e-12, 1e-9 * span) of their predecessor dropped; stored as float32.
// Flagged fields get no samples. Restates core_analysis.py:1599-1611 with
// boundary_area_loss_fraction (:759-777) and _clean_vertex_samples (:1424-1439).
//
// One warp per source: the candidate pairs are compacted into shared memory in
// list order, each lane ranks its pairs (stable: ties keep list order), and the
// sorted run is filtered and compacted into the output row.
#include <math.h>

#include "kernels.cuh"

namespace fcw {

namespace {

constexpr int kWarps = 4;  // sources per CTA

// Disc-area fraction clipped by a straight boundary at distance d (NaN for r
// not finite or <= 0). Explicitly rounded operations: no contraction into FMAs.
__device__ __forceinline__ double loss_fraction(double r, double d) {
    if (!isfinite(r) || r <= 0.0) return __longlong_as_double(0x7ff8000000000000LL);
    if (!isfinite(d)) return 0.0;
    if (d >= r) return 0.0;
    const double x = fmin(1.0, fmax(0.0, __ddiv_rn(d, r)));
    const double s = sqrt(fmax(0.0, __dsub_rn(1.0, __dmul_rn(x, x))));
    return __ddiv_rn(__dsub_rn(acos(x), __dmul_rn(x, s)), 3.141592653589793);
}

__global__ void __launch_bounds__(32 * kWarps) k_assemble_samples(SampleArgs a) {
    __shared__ double cr[kWarps][kMaxSamples], ca[kWarps][kMaxSamples];  // candidates, list order
    __shared__ double sr[kWarps][kMaxSamples], sa[kWarps][kMaxSamples];  // sorted
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t k = (int64_t)blockIdx.x * kWarps + w;
    if (k >= a.n) return;
    const double* o = a.records + k * a.stride;
    const int nt = a.n_targets, ne = nt > 0 ? (nt - 1) * a.n_between : 0, np_ = nt + ne;
    float* ro = a.radii_out + k * a.capacity;
    float* ao = a.areas_out + k * a.capacity;
    if (o[5] != 0.0) {  // flagged field
        if (lane == 0) a.count_out[k] = 0;
        return;
    }
    const double db = (double)(float)o[2];  // the analysis stores the distance to boundary as float32
    const bool capped = !isnan(a.cap);
    const unsigned below = (1u << lane) - 1u;

    // candidates in the reference's list order: solved radii, then supplementary samples
    int n = 0;
    for (int base = 0; base < np_; base += 32) {
        const int j = base + lane;
        double r = 0.0, ar = 0.0;
        bool ok = false;
        if (j < nt) {
            r = o[7 + j];
            ar = a.targets[j];
            ok = isfinite(r);
        } else if (j < np_) {
            const int e = j - nt;
            r = o[7 + 2 * nt + e];
            ar = o[7 + 2 * nt + ne + e];
            ok = isfinite(r) && isfinite(ar);
            if (ok && capped && loss_fraction(r, db) > a.cap) ok = false;
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const int p = n + __popc(m & below);
            cr[w][p] = r;
            ca[w][p] = ar;
        }
        n += __popc(m);
    }
    __syncwarp();
    if (n == 0) {
        if (lane == 0) a.count_out[k] = 0;
        return;
    }
    // stable ranks
    for (int i = lane; i < n; i += 32) {
        const double ri = cr[w][i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double rj = cr[w][j];
            rank += (rj < ri || (rj == ri && j < i)) ? 1 : 0;
        }
        sr[w][rank] = ri;
        sa[w][rank] = ca[w][i];
    }
    __syncwarp();
    const double tol = fmax(1e-12, 1e-9 * __dsub_rn(sr[w][n - 1], sr[w][0]));
    int kept = 0;
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        const bool keep = i < n && (i == 0 || __dsub_rn(sr[w][i], sr[w][i - 1]) > tol);
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int p = kept + __popc(m & below);
            ro[p] = (float)sr[w][i];
            ao[p] = (float)sa[w][i];
        }
        kept += __popc(m);
    }
    if (lane == 0) a.count_out[k] = kept;
}

}  // namespace

void launch_assemble_samples(const SampleArgs& a, cudaStream_t st) {
    if (a.n <= 0) return;
    const int64_t blocks = (a.n + kWarps - 1) / kWarps;
    k_assemble_samples<<<(unsigned)blocks, 32 * kWarps, 0, st>>>(a);
}

}  // namespace fcw
