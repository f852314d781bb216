// Multi-right-hand-side supernodal triangular solves, one etree level per launch.
//
// Right-hand sides R and results B are n x K row-major (a vertex row holds K
// contiguous right-hand sides). The forward sweep reads R and writes the
// forward result into B; the backward sweep turns B into the solution in
// place. R is never written, because several CTAs of one supernode (its row
// chunks) each rebuild that supernode's right-hand side.
//
// A CTA owns one task of one supernode and one column tile of the right-hand
// sides (64 columns in FP64, 128 in FP32: a tile row is 512 bytes either way).
// Every row of a tile is a contiguous 512-byte segment of an n x K array, so
// all row traffic (right-hand sides, children's update rows, the ancestors'
// solution rows, results) moves as 16-byte cp.async copies or vector stores,
// and a CTA issues all the copies of a stage before it waits for any of them.
//
// Dense products run on shared-memory tiles. FP64 uses the FP64 tensor path
// (mma.sync m8n8k4: one instruction per 256 multiply-adds; each of the 8 warps
// owns 8 columns and walks the 8-row tiles the supernode needs). FP32 uses
// register tiles on the FMA pipes (a thread owns 4 rows x KT/16 columns in
// 16-byte column groups).
//
// The panels below the diagonal blocks hold Q_s = L_rs inv(L_ss) (formed once
// after the factorisation), so nothing waits for X_s:
//
// Forward (leaves -> root), multifrontal: supernode s forms
//   W   = b_s - the children's update rows that land on s's columns
//   X_s = inv(L_ss) W                                   (written to B)
//   U_s = Q_s W + the children's update rows that land on s's structure
// and leaves U_s (nr x K) for its parent. Children's rows are listed per front
// row in ascending child order and added in that order, so results are
// deterministic. A supernode with a long structure is split into 64-row tasks;
// each forms W and its own rows of U_s, and the first also X_s.
//
// Backward (root -> leaves): X_s = inv(L_ss)^T y_s - Q_s^T X_r, where X_r are
// the structure rows (ancestors, final; gathered two chunks in flight). Long
// structures are split over several CTAs (split-K); each writes a partial sum
// of Q_s^T X_r, and the CTA that arrives last (atomic ticket, no waiting) adds
// the partials in split order and finishes the supernode.
//
// Heat right-hand sides are columns of the identity: the forward sweep builds
// them from the source list, and only supernodes on a source's path to the
// root (`reach`, per supernode and 64-column tile) are solved; the others' forward results
// are zero.
#include <type_traits>

#include "kernels.cuh"
#include "sweep_rows.cuh"

namespace fcw {

namespace {

constexpr int PT = kMaxWidth;   // rows of a backward partial-sum slot (= widest supernode)
constexpr int RC = 32;          // structure rows per backward chunk
// Tiles are TR = 64 rows (any supernode); the backward sweep also has TR = 32
// for the levels whose supernodes are all at most 32 wide (the leaves), where
// smaller tiles and accumulators let three CTAs share an SM.

// Column tile of each precision when K allows it (512-byte rows).
template <typename T>
constexpr int wide_tile() { return sizeof(T) == 4 ? 128 : 64; }
// Most children's update rows a forward CTA stages per gather chunk. The
// launcher picks the count per level (SolveArgs::stage): none on levels without
// children, else what keeps two CTAs on an SM (three for FP32 with KT = 64).
template <typename T, int TR>
constexpr int stage_rows() { return sizeof(T) == 4 ? 112 : 80; }
template <typename T, int KT>
constexpr int stage_used() { return sizeof(T) == 8 ? 80 : (KT == 128 ? 88 : 96); }
// FP32 forward CTAs hold the inverse and the chunk's Q rows in two tiles (both
// products start as soon as W is formed); FP64 tiles are twice the size, so
// there the Q rows replace the inverse after X_s.
template <typename T>
constexpr bool separate_q() { return sizeof(T) == 4; }

// Shared-tile leading dimensions, chosen so that the product's operand reads
// are free of bank conflicts: FP64 tensor fragments read 8 rows x 4 depths
// (row stride TR + 4 doubles = 8 banks apart), FP32 register tiles read rows ty and
// ty+1 of a row-major A (odd stride) or adjacent columns of a transposed one.
template <typename T, int TR>
constexpr int ld_fwd_a() { return sizeof(T) == 8 ? TR + 4 : TR + 1; }  // forward inverse / panel, row-major
template <typename T, int TR>
constexpr int ld_bwd_a() { return sizeof(T) == 8 ? TR + 4 : TR; }      // backward panel / inverse, transposed
template <typename T, int KT>
constexpr int ld_rows() { return sizeof(T) == 8 ? KT + 4 : KT; }    // right-hand-side rows (W, X, C, gathers)
template <typename T>
constexpr int depth_pad() { return sizeof(T) == 8 ? 4 : 1; }        // product depth granularity


// ---------------------------------------------------------------------------
// Accumulators. C (rows < nrows, KT columns) += A B, with A either row-major
// (rows(): A[i*lda + k]) or transposed (cols(): A[k*lda + i]) and B row-major
// (Bm[k*ldb + c]). visit(nrows, f) hands each thread's results to
// f(row, col, T* v), v holding V adjacent columns.
// ---------------------------------------------------------------------------

// V adjacent elements (8 or 16 bytes, aligned) through L2 only: values other CTAs wrote.
template <typename T, int V>
__device__ __forceinline__ void ld_cg(const T* p, T* w) {
    if constexpr (V * sizeof(T) == 16 && sizeof(T) == 4) {
        const float4 x = __ldcg(reinterpret_cast<const float4*>(p));
        w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
    } else if constexpr (V * sizeof(T) == 16) {
        const double2 x = __ldcg(reinterpret_cast<const double2*>(p));
        w[0] = x.x; w[1] = x.y;
    } else {
        static_assert(V == 2 && sizeof(T) == 4, "8-byte groups are float pairs");
        const float2 x = __ldcg(reinterpret_cast<const float2*>(p));
        w[0] = x.x; w[1] = x.y;
    }
}

// Calls f(std::integral_constant<int, m>) with m = min(n, N), for n >= 1: the row
// blocks a product needs, as a compile-time count.
template <int N, class F>
__device__ __forceinline__ void upto(int n, F&& f) {
    if constexpr (N > 1) {
        if (n < N) {
            upto<N - 1>(n, f);
            return;
        }
    }
    f(std::integral_constant<int, N>{});
}

// FP32 register tiles: thread (ty, tx) owns rows ty + 16a (a < NA) and 16-byte
// column groups at vec*tx + 16*vec*h.
template <typename T, int KT, int NA>
struct AccScalar {
    static constexpr int NB = KT / 16, G = vec<T>(), V = G;
    T c[NA][NB];

    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int b = 0; b < NB; ++b) c[a][b] = T(0);
    }
    __device__ __forceinline__ void negate() {
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int b = 0; b < NB; ++b) c[a][b] = -c[a][b];
    }

    template <int MA>
    __device__ __forceinline__ void rows_n(const T* A, int lda, const T* Bm, int ldb, int depth) {
        const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
        const T* ap = A + ty * lda;
        const T* bp = Bm + G * tx;
        for (int j = 0; j < depth; ++j) {
            T w[NB];
#pragma unroll
            for (int h = 0; h < NB / G; ++h) ldv(bp + j * ldb + 16 * G * h, &w[G * h]);
#pragma unroll
            for (int a = 0; a < MA; ++a) {
                const T l = ap[16 * a * lda + j];
#pragma unroll
                for (int b = 0; b < NB; ++b) c[a][b] += l * w[b];
            }
        }
    }

    template <int MA>
    __device__ __forceinline__ void cols_n(const T* A, int lda, const T* Bm, int ldb, int depth) {
        const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
        const T* bp = Bm + G * tx;
        for (int j = 0; j < depth; ++j) {
            T w[NB], l[MA];
#pragma unroll
            for (int h = 0; h < NB / G; ++h) ldv(bp + j * ldb + 16 * G * h, &w[G * h]);
#pragma unroll
            for (int a = 0; a < MA; ++a) l[a] = A[j * lda + ty + 16 * a];
#pragma unroll
            for (int a = 0; a < MA; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) c[a][b] += l[a] * w[b];
        }
    }

    // A lower triangular (row-major, zeros above the diagonal): depth block q of 16 reaches
    // only the row blocks a >= q; the skipped products are exact zeros.
    template <int MA>
    __device__ __forceinline__ void rows_lower_n(const T* A, int lda, const T* Bm, int ldb, int depth) {
        const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
        const T* ap = A + ty * lda;
        const T* bp = Bm + G * tx;
#pragma unroll
        for (int q = 0; q < MA; ++q) {
            const int j1 = min(depth, 16 * q + 16);
            for (int j = 16 * q; j < j1; ++j) {
                T w[NB];
#pragma unroll
                for (int h = 0; h < NB / G; ++h) ldv(bp + j * ldb + 16 * G * h, &w[G * h]);
#pragma unroll
                for (int a = q; a < MA; ++a) {
                    const T l = ap[16 * a * lda + j];
#pragma unroll
                    for (int b = 0; b < NB; ++b) c[a][b] += l * w[b];
                }
            }
        }
    }

    // A read transposed (A[k*lda + i]) from a lower-triangular block: row i needs depth
    // k >= i, so depth block q reaches only the row blocks a <= q.
    template <int MA>
    __device__ __forceinline__ void cols_upper_n(const T* A, int lda, const T* Bm, int ldb, int depth) {
        const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
        const T* bp = Bm + G * tx;
#pragma unroll
        for (int q = 0; q < MA; ++q) {
            const int j1 = min(depth, 16 * q + 16);
            for (int j = 16 * q; j < j1; ++j) {
                T w[NB], l[MA];
#pragma unroll
                for (int h = 0; h < NB / G; ++h) ldv(bp + j * ldb + 16 * G * h, &w[G * h]);
#pragma unroll
                for (int a = 0; a <= q; ++a) l[a] = A[j * lda + ty + 16 * a];
#pragma unroll
                for (int a = 0; a <= q; ++a)
#pragma unroll
                    for (int b = 0; b < NB; ++b) c[a][b] += l[a] * w[b];
            }
        }
    }

    // only the 16-row blocks holding one of the first nrows rows are computed
    __device__ __forceinline__ void rows(const T* A, int lda, const T* Bm, int ldb, int depth, int nrows) {
        const int na = (nrows + 15) >> 4;
        if (na > 0) upto<NA>(na, [&](auto m) { rows_n<decltype(m)::value>(A, lda, Bm, ldb, depth); });
    }
    __device__ __forceinline__ void cols(const T* A, int lda, const T* Bm, int ldb, int depth, int nrows) {
        const int na = (nrows + 15) >> 4;
        if (na > 0) upto<NA>(na, [&](auto m) { cols_n<decltype(m)::value>(A, lda, Bm, ldb, depth); });
    }
    // square triangular products (depth <= 16 * row blocks)
    __device__ __forceinline__ void rows_lower(const T* A, int lda, const T* Bm, int ldb, int depth, int nrows) {
        const int na = (nrows + 15) >> 4;
        if (na > 0) upto<NA>(na, [&](auto m) { rows_lower_n<decltype(m)::value>(A, lda, Bm, ldb, depth); });
    }
    __device__ __forceinline__ void cols_upper(const T* A, int lda, const T* Bm, int ldb, int depth, int nrows) {
        const int na = (nrows + 15) >> 4;
        if (na > 0) upto<NA>(na, [&](auto m) { cols_upper_n<decltype(m)::value>(A, lda, Bm, ldb, depth); });
    }

    template <class F>
    __device__ __forceinline__ void visit(int nrows, F&& f) {
        const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const int t = ty + 16 * a;
            if (t < nrows)
#pragma unroll
                for (int h = 0; h < NB / G; ++h) f(t, G * tx + 16 * G * h, &c[a][G * h]);
        }
    }
};

// FP64 tensor tiles (KT = 64): warp w owns columns [8w, 8w+8) and the 8-row
// m8n8k4 tiles down to row 8*MT; lane (g = lane/4, t = lane%4) holds rows 8m+g,
// columns 8w+2t and 8w+2t+1. The depth must be a multiple of 4 with the padded
// depths zero in both operands.
template <int MT>
struct AccDmma {
    static constexpr int V = 2;
    double c[MT][2];

    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int m = 0; m < MT; ++m) c[m][0] = c[m][1] = 0.0;
    }
    __device__ __forceinline__ void negate() {
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            c[m][0] = -c[m][0];
            c[m][1] = -c[m][1];
        }
    }

    static __device__ __forceinline__ void mma(double (&d)[2], double a, double b) {
        asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
            : "+d"(d[0]), "+d"(d[1])
            : "d"(a), "d"(b));
    }

    template <int MM, bool TRANS>
    __device__ __forceinline__ void run(const double* A, int lda, const double* Bm, int ldb, int depth) {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, n0 = 8 * (threadIdx.x >> 5);
        const double* bp = Bm + t * ldb + n0 + g;
        for (int k = 0; k < depth; k += 4) {
            const double b = bp[k * ldb];
#pragma unroll
            for (int m = 0; m < MM; ++m) {
                const double a = TRANS ? A[(k + t) * lda + 8 * m + g] : A[(8 * m + g) * lda + k + t];
                mma(c[m], a, b);
            }
        }
    }

    // Triangular A (lower, zeros above the diagonal): depth steps [8q, 8q+8) reach the row
    // tiles m >= q (row-major: rows need k <= row) or m <= q (transposed: k >= row).
    template <int MM, bool TRANS>
    __device__ __forceinline__ void run_tri(const double* A, int lda, const double* Bm, int ldb, int depth) {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, n0 = 8 * (threadIdx.x >> 5);
        const double* bp = Bm + t * ldb + n0 + g;
#pragma unroll
        for (int q = 0; q < MM; ++q) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = 8 * q + 4 * h;
                if (k >= depth) break;
                const double b = bp[k * ldb];
#pragma unroll
                for (int m = TRANS ? 0 : q; m < (TRANS ? q + 1 : MM); ++m) {
                    const double a = TRANS ? A[(k + t) * lda + 8 * m + g] : A[(8 * m + g) * lda + k + t];
                    mma(c[m], a, b);
                }
            }
        }
    }
    __device__ __forceinline__ void rows_lower(const double* A, int lda, const double* Bm, int ldb, int depth,
                                               int nrows) {
        const int nm = (nrows + 7) >> 3;
        if (nm > 0) upto<MT>(nm, [&](auto m) { run_tri<decltype(m)::value, false>(A, lda, Bm, ldb, depth); });
    }
    __device__ __forceinline__ void cols_upper(const double* A, int lda, const double* Bm, int ldb, int depth,
                                               int nrows) {
        const int nm = (nrows + 7) >> 3;
        if (nm > 0) upto<MT>(nm, [&](auto m) { run_tri<decltype(m)::value, true>(A, lda, Bm, ldb, depth); });
    }

    template <bool TRANS>
    __device__ __forceinline__ void dispatch(const double* A, int lda, const double* Bm, int ldb, int depth,
                                             int nrows) {
        const int nm = (nrows + 7) >> 3;
        if (nm > 0) upto<MT>(nm, [&](auto m) { run<decltype(m)::value, TRANS>(A, lda, Bm, ldb, depth); });
    }
    __device__ __forceinline__ void rows(const double* A, int lda, const double* Bm, int ldb, int depth,
                                         int nrows) {
        dispatch<false>(A, lda, Bm, ldb, depth, nrows);
    }
    __device__ __forceinline__ void cols(const double* A, int lda, const double* Bm, int ldb, int depth,
                                         int nrows) {
        dispatch<true>(A, lda, Bm, ldb, depth, nrows);
    }

    template <class F>
    __device__ __forceinline__ void visit(int nrows, F&& f) {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, n0 = 8 * (threadIdx.x >> 5);
#pragma unroll
        for (int m = 0; m < MT; ++m)
            if (8 * m + g < nrows) f(8 * m + g, n0 + 2 * t, c[m]);
    }
};

template <typename T, int KT, int TR>
struct AccSel {
    using type = AccScalar<T, KT, TR / 16>;
};
template <int TR>
struct AccSel<double, 64, TR> {
    using type = AccDmma<TR / 8>;
};
template <typename T, int KT, int TR>
using Acc = typename AccSel<T, KT, TR>::type;

// Zero rows [r0, r1) x columns [0, ncols) of a shared tile (padding of a product's depth).
template <typename T>
__device__ __forceinline__ void zero_rows(T* D, int ld, int r0, int r1, int ncols) {
    for (int e = threadIdx.x; e < (r1 - r0) * ncols; e += NT) {
        const int r = e / ncols, c = e - r * ncols;
        D[(r0 + r) * ld + c] = T(0);
    }
}
// Zero columns [c0, c1) of rows [0, nrows).
template <typename T>
__device__ __forceinline__ void zero_cols(T* D, int ld, int nrows, int c0, int c1) {
    const int w = c1 - c0;
    for (int e = threadIdx.x; e < nrows * w; e += NT) {
        const int r = e / w, c = e - r * w;
        D[r * ld + c0 + c] = T(0);
    }
}


template <typename T, int KT, int TR>
__global__ void __launch_bounds__(NT, 3) k_fwd(SolveArgs<T> a, int32_t t0) {
    constexpr int VPR = KT / vec<T>(), LW = ld_rows<T, KT>(), LA = ld_fwd_a<T, TR>(), DP = depth_pad<T>();
    using AccT = Acc<T, KT, TR>;
    constexpr bool kSepQ = separate_q<T>();
    extern __shared__ __align__(16) unsigned char smraw[];
    T* Wt = reinterpret_cast<T*>(smraw);   // TR x LW: W, then this chunk's update rows
    T* Li = Wt + TR * LW;                   // TR x LA: inverse diagonal block (first chunk)
    T* Pn = kSepQ ? Li + TR * LA : Li;      // TR x LA: this chunk's rows of Q_s
    T* St = Pn + TR * LA;                   // a.stage x KT: children's update rows
    __shared__ int grs[TR + 1];
    __shared__ unsigned char live[stage_rows<T, TR>()];
    static_assert(sizeof(T) == 4 || KT == kReachCols, "the heat solve's reach tiles are its column tiles");
    const int2 task = a.tasks[t0 + blockIdx.x];
    const int s = task.x, chunk = task.y;
    if (a.reach && !a.reach[(int64_t)s * a.reach_tiles + blockIdx.y]) return;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x;
    const int K = a.K, k0 = blockIdx.y * KT;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], nr = m - ns;
    const int nsp = (ns + DP - 1) / DP * DP;  // product depth
    const int64_t fb = p.sn_rowptr[s];
    const int q0 = chunk * TR;
    const int nq = nr > 0 ? min(TR, nr - q0) : 0;
    const bool want_x = chunk == 0;
    const bool q_early = nq > 0 && (kSepQ || !want_x);  // Q rows come with the first copies
    const T* Q = a.val + p.sn_valptr[s] + (int64_t)(ns + q0) * ns;

    // the inverse block, this chunk's rows of Q_s, the right-hand side rows and
    // the first children's rows are in flight together (identity right-hand
    // sides are built in place)
    if (want_x) {
        const T* inv = a.inv + p.sn_invptr[s];
        for (int e = tid; e < ns * ns; e += NT) {
            const int i = e / ns, j = e - i * ns;
            copy_async(&Li[i * LA + j], inv + e);
        }
    }
    if (q_early)
        for (int e = tid; e < nq * ns; e += NT) {
            const int r = e / ns, j = e - r * ns;
            copy_async(&Pn[r * LA + j], Q + e);
        }
    if (a.delta_src) {
        for (int e = tid; e < ns * KT; e += NT) {
            const int f = e / KT, c = e - f * KT;
            Wt[f * LW + c] = (a.delta_src[k0 + c] == c0 + f) ? T(1) : T(0);
        }
    } else {
        for (int i = tid; i < ns * VPR; i += NT) {
            const int f = i / VPR, v = i - f * VPR;
            copy16_async(Wt + f * LW + v * vec<T>(), a.R + (int64_t)(c0 + f) * K + k0 + v * vec<T>());
        }
    }
    if (nsp > ns) {  // padded depth: zero in both operands
        zero_rows(Wt, LW, ns, nsp, KT);
        if (want_x) zero_cols(Li, LA, ns, ns, nsp);
        if (q_early) zero_cols(Pn, LA, nq, ns, nsp);
    }
    const GatherRange g1 = gather_open(a, fb, 0, ns, grs);
    if (g1.E > 0) gather_issue<T, KT, TR>(a, g1, 0, k0, St, live);
    copy_async_commit();
    gather_finish<T, KT, TR, true>(a, g1, k0, Wt, LW, ns, St, live, grs);

    // the children's rows of this chunk's update rows arrive while X_s and U_s are formed
    GatherRange g2{0, 0};
    if (nq > 0) {
        g2 = gather_open(a, fb, ns + q0, nq, grs);
        if (g2.E > 0) gather_issue<T, KT, TR>(a, g2, 0, k0, St, live);
        copy_async_commit();
    }
    AccT acc;
    if (want_x) {  // X = inv(L_ss) W, straight from the registers to B
        acc.zero();
        acc.rows_lower(Li, LA, Wt, LW, nsp, ns);
        T* xb = a.B + (int64_t)c0 * K + k0;
        acc.visit(ns, [&](int r, int c, T* v) { st_n<T, AccT::V>(xb + (int64_t)r * K + c, v); });
    }
    if (nq <= 0) return;
    if (!q_early) {  // one shared tile: the Q rows take the inverse's place now
        __syncthreads();
        for (int e = tid; e < nq * ns; e += NT) {
            const int r = e / ns, j = e - r * ns;
            copy_async(&Pn[r * LA + j], Q + e);
        }
        if (nsp > ns) zero_cols(Pn, LA, nq, ns, nsp);
        copy_async_commit();
        copy_async_wait();
        __syncthreads();
    }
    // U_s rows of this chunk = Q_s W + the children's rows landing on them
    acc.zero();
    acc.rows(Pn, LA, Wt, LW, nsp, nq);
    __syncthreads();  // every thread is done reading W
    acc.visit(nq, [&](int r, int c, T* v) { st_n<T, AccT::V>(Wt + r * LW + c, v); });
    gather_finish<T, KT, TR, false>(a, g2, k0, Wt, LW, nq, St, live, grs);
    tile_rows_to_global<T, KT>(a.U + (a.uoff[s] + q0) * (int64_t)K + k0, K, Wt, LW, nq);
}

template <typename T, int KT, int TR>
__global__ void __launch_bounds__(NT, 3) k_bwd(SolveArgs<T> a, int32_t t0) {
    constexpr int VPR = KT / vec<T>(), LW = ld_rows<T, KT>(), LA = ld_bwd_a<T, TR>(), DP = depth_pad<T>();
    constexpr int PS = RC * LA, XS = RC * LW;  // one chunk buffer: panel rows, gathered solution rows
    static_assert(2 * (PS + XS) >= TR * LW + TR * LA, "the finishing tiles alias the chunk buffers");
    static_assert(sizeof(T) == 4 || KT == kReachCols, "the heat solve's reach tiles are its column tiles");
    using AccT = Acc<T, KT, TR>;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* buf = reinterpret_cast<T*>(smraw);
    T* Ys = buf;             // TR x LW: y_s, after the gather
    T* Ms = buf + TR * LW;   // TR x LA inverse diagonal block, after the gather
    __shared__ int last_arrival;
    const int2 task = a.tasks[t0 + blockIdx.x];
    const int s = task.x, split = task.y;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x;
    const int K = a.K, k0 = blockIdx.y * KT;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], nr = m - ns;
    const int nsp = (ns + DP - 1) / DP * DP;
    const int nspl = a.nsplit[s];
    const int q0 = split * kSplitRows, q1 = min(nr, q0 + kSplitRows);
    const T* P = a.val + p.sn_valptr[s];
    const int32_t* rows = p.rows + p.sn_rowptr[s];

    // chunk ci of the split's structure rows into buffer ci & 1
    auto issue = [&](int ci) {
        const int qq = q0 + ci * RC, nc = min(RC, q1 - qq), ncp = (nc + DP - 1) / DP * DP;
        T* Ps = buf + (ci & 1) * (PS + XS);
        T* Xg = Ps + PS;
        for (int e = tid; e < nc * ns; e += NT) {
            const int r = e / ns, j = e - r * ns;
            copy_async(&Ps[r * LA + j], P + (int64_t)(ns + qq + r) * ns + j);
        }
        for (int i = tid; i < nc * VPR; i += NT) {
            const int r = i / VPR, v = i - r * VPR;
            copy16_async(Xg + r * LW + v * vec<T>(), a.B + (int64_t)rows[ns + qq + r] * K + k0 + v * vec<T>());
        }
        if (ncp > nc) {
            zero_rows(Ps, LA, nc, ncp, TR);
            zero_rows(Xg, LW, nc, ncp, KT);
        }
        copy_async_commit();
    };
    AccT acc;
    acc.zero();
    const int nchunks = q1 > q0 ? (q1 - q0 + RC - 1) / RC : 0;
    if (nchunks > 0) issue(0);
    for (int ci = 0; ci < nchunks; ++ci) {
        if (ci + 1 < nchunks) {
            issue(ci + 1);
            copy_async_wait_prev();
        } else {
            copy_async_wait();
        }
        __syncthreads();
        const T* Ps = buf + (ci & 1) * (PS + XS);
        const int nc = min(RC, q1 - q0 - ci * RC);
        acc.cols(Ps, LA, Ps + PS, LW, (nc + DP - 1) / DP * DP, ns);
        __syncthreads();
    }

    const bool zero_y = a.reach && !a.reach[(int64_t)s * a.reach_tiles + blockIdx.y];
    if (nspl > 1) {
        T* part = a.part + a.poff[s] * (int64_t)PT * K + k0;
        T* mine = part + (int64_t)split * PT * K;
        acc.visit(ns, [&](int r, int c, T* v) { st_n<T, AccT::V>(mine + (int64_t)r * K + c, v); });
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            const int ticket = atomicAdd(&a.counters[(int64_t)s * a.ktiles + blockIdx.y], 1);
            last_arrival = ticket == nspl - 1;
        }
        __syncthreads();
        if (!last_arrival) return;
        __threadfence();
        // the partial sums in split order; four splits' vectors are loaded before any is added,
        // so the loads overlap instead of waiting on one another
        acc.visit(ns, [&](int r, int c, T* v) {
            constexpr int V = AccT::V;
            const T* base = part + (int64_t)r * K + c;
            const int64_t ss = (int64_t)PT * K;  // one split's slot
            T sum[V];
#pragma unroll
            for (int q = 0; q < V; ++q) sum[q] = T(0);
            int sp = 0;
            for (; sp + 4 <= nspl; sp += 4) {
                T w[4][V];
#pragma unroll
                for (int u = 0; u < 4; ++u) ld_cg<T, V>(base + (sp + u) * ss, w[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int q = 0; q < V; ++q) sum[q] += w[u][q];
            }
            for (; sp < nspl; ++sp) {
                T w[V];
                ld_cg<T, V>(base + sp * ss, w);
#pragma unroll
                for (int q = 0; q < V; ++q) sum[q] += w[q];
            }
#pragma unroll
            for (int q = 0; q < V; ++q) v[q] = sum[q];
        });
        if (tid == 0) a.counters[(int64_t)s * a.ktiles + blockIdx.y] = 0;
    }
    // X_s = inv(L_ss)^T y_s - Q_s^T X_r (y_s = 0 off the sources' paths)
    acc.negate();
    if (!zero_y) {
        const T* inv = a.inv + p.sn_invptr[s];
        for (int e = tid; e < ns * ns; e += NT) {
            const int i = e / ns, j = e - i * ns;
            copy_async(&Ms[i * LA + j], inv + e);
        }
        for (int i = tid; i < ns * VPR; i += NT) {
            const int r = i / VPR, v = i - r * VPR;
            copy16_async(Ys + r * LW + v * vec<T>(), a.B + (int64_t)(c0 + r) * K + k0 + v * vec<T>());
        }
        copy_async_commit();
        if (nsp > ns) {
            zero_rows(Ms, LA, ns, nsp, TR);
            zero_rows(Ys, LW, ns, nsp, KT);
        }
        copy_async_wait();
        __syncthreads();
        acc.cols_upper(Ms, LA, Ys, LW, nsp, ns);
    }
    T* out = a.B + (int64_t)c0 * K + k0;
    acc.visit(ns, [&](int r, int c, T* v) { st_n<T, AccT::V>(out + (int64_t)r * K + c, v); });
}

// reach[s * tiles + t]: some source of column tile t (kReachCols columns) has supernode s on
// its path to the root.
__global__ void k_reach(const int32_t* __restrict__ col_sn, const int32_t* __restrict__ parent,
                        const int32_t* __restrict__ src, int32_t K, int32_t nlevels, int32_t tiles,
                        uint8_t* __restrict__ reach) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const int s0 = src[k];
    if (s0 < 0) return;
    const int t = k / kReachCols;
    int s = col_sn[s0];
    // the parent chain is strictly increasing and at most nlevels long
    for (int it = 0; s >= 0 && it <= nlevels; ++it) {
        reach[(int64_t)s * tiles + t] = 1;
        s = parent[s];
    }
}

template <typename T, int KT, int TR>
constexpr size_t fwd_smem(int stage = stage_rows<T, TR>()) {
    return (size_t)(TR * ld_rows<T, KT>() + (separate_q<T>() ? 2 : 1) * TR * ld_fwd_a<T, TR>() + stage * KT) *
           sizeof(T);
}
template <typename T, int KT, int TR>
constexpr size_t bwd_smem() {
    return (size_t)2 * (RC * ld_bwd_a<T, TR>() + RC * ld_rows<T, KT>()) * sizeof(T);
}

// forward sweeps run 64-row tiles; backward sweeps 64- or 32-row tiles
template <typename T, int KT>
cudaError_t set_smem() {
    cudaError_t e = cudaFuncSetAttribute(k_fwd<T, KT, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fwd_smem<T, KT, 64>());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_bwd<T, KT, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bwd_smem<T, KT, 64>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_bwd<T, KT, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bwd_smem<T, KT, 32>());
}

template <typename T, int KT, int TR>
void fwd_launch(const SolveArgs<T>& args, int32_t t0, int32_t ntasks, bool gathers, cudaStream_t st) {
    SolveArgs<T> a = args;
    a.stage = gathers ? stage_used<T, KT>() : 0;
    k_fwd<T, KT, TR><<<dim3(ntasks, a.K / KT), NT, fwd_smem<T, KT, TR>(a.stage), st>>>(a, t0);
}
template <typename T, int KT, int TR>
void bwd_launch(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, cudaStream_t st) {
    k_bwd<T, KT, TR><<<dim3(ntasks, a.K / KT), NT, bwd_smem<T, KT, TR>(), st>>>(a, t0);
}

}  // namespace

cudaError_t configure_solve_kernels() {
    cudaError_t e;
    if ((e = set_smem<double, 64>())) return e;
    if ((e = set_smem<float, 64>())) return e;
    return set_smem<float, 128>();
}

template <typename T>
void launch_fwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, bool gathers, cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    constexpr int W = wide_tile<T>();
    if (W != 64 && a.K % W == 0)
        fwd_launch<T, W, 64>(a, t0, ntasks, gathers, st);
    else
        fwd_launch<T, 64, 64>(a, t0, ntasks, gathers, st);
}

template <typename T>
void launch_bwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, int32_t tile_rows, cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    constexpr int W = wide_tile<T>();
    const bool wide = W != 64 && a.K % W == 0;
    if (tile_rows == 32)
        wide ? bwd_launch<T, W, 32>(a, t0, ntasks, st) : bwd_launch<T, 64, 32>(a, t0, ntasks, st);
    else
        wide ? bwd_launch<T, W, 64>(a, t0, ntasks, st) : bwd_launch<T, 64, 64>(a, t0, ntasks, st);
}

void launch_reach(const DevPlan& p, const int32_t* src, int32_t K, uint8_t* reach, cudaStream_t st) {
    const int32_t tiles = K / kReachCols;
    cudaMemsetAsync(reach, 0, (size_t)p.nsuper * tiles, st);
    k_reach<<<(K + 127) / 128, 128, 0, st>>>(p.col_sn, p.sn_parent, src, K, p.nlevels, tiles, reach);
}

template void launch_fwd_level<double>(const SolveArgs<double>&, int32_t, int32_t, bool, cudaStream_t);
template void launch_fwd_level<float>(const SolveArgs<float>&, int32_t, int32_t, bool, cudaStream_t);
template void launch_bwd_level<double>(const SolveArgs<double>&, int32_t, int32_t, int32_t, cudaStream_t);
template void launch_bwd_level<float>(const SolveArgs<float>&, int32_t, int32_t, int32_t, cudaStream_t);

}  // namespace fcw
