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
// The dense work is register-tiled products staged in shared memory (256
// threads; a thread owns 4 rows x KT/16 columns in 16-byte groups of
// adjacent columns, read as vectors).
//
// Forward (leaves -> root), multifrontal: supernode s forms
//   W   = b_s - the children's update rows that land on s's columns
//   X_s = inv(L_ss) W                                   (written to B)
//   U_s = L_rs X_s + the children's update rows that land on s's structure
// and leaves U_s (nr x K) for its parent. Children's rows are listed per front
// row in ascending child order and added in that order, so results are
// deterministic. A supernode with a long structure is split into 64-row tasks
// that each recompute X_s (cheap) and write their own rows of U_s.
//
// Backward (root -> leaves): C = y_s - L_rs^T X_r (gather of the structure
// rows, which belong to ancestors and are final; two chunks in flight),
// X_s = inv(L_ss)^T C. Long structures are split over several CTAs (split-K);
// each writes a partial sum, and the CTA that arrives last (atomic ticket, no
// waiting) adds the partials in split order and finishes the supernode.
//
// Heat right-hand sides are columns of the identity: the forward sweep builds
// them from the source list, and only supernodes on a source's path to the
// root (`reach`) are solved; the others' forward results are zero.
#include "kernels.cuh"

namespace fcw {

namespace {

constexpr int NT = 256;         // threads per CTA
constexpr int TR = kMaxWidth;   // rows of a tile (= widest supernode)
constexpr int LDP = TR + 1;     // leading dimension of the forward inverse / panel tiles
constexpr int RC = 32;          // structure rows per backward chunk

// Column tile of each precision when K allows it (512-byte rows).
template <typename T>
constexpr int wide_tile() { return sizeof(T) == 4 ? 128 : 64; }
// Children's update rows staged per forward gather chunk (two CTAs per SM).
template <typename T>
constexpr int stage_rows() { return sizeof(T) == 4 ? 112 : 88; }
template <typename T>
constexpr int vec() { return 16 / (int)sizeof(T); }  // elements per 16-byte vector

// One 16-byte vector (vec<T>() elements) between memory and registers.
template <typename T>
__device__ __forceinline__ void ldv(const T* p, T* w) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else {
        const double2 v = *reinterpret_cast<const double2*>(p);
        w[0] = v.x; w[1] = v.y;
    }
}

template <typename T>
__device__ __forceinline__ void stv(T* p, const T* w) {
    if constexpr (sizeof(T) == 4)
        *reinterpret_cast<float4*>(p) = make_float4(w[0], w[1], w[2], w[3]);
    else
        *reinterpret_cast<double2*>(p) = make_double2(w[0], w[1]);
}

// Column of a thread's b-th accumulator: 16-byte groups of adjacent columns,
// 16 groups apart, so a half-warp reads 256 contiguous bytes per vector load.
template <typename T>
__device__ __forceinline__ int col_of(int tx, int b) {
    constexpr int G = vec<T>();
    return G * tx + (b % G) + 16 * G * (b / G);
}

template <typename T, int NB>
__device__ __forceinline__ void zero(T (&acc)[4][NB]) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[a][b] = T(0);
}

// acc[a][b] += sum_{j<depth} A[(ty+16a)*lda + j] * Bm[j*ldb + col_of(tx,b)], a < NA
template <typename T, int NB, int NA>
__device__ __forceinline__ void mma_rows_n(T (&acc)[4][NB], const T* A, int lda, const T* Bm, int ldb, int depth,
                                           int ty, int tx) {
    constexpr int G = vec<T>();
    const T* ap = A + ty * lda;
    const T* bp = Bm + G * tx;
    for (int j = 0; j < depth; ++j) {
        T w[NB];
#pragma unroll
        for (int h = 0; h < NB / G; ++h) ldv(bp + j * ldb + 16 * G * h, &w[G * h]);
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const T l = ap[16 * a * lda + j];
#pragma unroll
            for (int b = 0; b < NB; ++b) acc[a][b] += l * w[b];
        }
    }
}

// acc[a][b] += sum_{j<depth} A[j*lda + ty+16a] * Bm[j*ldb + col_of(tx,b)], a < NA   (A transposed)
template <typename T, int NB, int NA>
__device__ __forceinline__ void mma_cols_n(T (&acc)[4][NB], const T* A, int lda, const T* Bm, int ldb, int depth,
                                           int ty, int tx) {
    constexpr int G = vec<T>();
    const T* bp = Bm + G * tx;
    for (int j = 0; j < depth; ++j) {
        T w[NB], l[NA];
#pragma unroll
        for (int h = 0; h < NB / G; ++h) ldv(bp + j * ldb + 16 * G * h, &w[G * h]);
#pragma unroll
        for (int a = 0; a < NA; ++a) l[a] = A[j * lda + ty + 16 * a];
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int b = 0; b < NB; ++b) acc[a][b] += l[a] * w[b];
    }
}

// Only the 16-row blocks that hold one of the first `nrows` rows are computed.
template <typename T, int NB>
__device__ __forceinline__ void mma_rows(T (&acc)[4][NB], const T* A, int lda, const T* Bm, int ldb, int depth,
                                         int nrows, int ty, int tx) {
    switch ((nrows + 15) >> 4) {
        case 0: break;
        case 1: mma_rows_n<T, NB, 1>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
        case 2: mma_rows_n<T, NB, 2>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
        case 3: mma_rows_n<T, NB, 3>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
        default: mma_rows_n<T, NB, 4>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
    }
}

template <typename T, int NB>
__device__ __forceinline__ void mma_cols(T (&acc)[4][NB], const T* A, int lda, const T* Bm, int ldb, int depth,
                                         int nrows, int ty, int tx) {
    switch ((nrows + 15) >> 4) {
        case 0: break;
        case 1: mma_cols_n<T, NB, 1>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
        case 2: mma_cols_n<T, NB, 2>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
        case 3: mma_cols_n<T, NB, 3>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
        default: mma_cols_n<T, NB, 4>(acc, A, lda, Bm, ldb, depth, ty, tx); break;
    }
}

// Rows ty+16a < nrows of acc into the row-major tile D (leading dimension ld).
template <typename T, int NB>
__device__ __forceinline__ void store_rows(T* D, int64_t ld, const T (&acc)[4][NB], int nrows, int ty, int tx) {
    constexpr int G = vec<T>();
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int t = ty + 16 * a;
        if (t < nrows)
#pragma unroll
            for (int h = 0; h < NB / G; ++h) stv(D + t * ld + G * tx + 16 * G * h, &acc[a][G * h]);
    }
}

// Asynchronous global -> shared copies (cp.async): single elements through L1,
// 16-byte vectors around it.
template <typename T>
__device__ __forceinline__ void copy_async(T* smem, const T* gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy16_async(void* smem, const void* gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void copy_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Rows [0, nrows) of a KT-wide shared tile to an n x K array (g = first row, first column).
template <typename T, int KT>
__device__ __forceinline__ void tile_rows_to_global(T* g, int64_t K, const T* D, int nrows) {
    constexpr int VPR = KT / vec<T>();
    for (int i = threadIdx.x; i < nrows * VPR; i += NT) {
        const int r = i / VPR, v = i - r * VPR;
        *reinterpret_cast<uint4*>(g + r * K + v * vec<T>()) =
            *reinterpret_cast<const uint4*>(D + r * KT + v * vec<T>());
    }
}

// ---------------------------------------------------------------------------
// Children's update rows of front rows [f0, f0+nrows): entries [eb, eb+E) of the
// gather lists; grs[r] .. grs[r+1] (relative to eb) are those of row r.
// ---------------------------------------------------------------------------
struct GatherRange {
    int eb, E;
};

template <typename T>
__device__ __forceinline__ GatherRange gather_open(const SolveArgs<T>& a, int64_t fb, int f0, int nrows, int* grs) {
    GatherRange g;
    g.eb = a.gm_ptr[fb + f0];
    g.E = a.gm_ptr[fb + f0 + nrows] - g.eb;
    for (int r = threadIdx.x; r <= nrows; r += NT) grs[r] = a.gm_ptr[fb + f0 + r] - g.eb;
    return g;
}

// Async copies of the staged chunk that starts at entry e0; live[e] = 0 for rows
// of children off the sources' paths (their update rows were never written).
template <typename T, int KT>
__device__ __forceinline__ void gather_issue(const SolveArgs<T>& a, const GatherRange& g, int e0, int k0, T* St,
                                             unsigned char* live) {
    constexpr int VPR = KT / vec<T>(), SG = stage_rows<T>();
    const int ne = min(g.E - e0, SG);
    for (int i = threadIdx.x; i < ne * VPR; i += NT) {
        const int e = i / VPR, v = i - e * VPR;
        const int ge = g.eb + e0 + e;
        const bool on = !a.reach || a.reach[a.gm_child[ge]];
        if (v == 0) live[e] = on;
        if (on) copy16_async(St + e * KT + v * vec<T>(), a.U + (int64_t)a.gm_src[ge] * a.K + k0 + v * vec<T>());
    }
}

// D rows (+ or -)= the staged entries [e0, e1) that belong to them, in entry order.
template <typename T, int KT, bool SUB>
__device__ __forceinline__ void gather_accumulate(T* D, const T* St, const unsigned char* live, const int* grs,
                                                  int nrows, int e0, int e1) {
    constexpr int G = vec<T>(), TPR = KT / G, RG = NT / TPR;  // threads per row (one vector each), rows in parallel
    const int c = G * (threadIdx.x % TPR);
    for (int r = threadIdx.x / TPR; r < nrows; r += RG) {
        const int lo = max(grs[r], e0), hi = min(grs[r + 1], e1);
        if (lo >= hi) continue;
        T v[G], u[G];
        ldv(D + r * KT + c, v);
        for (int e = lo; e < hi; ++e) {
            if (!live[e - e0]) continue;
            ldv(St + (e - e0) * KT + c, u);
#pragma unroll
            for (int q = 0; q < G; ++q) v[q] = SUB ? v[q] - u[q] : v[q] + u[q];
        }
        stv(D + r * KT + c, v);
    }
}

// Waits for every copy this CTA has in flight (the caller has issued the
// range's first chunk), then adds the range chunk by chunk.
template <typename T, int KT, bool SUB>
__device__ __forceinline__ void gather_finish(const SolveArgs<T>& a, const GatherRange& g, int k0, T* D, int nrows,
                                              T* St, unsigned char* live, const int* grs) {
    constexpr int SG = stage_rows<T>();
    int e0 = 0;
    do {
        if (e0 > 0) {
            gather_issue<T, KT>(a, g, e0, k0, St, live);
            copy_async_commit();
        }
        copy_async_wait();
        __syncthreads();
        if (g.E > 0) gather_accumulate<T, KT, SUB>(D, St, live, grs, nrows, e0, min(g.E, e0 + SG));
        __syncthreads();
        e0 += SG;
    } while (e0 < g.E);
}

template <typename T, int KT>
__global__ void __launch_bounds__(NT, 2) k_fwd(SolveArgs<T> a, int32_t t0) {
    constexpr int NB = KT / 16, VPR = KT / vec<T>();
    extern __shared__ __align__(16) unsigned char smraw[];
    T* Wt = reinterpret_cast<T*>(smraw);   // TR x KT: W, then X, then this chunk's update rows
    T* Lp = Wt + TR * KT;                   // TR x LDP: inverse diagonal block, then the panel chunk
    T* St = Lp + TR * LDP;                  // stage_rows x KT: children's update rows
    __shared__ int grs[TR + 1];
    __shared__ unsigned char live[stage_rows<T>()];
    const int2 task = a.tasks[t0 + blockIdx.x];
    const int s = task.x, chunk = task.y;
    if (a.reach && !a.reach[s]) return;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;
    const int K = a.K, k0 = blockIdx.y * KT;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], nr = m - ns;
    const int64_t fb = p.sn_rowptr[s];
    const int q0 = chunk * TR;
    const int nq = nr > 0 ? min(TR, nr - q0) : 0;

    // the inverse block, the right-hand side rows and the first children's rows
    // are in flight together (identity right-hand sides are built in place)
    const T* inv = a.inv + p.sn_invptr[s];
    for (int e = tid; e < ns * ns; e += NT) {
        const int i = e / ns, j = e - i * ns;
        copy_async(&Lp[i * LDP + j], inv + e);
    }
    if (a.delta_src) {
        for (int e = tid; e < ns * KT; e += NT) {
            const int f = e / KT, c = e - f * KT;
            Wt[f * KT + c] = (a.delta_src[k0 + c] == c0 + f) ? T(1) : T(0);
        }
    } else {
        for (int i = tid; i < ns * VPR; i += NT) {
            const int f = i / VPR, v = i - f * VPR;
            copy16_async(Wt + f * KT + v * vec<T>(), a.R + (int64_t)(c0 + f) * K + k0 + v * vec<T>());
        }
    }
    const GatherRange g1 = gather_open(a, fb, 0, ns, grs);
    if (g1.E > 0) gather_issue<T, KT>(a, g1, 0, k0, St, live);
    copy_async_commit();
    gather_finish<T, KT, true>(a, g1, k0, Wt, ns, St, live, grs);

    // X = inv(L_ss) W, written over W
    T acc[4][NB];
    zero(acc);
    mma_rows(acc, Lp, LDP, Wt, KT, ns, ns, ty, tx);
    __syncthreads();
    store_rows(Wt, KT, acc, ns, ty, tx);
    __syncthreads();
    if (chunk == 0) tile_rows_to_global<T, KT>(a.B + (int64_t)c0 * K + k0, K, Wt, ns);
    if (nq <= 0) return;

    // U_s rows of this chunk = L_rs X + the children's rows landing on them; the
    // panel rows take the inverse's place
    const T* P = a.val + p.sn_valptr[s] + (int64_t)(ns + q0) * ns;
    for (int e = tid; e < nq * ns; e += NT) {
        const int r = e / ns, j = e - r * ns;
        copy_async(&Lp[r * LDP + j], P + e);
    }
    const GatherRange g2 = gather_open(a, fb, ns + q0, nq, grs);
    if (g2.E > 0) gather_issue<T, KT>(a, g2, 0, k0, St, live);
    copy_async_commit();
    copy_async_wait();
    __syncthreads();
    zero(acc);
    mma_rows(acc, Lp, LDP, Wt, KT, ns, nq, ty, tx);
    __syncthreads();
    store_rows(Wt, KT, acc, nq, ty, tx);
    gather_finish<T, KT, false>(a, g2, k0, Wt, nq, St, live, grs);
    tile_rows_to_global<T, KT>(a.U + (a.uoff[s] + q0) * (int64_t)K + k0, K, Wt, nq);
}

template <typename T, int KT>
__global__ void __launch_bounds__(NT) k_bwd(SolveArgs<T> a, int32_t t0) {
    constexpr int NB = KT / 16, VPR = KT / vec<T>(), G = vec<T>();
    constexpr int PS = RC * TR, XS = RC * KT;  // one chunk buffer: panel rows, gathered solution rows
    static_assert(2 * (PS + XS) >= TR * KT + TR * TR, "the finishing tiles alias the chunk buffers");
    extern __shared__ __align__(16) unsigned char smraw[];
    T* buf = reinterpret_cast<T*>(smraw);
    T* Cs = buf;             // TR x KT, after the gather
    T* Ms = buf + TR * KT;   // TR x TR inverse diagonal block, after the gather
    __shared__ int last_arrival;
    const int2 task = a.tasks[t0 + blockIdx.x];
    const int s = task.x, split = task.y;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;
    const int K = a.K, k0 = blockIdx.y * KT;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], nr = m - ns;
    const int nspl = a.nsplit[s];
    const int q0 = split * kSplitRows, q1 = min(nr, q0 + kSplitRows);
    const T* P = a.val + p.sn_valptr[s];
    const int32_t* rows = p.rows + p.sn_rowptr[s];

    // chunk ci of the split's structure rows into buffer ci & 1
    auto issue = [&](int ci) {
        const int qq = q0 + ci * RC, nc = min(RC, q1 - qq);
        T* Ps = buf + (ci & 1) * (PS + XS);
        T* Xg = Ps + PS;
        for (int e = tid; e < nc * ns; e += NT) {
            const int r = e / ns, j = e - r * ns;
            copy_async(&Ps[r * TR + j], P + (int64_t)(ns + qq + r) * ns + j);
        }
        for (int i = tid; i < nc * VPR; i += NT) {
            const int r = i / VPR, v = i - r * VPR;
            copy16_async(Xg + r * KT + v * vec<T>(), a.B + (int64_t)rows[ns + qq + r] * K + k0 + v * vec<T>());
        }
        copy_async_commit();
    };
    T acc[4][NB];
    zero(acc);
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
        mma_cols(acc, Ps, TR, Ps + PS, KT, min(RC, q1 - q0 - ci * RC), ns, ty, tx);
        __syncthreads();
    }

    const bool zero_y = a.reach && !a.reach[s];
    if (nspl > 1) {
        T* part = a.part + a.poff[s] * (int64_t)TR * K + k0;
        store_rows(part + (int64_t)split * TR * K, (int64_t)K, acc, ns, ty, tx);
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            const int ticket = atomicAdd(&a.counters[(int64_t)s * a.ktiles + blockIdx.y], 1);
            last_arrival = ticket == nspl - 1;
        }
        __syncthreads();
        if (!last_arrival) return;
        __threadfence();
#pragma unroll
        for (int aa = 0; aa < 4; ++aa) {
            const int t = ty + 16 * aa;
            if (t < ns)
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    T sum = T(0);
                    for (int sp = 0; sp < nspl; ++sp)
                        sum += __ldcg(&part[((int64_t)sp * TR + t) * K + col_of<T>(tx, b)]);
                    acc[aa][b] = sum;
                }
        }
        if (tid == 0) a.counters[(int64_t)s * a.ktiles + blockIdx.y] = 0;
    }
    // C = y - acc; X_s = inv(L_ss)^T C
    const T* inv = a.inv + p.sn_invptr[s];
    for (int e = tid; e < ns * ns; e += NT) {
        const int i = e / ns, j = e - i * ns;
        copy_async(&Ms[i * TR + j], inv + e);
    }
    copy_async_commit();
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int t = ty + 16 * aa;
        if (t < ns)
#pragma unroll
            for (int h = 0; h < NB / G; ++h) {
                T y[G];
#pragma unroll
                for (int q = 0; q < G; ++q) y[q] = T(0);
                if (!zero_y) ldv(a.B + (int64_t)(c0 + t) * K + k0 + G * tx + 16 * G * h, y);
#pragma unroll
                for (int q = 0; q < G; ++q) y[q] -= acc[aa][G * h + q];
                stv(Cs + t * KT + G * tx + 16 * G * h, y);
            }
    }
    copy_async_wait();
    __syncthreads();
    zero(acc);
    mma_cols(acc, Ms, TR, Cs, KT, ns, ns, ty, tx);
    store_rows(a.B + (int64_t)c0 * K + k0, (int64_t)K, acc, ns, ty, tx);
}

__global__ void k_reach(const int32_t* __restrict__ col_sn, const int32_t* __restrict__ parent,
                        const int32_t* __restrict__ src, int32_t K, int32_t nlevels, uint8_t* __restrict__ reach) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const int s0 = src[k];
    if (s0 < 0) return;
    int s = col_sn[s0];
    // the parent chain is strictly increasing and at most nlevels long
    for (int it = 0; s >= 0 && it <= nlevels; ++it) {
        reach[s] = 1;
        s = parent[s];
    }
}

template <typename T, int KT>
constexpr size_t fwd_smem() { return (size_t)(TR * KT + TR * LDP + stage_rows<T>() * KT) * sizeof(T); }
template <typename T, int KT>
constexpr size_t bwd_smem() { return (size_t)2 * (RC * TR + RC * KT) * sizeof(T); }

template <typename T, int KT>
cudaError_t set_smem() {
    cudaError_t e = cudaFuncSetAttribute(k_fwd<T, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fwd_smem<T, KT>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_bwd<T, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bwd_smem<T, KT>());
}

}  // namespace

cudaError_t configure_solve_kernels() {
    cudaError_t e;
    if ((e = set_smem<double, 64>())) return e;
    if ((e = set_smem<float, 64>())) return e;
    return set_smem<float, 128>();
}

template <typename T>
void launch_fwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    constexpr int W = wide_tile<T>();
    if (W != 64 && a.K % W == 0)
        k_fwd<T, W><<<dim3(ntasks, a.K / W), NT, fwd_smem<T, W>(), st>>>(a, t0);
    else
        k_fwd<T, 64><<<dim3(ntasks, a.K / 64), NT, fwd_smem<T, 64>(), st>>>(a, t0);
}

template <typename T>
void launch_bwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    constexpr int W = wide_tile<T>();
    if (W != 64 && a.K % W == 0)
        k_bwd<T, W><<<dim3(ntasks, a.K / W), NT, bwd_smem<T, W>(), st>>>(a, t0);
    else
        k_bwd<T, 64><<<dim3(ntasks, a.K / 64), NT, bwd_smem<T, 64>(), st>>>(a, t0);
}

void launch_reach(const DevPlan& p, const int32_t* src, int32_t K, uint8_t* reach, cudaStream_t st) {
    cudaMemsetAsync(reach, 0, (size_t)p.nsuper, st);
    k_reach<<<(K + 127) / 128, 128, 0, st>>>(p.col_sn, p.sn_parent, src, K, p.nlevels, reach);
}

template void launch_fwd_level<double>(const SolveArgs<double>&, int32_t, int32_t, cudaStream_t);
template void launch_fwd_level<float>(const SolveArgs<float>&, int32_t, int32_t, cudaStream_t);
template void launch_bwd_level<double>(const SolveArgs<double>&, int32_t, int32_t, cudaStream_t);
template void launch_bwd_level<float>(const SolveArgs<float>&, int32_t, int32_t, cudaStream_t);

}  // namespace fcw
