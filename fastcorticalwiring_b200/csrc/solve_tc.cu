// FP32 supernodal sweeps on the Blackwell tensor cores (the mixed Poisson solve).
//
// Same algorithm and task graph as the FP32 sweeps of solve.cu (multifrontal
// forward, split-K backward, one etree level per launch); the dense products
// run as tcgen05.mma kind::tf32 with FP32 accumulators in tensor memory:
//
//   * Each FP32 operand is split into two TF32 terms (hi = rna(x), lo =
//     rna(x - hi)) and hi*hi + hi*lo + lo*hi accumulate, which keeps the product
//     at FP32 accuracy (the dropped lo*lo term is below 2^-22 |a||b|).
//   * Every operand is K-major (the product's depth contiguous in 16-byte
//     chunks of core matrices; tc.cuh): a transposed, MN-major operand read as
//     kind::tf32 with no swizzle comes back as zeros on this hardware, so the
//     transposes are made when the operands are written instead.
//   * The panel operands are prepared once per factorisation: the stacked
//     [inv(L_ss); Q_s] of each supernode, split into hi and lo arrays in
//     core-matrix order, once as stored (rows x columns, the forward's A) and
//     once transposed in 32-row chunks (the backward's A = Q_s^T, inv(L_ss)^T).
//     A task's slice is one contiguous range, fetched by the TMA engine as two
//     bulk copies.
//   * A supernode's own right-hand-side rows (forward: R, backward: y_s) are a
//     64-row x 64-column box of the n x K array, fetched by a tiled TMA load with
//     128-byte swizzle; children's update rows and ancestors' solution rows are
//     gathered by index with 16-byte cp.async copies, as in solve.cu.
//   * Threads split the right-hand-side tile into TF32 terms, transposed into the
//     K-major core-matrix layout, one thread issues the MMAs, a tcgen05.commit arrives on an
//     mbarrier, and the accumulator comes back through tcgen05.ld to a shared
//     tile that is written out with 16-byte row-segment stores.
//
// A CTA is one task x 64 columns (the MMA's N); M = 128 forward, 64 backward. Every wait (TMA and
// MMA completion) is bounded: past about two seconds the CTA raises
// KERR_TIMEOUT in a.err, frees its tensor memory and returns.
#include "kernels.cuh"
#include "sweep_rows.cuh"
#include "tc.cuh"

namespace fcw {
namespace {

constexpr int TCN = kTcCols;            // right-hand-side columns per CTA (N of the MMA)
constexpr int TCM = 64;                 // rows of a task's product (M of the MMA)
constexpr int TC_LS = TCN + 4;          // row stride (floats) of the output and gathered-row tiles
constexpr int TC_STAGE = 48;            // children's update rows staged per gather chunk (forward)
constexpr int TCF = 128;                // rows of a forward task's product (M = 128)
constexpr int TC_RC = 32;               // structure rows per backward chunk
constexpr int TC_PT = kMaxWidth;        // rows of a backward partial-sum slot
constexpr uint32_t TC_TILE = 64u * TCN * 4u;   // a 64 x 64 FP32 tile (16 KB)
// A backward A of M = 64 (8 groups of 8 columns) holds only ns8 / 8 groups: the product reads up to
// 7 groups of 8 k-chunks (7 KB) past a chunk tile, 4 KB past the inverse block's tile
constexpr uint32_t TC_SLACK = 7168;

// Byte offset of element (r, c) of the own-row tile: two TMA boxes of 64 rows x 32
// columns (128-byte rows), 128-byte swizzle (16-byte chunk index XOR row % 8).
__device__ __forceinline__ uint32_t swz(int r, int c) {
    const uint32_t box = (uint32_t)(c >> 5), ch = (uint32_t)((c & 31) >> 2);
    return box * 8192u + (uint32_t)r * 128u + ((ch ^ (uint32_t)(r & 7)) << 4) + (uint32_t)(c & 3) * 4u;
}

// Own-row tile rows [0, nrows) -= the staged children's rows [e0, e1) that land on them.
__device__ __forceinline__ void gather_sub_swz(unsigned char* Tt, const float* St, const unsigned char* live,
                                               const int* grs, int nrows, int e0, int e1) {
    constexpr int TPR = TCN / 4, RG = NT / TPR;
    const int c = 4 * (threadIdx.x % TPR);
    for (int r = threadIdx.x / TPR; r < nrows; r += RG) {
        const int lo = max(grs[r], e0), hi = min(grs[r + 1], e1);
        if (lo >= hi) continue;
        float4* d = reinterpret_cast<float4*>(Tt + swz(r, c));
        float4 v = *d;
        for (int e = lo; e < hi; ++e) {
            if (!live[e - e0]) continue;
            const float4 u = *reinterpret_cast<const float4*>(St + (e - e0) * TCN + c);
            v.x -= u.x;
            v.y -= u.y;
            v.z -= u.z;
            v.w -= u.w;
        }
        *d = v;
    }
}

// gather_finish of solve.cu on the swizzled own-row tile (subtracting).
__device__ __forceinline__ void gather_finish_swz(const SolveArgs<float>& a, const GatherRange& g, int k0,
                                                  unsigned char* Tt, int nrows, float* St, unsigned char* live,
                                                  const int* grs) {
    const int SG = a.stage;
    int e0 = 0;
    do {
        if (e0 > 0) {
            gather_issue<float, TCN, TCM>(a, g, e0, k0, St, live);
            copy_async_commit();
        }
        copy_async_wait();
        __syncthreads();
        if (g.E > 0) gather_sub_swz(Tt, St, live, grs, nrows, e0, min(g.E, e0 + SG));
        __syncthreads();
        e0 += SG;
    } while (e0 < g.E);
}

// Rows [0, nk) of the swizzled own-row tile (k x 64 columns) as the K-major B operand:
// element (n, k) at core (n / 8, k / 4) of round_up(nk, 8) / 4 k-chunks per 8-column group,
// split into TF32 hi and lo; rows k >= nk are zero. B hi overlays the tile, so every thread
// reads its values before any thread writes. Item i = (k-chunk, column group, column in
// group) with the column fastest: a warp reads 32 consecutive columns of a row (conflict
// free under the swizzle) and 8 lanes fill one 128-byte core.
__device__ __forceinline__ void split_own_rows(const unsigned char* Tt, int nk, float* Bhi, float* Blo) {
    constexpr int PER = (64 * TCN / 4) / NT;
    const int nk8 = (nk + 7) & ~7, kcores = nk8 >> 2;
    float4 w[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * NT;
        const int n = i & 63, kc = i >> 6;
        float x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = 4 * kc + q;
            x[q] = k < nk ? *reinterpret_cast<const float*>(Tt + swz(k, n)) : 0.0f;
        }
        w[j] = make_float4(x[0], x[1], x[2], x[3]);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * NT;
        const int n = i & 63, kc = i >> 6;
        if (kc >= kcores) continue;
        const uint32_t off = ((uint32_t)((n >> 3) * kcores + kc) << 5) + (uint32_t)((n & 7) << 2);  // floats
        float4 h, l;
        tc::split_tf32(w[j].x, h.x, l.x);
        tc::split_tf32(w[j].y, h.y, l.y);
        tc::split_tf32(w[j].z, h.z, l.z);
        tc::split_tf32(w[j].w, h.w, l.w);
        *reinterpret_cast<float4*>(Bhi + off) = h;
        *reinterpret_cast<float4*>(Blo + off) = l;
    }
}

// Rows [0, nk) of a gathered-row tile (TC_RC rows x 64 columns, row stride TC_LS) as the
// K-major B operand of TC_RC rows (8 k-chunks per 8-column group; rows >= nk zero), split
// into TF32 hi and lo (separate buffers).
__device__ __forceinline__ void split_gathered(const float* Xg, int nk, float* Bhi, float* Blo) {
    constexpr int PER = (TC_RC * TCN / 4) / NT, KC = TC_RC / 4;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * NT;
        const int n = i & 63, kc = i >> 6;
        float x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = 4 * kc + q;
            x[q] = k < nk ? Xg[k * TC_LS + n] : 0.0f;
        }
        const uint32_t off = ((uint32_t)((n >> 3) * KC + kc) << 5) + (uint32_t)((n & 7) << 2);
        float4 h, l;
        tc::split_tf32(x[0], h.x, l.x);
        tc::split_tf32(x[1], h.y, l.y);
        tc::split_tf32(x[2], h.z, l.z);
        tc::split_tf32(x[3], h.w, l.w);
        *reinterpret_cast<float4*>(Bhi + off) = h;
        *reinterpret_cast<float4*>(Blo + off) = l;
    }
}

// D (+)= A B (M rows, N = 64) over ksteps steps of K = 8 with two TF32 terms per operand.
// Both operands K-major: A in groups of 8 rows with a_kcores 16-byte k-chunks each, B in
// groups of 8 columns with b_kcores k-chunks each; a step advances both by two chunks.
template <int M>
__device__ __forceinline__ void issue_split_mma(uint32_t d, const float* Ahi, const float* Alo, uint32_t a_kcores,
                                                const float* Bhi, const float* Blo, uint32_t b_kcores, int ksteps,
                                                bool accumulate) {
    const uint32_t idesc = tc::idesc_tf32(M, TCN, false, false, false);
    const uint32_t ah = tc::smem_u32(Ahi), al = tc::smem_u32(Alo), bh = tc::smem_u32(Bhi), bl = tc::smem_u32(Blo);
    const uint32_t a_sbo = a_kcores * 128u, b_sbo = b_kcores * 128u;
    for (int ks = 0; ks < ksteps; ++ks) {
        const uint32_t step = (uint32_t)ks * 256u;
        const uint64_t dah = tc::sdesc(ah + step, 128u, a_sbo);
        const uint64_t dal = tc::sdesc(al + step, 128u, a_sbo);
        const uint64_t dbh = tc::sdesc(bh + step, 128u, b_sbo);
        const uint64_t dbl = tc::sdesc(bl + step, 128u, b_sbo);
        tc::mma_tf32(d, dah, dbh, idesc, (accumulate || ks > 0) ? 1u : 0u);
        tc::mma_tf32(d, dah, dbl, idesc, 1u);
        tc::mma_tf32(d, dal, dbh, idesc, 1u);
    }
}

// Accumulator rows of an M = 64 product: row r sits in TMEM lane (r % 16) + 32 (r / 16).
// Warp w reads lane quarter w % 4 and column half w / 4; lanes 0-15 hold rows.
__device__ __forceinline__ void acc_half(uint32_t tmem, int col0, float* v32) {
    const int warp = threadIdx.x >> 5;
    const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(col0 + 32 * (warp >> 2));
    tc::tmem_ld16(base, v32);
    tc::tmem_ld16(base + 16, v32 + 16);
}
__device__ __forceinline__ int acc_row() { return 16 * ((threadIdx.x >> 5) & 3) + (threadIdx.x & 15); }
__device__ __forceinline__ bool acc_lane() { return (threadIdx.x & 31) < 16; }
__device__ __forceinline__ int acc_col() { return 32 * (threadIdx.x >> 7); }

// All threads wait; if any gives up, every thread sees `bail` set (CTA-uniform).
__device__ __forceinline__ bool wait_all(uint64_t* bar, uint32_t parity, int* bail, int* err) {
    if (!tc::mbar_wait(bar, parity)) atomicOr(bail, 1);
    __syncthreads();
    if (*bail) {
        if (threadIdx.x == 0 && err) atomicOr(err, KERR_TIMEOUT);
        return false;
    }
    return true;
}

__device__ __forceinline__ unsigned char* align1k(unsigned char* p) {
    const uint32_t s = tc::smem_u32(p);
    return p + (((s + 1023u) & ~1023u) - s);
}

// ---------------------------------------------------------------------------
// Forward: task (s, c) is one M = 128 product with W (the supernode's right-hand side less
// its children's update rows). c = 0: rows [0, 64) of A are inv(L_ss) (X_s, written to B)
// and rows [64, 128) the first 64 rows of Q_s (update rows [0, 64)); c >= 1: 128 rows of
// Q_s, update rows [64 + 128 (c - 1), ...). Update rows get the children's rows that land
// on them and go to U for the parent.
// Shared memory: R0 = A hi | A lo (64 KB; the output tile after the product), R1 = own-row
// TMA tile, then B hi | B lo (32 KB), R2 = children's update rows (TC_STAGE x 64 floats).
// ---------------------------------------------------------------------------
constexpr uint32_t TC_FTILE = (uint32_t)TCF * 64u * 4u;  // one A term: 128 rows x 64 columns (32 KB)
constexpr size_t kFwdTcSmem = 1024 + 2 * (size_t)TC_FTILE + 2 * TC_TILE + (size_t)TC_STAGE * TCN * 4;

__device__ __forceinline__ int fwd_first_row(int chunk) { return chunk == 0 ? 0 : 64 + (chunk - 1) * TCF; }

__global__ void __launch_bounds__(NT, 2) k_fwd_tc(SolveArgs<float> a, int32_t t0, int32_t ntiles,
                                                 const __grid_constant__ CUtensorMap rmap) {
    extern __shared__ unsigned char smraw_tc[];
    unsigned char* sm = align1k(smraw_tc);
    float* Ahi = reinterpret_cast<float*>(sm);
    float* Alo = reinterpret_cast<float*>(sm + TC_FTILE);
    float* Ot = reinterpret_cast<float*>(sm);
    unsigned char* Tt = sm + 2 * TC_FTILE;
    float* Bhi = reinterpret_cast<float*>(sm + 2 * TC_FTILE);
    float* Blo = reinterpret_cast<float*>(sm + 2 * TC_FTILE + TC_TILE);
    float* St = reinterpret_cast<float*>(sm + 2 * TC_FTILE + 2 * TC_TILE);
    __shared__ int grs[TCF + 1];
    __shared__ unsigned char live[TC_STAGE];
    __shared__ uint64_t bar_ld, bar_mma;
    __shared__ uint32_t tbase;
    __shared__ int bail;

    const int ti = blockIdx.x / ntiles, tile = blockIdx.x - ti * ntiles;
    const int2 task = a.tasks[t0 + ti];
    const int s = task.x, chunk = task.y;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int K = a.K, k0 = tile * TCN;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, nr = p.sn_m[s] - ns;
    const int ns8 = (ns + 7) & ~7, nr32 = (nr + 31) & ~31;
    const int64_t fb = p.sn_rowptr[s];
    const bool xtask = chunk == 0;
    const int q0 = fwd_first_row(chunk);             // first update row of the task
    const int qrows = xtask ? 64 : TCF;               // update rows the task's product holds
    const int nq = max(0, min(qrows, nr - q0));       // of which real
    const int qa = max(0, min(qrows, nr32 - q0));     // Q rows in the core array (padding zero)
    const uint32_t row_bytes = (uint32_t)ns8 * 4u;
    const int64_t cbase = a.core_ptr[s];

    if (tid == 0) {
        tc::mbar_init(&bar_ld, 1);
        tc::mbar_init(&bar_mma, 1);
        tc::fence_mbar_init();
        bail = 0;
    }
    if (warp == 0) tc::tmem_alloc(&tbase, TCN);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;
    if (tid == 0) {
        // A rows: [0, ns8) the inverse (chunk 0), then from row 64 (chunk 0) or 0 the Q rows
        const uint32_t inv_bytes = xtask ? (uint32_t)ns8 * row_bytes : 0u;
        const uint32_t q_bytes = (uint32_t)qa * row_bytes;
        const uint32_t qdst = (xtask ? 64u : 0u) * (uint32_t)(ns8 >> 2) * 16u;  // 8-row groups of ns8/4 cores
        tc::mbar_arrive_expect_tx(&bar_ld, 2 * (inv_bytes + q_bytes) + TC_TILE);
        if (inv_bytes) {
            tc::bulk_load(Ahi, a.core_hi + cbase, inv_bytes, &bar_ld);
            tc::bulk_load(Alo, a.core_lo + cbase, inv_bytes, &bar_ld);
        }
        if (q_bytes) {
            const int64_t qoff = cbase + (int64_t)(ns8 + q0) * ns8;
            tc::bulk_load(reinterpret_cast<unsigned char*>(Ahi) + qdst, a.core_hi + qoff, q_bytes, &bar_ld);
            tc::bulk_load(reinterpret_cast<unsigned char*>(Alo) + qdst, a.core_lo + qoff, q_bytes, &bar_ld);
        }
        tc::tma_load_2d(Tt, &rmap, k0, c0, &bar_ld);
        tc::tma_load_2d(Tt + 8192, &rmap, k0 + 32, c0, &bar_ld);
    }
    // the children's rows that land on this supernode's columns, while the TMA copies fly
    const GatherRange g1 = gather_open(a, fb, 0, ns, grs);
    if (g1.E > 0) gather_issue<float, TCN, TCF>(a, g1, 0, k0, St, live);
    copy_async_commit();
    bool ok = wait_all(&bar_ld, 0, &bail, a.err);
    if (ok) {
        gather_finish_swz(a, g1, k0, Tt, ns, St, live, grs);  // W = R - children's rows
        split_own_rows(Tt, ns, Bhi, Blo);
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_split_mma<TCF>(tmem, Ahi, Alo, (uint32_t)(ns8 >> 2), Bhi, Blo, (uint32_t)(ns8 >> 2), ns8 >> 3,
                                 false);
            tc::mma_commit(&bar_mma);
        }
        // the children's rows of this task's update rows arrive while the product runs
        GatherRange g2{0, 0};
        if (nq > 0) {
            g2 = gather_open(a, fb, ns + q0, nq, grs);
            if (g2.E > 0) gather_issue<float, TCN, TCF>(a, g2, 0, k0, St, live);
            copy_async_commit();
        }
        ok = wait_all(&bar_mma, 0, &bail, a.err);
        if (ok) {
            tc::fence_after_sync();
            // accumulator row r = TMEM lane r (M = 128): warp w reads lanes 32 (w % 4) .. + 31,
            // columns 32 (w / 4) .. + 31
            float v[32];
            const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(32 * (warp >> 2));
            tc::tmem_ld16(base, v);
            tc::tmem_ld16(base + 16, v + 16);
            {
                float* o = Ot + (32 * (warp & 3) + lane) * TC_LS + 32 * (warp >> 2);
#pragma unroll
                for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            }
            __syncthreads();
            const int u0 = xtask ? 64 : 0;  // output-tile row of the first update row
            if (xtask) tile_rows_to_global<float, TCN>(a.B + (int64_t)c0 * K + k0, K, Ot, TC_LS, ns);
            if (nq > 0) {
                gather_finish<float, TCN, TCF, false>(a, g2, k0, Ot + u0 * TC_LS, TC_LS, nq, St, live, grs);
                tile_rows_to_global<float, TCN>(a.U + (a.uoff[s] + q0) * (int64_t)K + k0, K, Ot + u0 * TC_LS,
                                                TC_LS, nq);
            }
        }
    }
    if (!ok) {  // let copies and products in flight land before the memory is released
        tc::mbar_wait(&bar_ld, 0, 100000000ull);
        tc::mbar_wait(&bar_mma, 0, 100000000ull);
        copy_async_wait();
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, TCN);
}

// ---------------------------------------------------------------------------
// Backward: task (s, split): acc = sum over 32-row chunks of Q_s^T X_r (TMEM columns
// [0, 64)), double-buffered; then (last split) inv(L_ss)^T y_s (columns [64, 128)) and
// X_s = inv^T y_s - acc. Stage b: A hi | A lo | slack | gathered rows | B hi | B lo.
// The finishing phase reuses the stages: A hi | A lo | slack, then the own-row TMA tile
// (B hi over it) and B lo; the output tile over A.
// ---------------------------------------------------------------------------
constexpr uint32_t TC_BA = (uint32_t)TC_RC * TCM * 4u;               // one A term of a chunk (8 KB)
constexpr uint32_t TC_BX = (uint32_t)TC_RC * TC_LS * 4u;             // gathered rows (8.5 KB)
constexpr uint32_t TC_BB = (uint32_t)TC_RC * TCN * 4u;               // one B term of a chunk (8 KB)
constexpr uint32_t TC_BSTAGE = (2 * TC_BA + TC_SLACK + TC_BX + 2 * TC_BB + 1023u) & ~1023u;
constexpr uint32_t TC_FA = ((2 * TC_TILE + TC_SLACK) + 1023u) & ~1023u;  // finishing A terms + slack
constexpr size_t kBwdTcSmem = 1024 + 2 * (size_t)TC_BSTAGE;
static_assert(TC_FA + 2 * TC_TILE <= 2 * TC_BSTAGE, "finishing tiles fit in the two stages");

__global__ void __launch_bounds__(NT, 2) k_bwd_tc(SolveArgs<float> a, int32_t t0, int32_t ntiles,
                                                 const __grid_constant__ CUtensorMap bmap) {
    extern __shared__ unsigned char smraw_tc[];
    unsigned char* sm = align1k(smraw_tc);
    __shared__ uint64_t bar_ld[2], bar_mma[2], bar_fin;
    __shared__ uint32_t tbase;
    __shared__ int bail, last_arrival;

    const int ti = blockIdx.x / ntiles, tile = blockIdx.x - ti * ntiles;
    const int2 task = a.tasks[t0 + ti];
    const int s = task.x, split = task.y;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int K = a.K, k0 = tile * TCN;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, nr = p.sn_m[s] - ns;
    const int ns8 = (ns + 7) & ~7;
    const uint32_t acores = (uint32_t)(ns8 >> 2);
    const int nspl = a.nsplit[s];
    const int q0 = split * kSplitRows, q1 = min(nr, q0 + kSplitRows);
    const int nchunks = q1 > q0 ? (q1 - q0 + TC_RC - 1) / TC_RC : 0;
    const int32_t* rows = p.rows + p.sn_rowptr[s];
    const int64_t cbase = a.core_ptr[s];
    const uint32_t cbytes = (uint32_t)TC_RC * (uint32_t)ns8 * 4u;  // one term of a 32-row chunk

    auto stage = [&](int b) { return sm + b * TC_BSTAGE; };
    auto sAhi = [&](int b) { return reinterpret_cast<float*>(stage(b)); };
    auto sAlo = [&](int b) { return reinterpret_cast<float*>(stage(b) + TC_BA); };
    auto sXg = [&](int b) { return reinterpret_cast<float*>(stage(b) + 2 * TC_BA + TC_SLACK); };
    auto sBhi = [&](int b) { return reinterpret_cast<float*>(stage(b) + 2 * TC_BA + TC_SLACK + TC_BX); };
    auto sBlo = [&](int b) { return reinterpret_cast<float*>(stage(b) + 2 * TC_BA + TC_SLACK + TC_BX + TC_BB); };

    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&bar_ld[b], 1);
            tc::mbar_init(&bar_mma[b], 1);
        }
        tc::mbar_init(&bar_fin, 1);
        tc::fence_mbar_init();
        bail = 0;
    }
    if (warp == 0) tc::tmem_alloc(&tbase, 2 * TCN);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;

    // chunk j of this split's structure rows into stage j & 1
    auto issue = [&](int j) {
        const int b = j & 1, qq = q0 + j * TC_RC, nc = min(TC_RC, q1 - qq);
        if (tid == 0) {
            tc::mbar_arrive_expect_tx(&bar_ld[b], 2 * cbytes);
            const int64_t off = cbase + (int64_t)(ns8 + qq) * ns8;  // chunk qq / 32 of the transposed array
            tc::bulk_load(sAhi(b), a.coreT_hi + off, cbytes, &bar_ld[b]);
            tc::bulk_load(sAlo(b), a.coreT_lo + off, cbytes, &bar_ld[b]);
        }
        float* Xg = sXg(b);
        for (int i = tid; i < nc * (TCN / 4); i += NT) {
            const int r = i / (TCN / 4), v = i - r * (TCN / 4);
            copy16_async(Xg + r * TC_LS + 4 * v, a.B + (int64_t)rows[ns + qq + r] * K + k0 + 4 * v);
        }
        copy_async_commit();
    };

    bool ok = true;
    int uses_fin = 0;
    if (nchunks > 0) issue(0);
    for (int j = 0; j < nchunks && ok; ++j) {
        const int b = j & 1;
        if (j + 1 < nchunks) {
            // stage (j + 1) & 1 last served chunk j - 1: its products must be done with it
            if (j >= 1 && !(ok = wait_all(&bar_mma[(j + 1) & 1], ((j - 1) >> 1) & 1, &bail, a.err))) break;
            issue(j + 1);
            copy_async_wait_prev();
        } else {
            copy_async_wait();
        }
        if (!(ok = wait_all(&bar_ld[b], (j >> 1) & 1, &bail, a.err))) break;
        const int nc = min(TC_RC, q1 - (q0 + j * TC_RC));
        split_gathered(sXg(b), nc, sBhi(b), sBlo(b));
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_split_mma<TCM>(tmem, sAhi(b), sAlo(b), TC_RC / 4, sBhi(b), sBlo(b), TC_RC / 4, (nc + 7) >> 3,
                                 j > 0);
            tc::mma_commit(&bar_mma[b]);
        }
    }
    if (ok && nchunks > 0) ok = wait_all(&bar_mma[(nchunks - 1) & 1], ((nchunks - 1) >> 1) & 1, &bail, a.err);

    bool finish = ok;
    if (ok && nspl > 1) {  // split-K: this split's partial sum, the last arrival finishes
        tc::fence_after_sync();
        float* part = a.part + a.poff[s] * (int64_t)TC_PT * K + k0;
        float v[32];
        acc_half(tmem, 0, v);
        if (acc_lane() && acc_row() < ns) {
            float* mine = part + ((int64_t)split * TC_PT + acc_row()) * K + acc_col();
#pragma unroll
            for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(mine + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            const int ticket = atomicAdd(&a.counters[(int64_t)s * a.ktiles + tile], 1);
            last_arrival = ticket == nspl - 1;
        }
        __syncthreads();
        finish = last_arrival != 0;
        if (finish) __threadfence();
    }
    if (finish) {
        // inv(L_ss)^T y_s: the inverse block's terms and the own rows y_s (TMA)
        float* Fhi = reinterpret_cast<float*>(sm);
        float* Flo = reinterpret_cast<float*>(sm + TC_TILE);
        unsigned char* Tt = sm + TC_FA;
        float* Bhi = reinterpret_cast<float*>(sm + TC_FA);
        float* Blo = reinterpret_cast<float*>(sm + TC_FA + TC_TILE);
        float* Ot = reinterpret_cast<float*>(sm);
        // the loads below overwrite shared memory the threads wrote (generic proxy)
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            const uint32_t ibytes = (uint32_t)ns8 * (uint32_t)ns8 * 4u;
            tc::mbar_arrive_expect_tx(&bar_fin, 2 * ibytes + TC_TILE);
            tc::bulk_load(Fhi, a.coreT_hi + cbase, ibytes, &bar_fin);
            tc::bulk_load(Flo, a.coreT_lo + cbase, ibytes, &bar_fin);
            tc::tma_load_2d(Tt, &bmap, k0, c0, &bar_fin);
            tc::tma_load_2d(Tt + 8192, &bmap, k0 + 32, c0, &bar_fin);
        }
        uses_fin = 1;
        if ((ok = wait_all(&bar_fin, 0, &bail, a.err))) {
            split_own_rows(Tt, ns, Bhi, Blo);
            tc::fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                issue_split_mma<TCM>(tmem + TCN, Fhi, Flo, acores, Bhi, Blo, acores, ns8 >> 3, false);
                tc::mma_commit(&bar_fin);
            }
            if ((ok = wait_all(&bar_fin, 1, &bail, a.err))) {
                tc::fence_after_sync();
                float y[32], acc[32];
                acc_half(tmem, TCN, y);
                if (nchunks > 0) acc_half(tmem, 0, acc);
                const int r = acc_row(), col = acc_col();
                if (nspl > 1) {  // the partial sums in split order (this CTA's own included)
                    const float* part = a.part + a.poff[s] * (int64_t)TC_PT * K + k0;
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[j] = 0.0f;
                    if (acc_lane() && r < ns)
                        for (int sp = 0; sp < nspl; ++sp) {
                            const float* q = part + ((int64_t)sp * TC_PT + r) * K + col;
#pragma unroll
                            for (int j = 0; j < 32; ++j) acc[j] += __ldcg(q + j);
                        }
                }
                if (acc_lane()) {
                    float* o = Ot + r * TC_LS + col;
#pragma unroll
                    for (int j = 0; j < 32; j += 4) {
                        float4 x;
                        x.x = nchunks > 0 ? y[j] - acc[j] : y[j];
                        x.y = nchunks > 0 ? y[j + 1] - acc[j + 1] : y[j + 1];
                        x.z = nchunks > 0 ? y[j + 2] - acc[j + 2] : y[j + 2];
                        x.w = nchunks > 0 ? y[j + 3] - acc[j + 3] : y[j + 3];
                        *reinterpret_cast<float4*>(o + j) = x;
                    }
                }
                __syncthreads();
                tile_rows_to_global<float, TCN>(a.B + (int64_t)c0 * K + k0, K, Ot, TC_LS, ns);
                if (nspl > 1 && tid == 0) a.counters[(int64_t)s * a.ktiles + tile] = 0;
            }
        }
    }
    if (!ok) {  // let copies and products in flight land before the memory is released
        for (int b = 0; b < 2; ++b) {
            tc::mbar_wait(&bar_ld[b], 0, 100000000ull);
            tc::mbar_wait(&bar_mma[b], 0, 100000000ull);
        }
        if (uses_fin) tc::mbar_wait(&bar_fin, 0, 100000000ull);
        copy_async_wait();
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 2 * TCN);
}

// Core arrays of the stacked [inv(L_ss); Q_s], one CTA per supernode (rows >= ns of the
// inverse part, rows >= nr of the Q part and columns >= ns are zero; hi = rna_tf32(x),
// lo = rna_tf32(x - hi) from the FP64 value):
//  * forward (hi, lo): element (row r, column i) at core_offset(r, i, ns8 / 4), the K-major
//    A of the forward products (rows x columns);
//  * backward (hiT, loT): the transposes, K-major over the rows: the inverse part
//    (rows j < ns8) at core_offset(i, j, ns8 / 4), then each 32-row chunk of Q_s (local row
//    q) at ns8 * ns8 + chunk * 32 * ns8 floats + core_offset(i, q, 8).
__global__ void k_build_cores(DevPlan p, const double* __restrict__ val, const double* __restrict__ inv,
                              const int64_t* __restrict__ core_ptr, float* __restrict__ hi, float* __restrict__ lo,
                              float* __restrict__ hiT, float* __restrict__ loT) {
    const int s = blockIdx.x;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, nr = p.sn_m[s] - ns;
    const int ns8 = (ns + 7) & ~7, nr32 = (nr + 31) & ~31, rows = ns8 + nr32;
    const double* P = val + p.sn_valptr[s];
    const double* I = inv + p.sn_invptr[s];
    const int64_t base = core_ptr[s];
    const int icores = ns8 >> 2;
    for (int e = threadIdx.x; e < rows * ns8; e += blockDim.x) {
        const int r = e / ns8, c = e - r * ns8;
        double x = 0.0;
        if (c < ns) {
            if (r < ns) x = I[r * ns + c];
            else if (r >= ns8 && r - ns8 < nr) x = P[(int64_t)(ns + r - ns8) * ns + c];
        }
        const float h = tc::to_tf32((float)x);
        const float l = tc::to_tf32((float)(x - (double)h));
        const int64_t off = base + (tc::core_offset(r, c, icores) >> 2);
        hi[off] = h;
        lo[off] = l;
        int64_t offT;
        if (r < ns8) {
            offT = base + (tc::core_offset(c, r, icores) >> 2);
        } else {
            const int q = r - ns8;
            offT = base + (int64_t)ns8 * ns8 + (int64_t)(q >> 5) * 32 * ns8 + (tc::core_offset(c, q & 31, 8) >> 2);
        }
        hiT[offT] = h;
        loT[offT] = l;
    }
}

}  // namespace

cudaError_t configure_tc_kernels() {
    cudaError_t e = cudaFuncSetAttribute(k_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdTcSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdTcSmem);
}

void launch_fwd_level_tc(const SolveArgs<float>& args, int32_t t0, int32_t ntasks, const CUtensorMap& rows_map,
                         cudaStream_t st) {
    if (ntasks <= 0 || args.K <= 0) return;
    SolveArgs<float> a = args;
    a.stage = TC_STAGE;
    const int ntiles = a.K / TCN;
    k_fwd_tc<<<(unsigned)(ntasks * ntiles), NT, kFwdTcSmem, st>>>(a, t0, ntiles, rows_map);
}

void launch_bwd_level_tc(const SolveArgs<float>& a, int32_t t0, int32_t ntasks, const CUtensorMap& rows_map,
                         cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    const int ntiles = a.K / TCN;
    k_bwd_tc<<<(unsigned)(ntasks * ntiles), NT, kBwdTcSmem, st>>>(a, t0, ntiles, rows_map);
}

void launch_build_cores(const DevPlan& p, const double* val, const double* inv, const int64_t* core_ptr, float* hi,
                        float* lo, float* hiT, float* loT, cudaStream_t st) {
    if (p.nsuper <= 0) return;
    k_build_cores<<<p.nsuper, 256, 0, st>>>(p, val, inv, core_ptr, hi, lo, hiT, loT);
}

int make_rows_map(CUtensorMap* map, const float* base, int64_t n, int32_t K) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return 1;
        encode = reinterpret_cast<Encode>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)K * sizeof(float)};
    const cuuint32_t box[2] = {32, 64};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 2;
}

}  // namespace fcw
