// One right-hand side (the single-source drop-in): the heat and Poisson solves of
// one source without a launch per elimination-tree level.
//
// Layouts. Per supernode s the stacked block A_s = [inv(L_ss); Q_s] (m x ns: the
// inverse diagonal block above the panel Q_s = L_rs inv(L_ss)) is stored twice, in the
// order each sweep reads it. Forward: 64-row chunks, each column-major with an even
// column stride rcp (the chunk's rows rounded up to even), element (r, j) of chunk c at
// c*64*ns + j*rcp + r. Backward: column-major over all rows with stride mp = even(m),
// element (R, j) at j*mp + R, so a strip of whole columns is contiguous. Every chunk and
// every strip starts on a 16-byte boundary and is moved into shared memory by one bulk
// copy (cp.async.bulk, completing on an mbarrier): a few large copies, since a CTA's
// bulk copies are served one after another. Threads that own consecutive rows read
// consecutive words.
//
// Forward (leaves -> root), supernode s, W = b_s - (children's update entries on s's columns):
//   X_s = inv(L_ss) W -> B,   U_s = Q_s W + (children's update entries on s's structure rows)
// Backward (root -> leaves): X_s = inv(L_ss)^T y_s - Q_s^T X_r = A_s^T [y_s; -X_r].
//
// Tasks. A forward task is up to three chunks of one supernode's rows (it forms W
// itself, so a supernode's tasks need nothing from each other); a backward task is a
// strip of whole columns over all rows (it finishes its columns of X_s, so there is no
// partial sum to combine). Either fits in 96 KB of shared memory, so a CTA copies all of
// its task's panel data before it waits for anything: after the dependency resolves,
// only the small vector gathers and the products from shared memory remain.
//
// Scheduling. A persistent CTA takes the next ticket, starts the task's bulk copies
// and loads the indices of the values it depends on, then reads those values: the
// children's update entries (forward) or the ancestors' solution entries (backward).
// Both arrays hold a pending bit pattern (all ones, a NaN that no arithmetic
// produces) when the sweep starts, and each entry is written once, by one 8-byte
// store, so a reader polls each entry until it is no longer pending: the value is the
// signal, with no flags or fences. Tickets follow the level order (leaves first
// forward, reversed backward), so a task only waits for tasks whose tickets were taken
// earlier by CTAs already running: progress does not depend on the grid size or on
// residency. Every wait is bounded (%globaltimer); one that gives up raises
// KERR_TIMEOUT, after which every other wait returns at once, so a sweep always ends.
//
// The heat right-hand side is one column of the identity: only the supernodes on the
// source's path to the root have nonzero forward results (the others' are zero in B
// beforehand), so the heat forward runs the forward tasks of the path alone.
#include <algorithm>
#include <vector>

#include "kernels.cuh"
#include "tc.cuh"

namespace fcw {

namespace {

constexpr int NTN = 256;                        // threads per CTA
constexpr int CR = kNarrowRows;                 // stacked rows per chunk
constexpr int kChunk = CR * kMaxWidth;          // doubles of a full chunk (32 KB)
constexpr int kTaskDoubles = kNarrowTaskDoubles; // panel data of one task (96 KB)
constexpr int FC = kTaskDoubles / kChunk;       // chunks of a forward task
constexpr uint64_t kWaitNs = 1000000000ull;

constexpr long long kPending = -1;  // bit pattern of an entry not yet written

__device__ __forceinline__ double ld_relaxed(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool pending(double v) { return __double_as_longlong(v) == kPending; }
__device__ __forceinline__ bool given_up(const int* err) {
    return (*reinterpret_cast<const volatile int*>(err) & KERR_TIMEOUT) != 0;
}

// v[k] = base[idx[k]] for the k in `active` (others 0), entries other CTAs of this launch
// write: each is polled until it is no longer pending. False (KERR_TIMEOUT raised) after
// about kWaitNs, or at once when another wait has already given up.
template <int N>
__device__ bool read_written(const double* base, const int (&idx)[N], unsigned active, double (&v)[N], int* err,
                             unsigned sleep_ns = 64) {
    unsigned pend = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        v[k] = 0.0;
        if ((active >> k) & 1u) {
            v[k] = ld_relaxed(base + idx[k]);
            if (pending(v[k])) pend |= 1u << k;
        }
    }
    if (!pend) return true;
    const uint64_t t0 = tc::global_ns();
    for (;;) {
#pragma unroll
        for (int k = 0; k < N; ++k)
            if ((pend >> k) & 1u) {
                v[k] = ld_relaxed(base + idx[k]);
                if (!pending(v[k])) pend &= ~(1u << k);
            }
        if (!pend) return true;
        if (given_up(err)) return false;
        if (tc::global_ns() - t0 > kWaitNs) {
            atomicOr(err, KERR_TIMEOUT);
            return false;
        }
        __nanosleep(sleep_ns);
    }
}
__device__ __forceinline__ double read_one(const double* p, int* err, unsigned sleep_ns = 64) {
    const int idx[1] = {0};
    double v[1];
    read_written<1>(p, idx, 1u, v, err, sleep_ns);
    return v[0];
}

// A bulk copy that does not land in time raises KERR_TIMEOUT; the second bounded wait
// lets a late copy finish before its buffer is reused.
__device__ __forceinline__ void wait_copies(uint64_t* bar, uint32_t parity, int* err) {
    if (!tc::mbar_wait(bar, parity)) {
        atomicOr(err, KERR_TIMEOUT);
        tc::mbar_wait(bar, parity);
    }
}

// Programmatic dependent launch: the next kernel of the stream may start (its CTAs take
// tickets and start their panel copies, which read nothing this kernel writes) while this
// one finishes; it reads this kernel's results only after griddepcontrol.wait.
__device__ __forceinline__ void allow_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void wait_predecessor() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__host__ __device__ __forceinline__ int chunk_rows(int m, int c) { return min(CR, m - CR * c); }
__host__ __device__ __forceinline__ int even(int x) { return (x + 1) & ~1; }

// Task shapes of the host's task lists. A front of at most FC chunks is one forward
// task; a larger one (the separators near the root, on the critical path) is one task
// per chunk, so its rows are formed in parallel. Backward strips hold as many whole
// columns as fit, at most 8 (one per warp) for fronts of more than 256 rows, in equal
// widths.
inline int fwd_chunks_per_task(int m) {
    const int nch = (m + CR - 1) / CR;
    return nch <= FC ? nch : 1;
}
inline int bwd_strip_width(int ns, int m) {
    const int fit = std::max(1, kTaskDoubles / even(m)), per = m > 256 ? std::min(8, fit) : fit;
    const int g = (ns + per - 1) / per;
    return (ns + g - 1) / g;
}

// Forward product of one chunk: red[cp*CR + r] = sum over columns j = cp (mod 4) of
// A[r][j] w[j]. Warp w owns rows 32 (w & 1) + lane and column part w >> 1.
__device__ __forceinline__ void rows_times(const double* At, int rc, int rcp, int ns, const double* w,
                                           double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r = (warp & 1) * 32 + lane, cp = warp >> 1;
    if (r < rc) {
        double acc = 0.0;
        for (int j = cp; j < ns; j += 4) acc = fma(At[j * rcp + r], w[j], acc);
        red[cp * CR + r] = acc;
    }
}
__device__ __forceinline__ double row_sum(const double* red, int r) {
    return (red[r] + red[CR + r]) + (red[2 * CR + r] + red[3 * CR + r]);
}

// Both layouts of one factor; the two arrays have the same size and offsets (at_ptr).
__global__ void k_build_narrow(DevPlan p, const double* __restrict__ val, const double* __restrict__ inv,
                               const int64_t* __restrict__ at_ptr, double* __restrict__ at_f,
                               double* __restrict__ at_b) {
    const int s = blockIdx.x;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], mp = even(m);
    const double* P = val + p.sn_valptr[s];
    const double* I = inv + p.sn_invptr[s];
    double* F = at_f + at_ptr[s];
    double* Bk = at_b + at_ptr[s];
    for (int e = threadIdx.x; e < m * ns; e += blockDim.x) {
        const int R = e / ns, j = e - R * ns;
        const double x = R < ns ? (j <= R ? I[R * ns + j] : 0.0) : P[R * ns + j];  // panel rows >= ns hold Q_s
        const int c = R / CR, r = R - c * CR;
        F[(int64_t)c * CR * ns + j * even(chunk_rows(m, c)) + r] = x;
        Bk[(int64_t)j * mp + R] = x;
    }
}

constexpr int kPre = 4;  // gather entries per row whose indices are loaded before the values

// A row's gather list (entries [e0, e1) of gm_*): the first kPre indices are loaded
// before any value is read.
struct RowGather {
    int e0 = 0, e1 = 0;
    int idx[kPre];
    int child[kPre];
};
template <bool DELTA>
__device__ __forceinline__ void gather_open(const NarrowArgs& a, int64_t frow, RowGather& g) {
    g.e0 = a.gm_ptr[frow];
    g.e1 = a.gm_ptr[frow + 1];
#pragma unroll
    for (int k = 0; k < kPre; ++k) {
        const bool in = g.e0 + k < g.e1;
        g.idx[k] = in ? a.gm_src[g.e0 + k] : 0;
        if (DELTA) g.child[k] = in ? a.gm_child[g.e0 + k] : -1;
    }
}
// Sum of the row's update entries (heat: only those of the path child `prev`, the
// others are never written), in list order, each read once it is written.
template <bool DELTA>
__device__ __forceinline__ double gather_sum(const NarrowArgs& a, const RowGather& g, int prev) {
    unsigned active = 0;
#pragma unroll
    for (int k = 0; k < kPre; ++k)
        if (g.e0 + k < g.e1 && (!DELTA || g.child[k] == prev)) active |= 1u << k;
    double v[kPre];
    read_written<kPre>(a.U, g.idx, active, v, a.err);
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kPre; ++k)
        if ((active >> k) & 1u) sum += v[k];
    for (int e = g.e0 + kPre; e < g.e1; ++e)
        if (!DELTA || a.gm_child[e] == prev) sum += read_one(a.U + a.gm_src[e], a.err);
    return sum;
}

// Forward tasks. DELTA: the heat solve of the identity column of a.order's source, over
// the tasks of its path (a.order: the source's elimination index, the path's task
// count, then (task, previous supernode on the path) pairs bottom-up); otherwise every
// task of a.tasks. U is pending on entry.
template <bool DELTA>
__global__ void __launch_bounds__(NTN, 2) k_fwd_tasks(NarrowArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double* dat = reinterpret_cast<double*>(smraw);  // the task's chunks, kChunk apart
    double* W = dat + kTaskDoubles;
    double* gs = W + kMaxWidth;                       // gathered children's entries of the task's rows
    double* red = gs + FC * CR;
    __shared__ uint64_t bar;
    __shared__ int task, task_prev;
    const int tid = threadIdx.x;
    const DevPlan& p = a.p;
    allow_dependents();
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    const int total = DELTA ? a.order[1] : a.ntasks;
    const int se = DELTA ? a.order[0] : -1;
    uint32_t parity = 0;
    bool inputs_ready = false;  // the previous kernel's results (right-hand side) are visible
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(a.ticket, 1);
            const bool stop = t >= total || given_up(a.err);
            task = stop ? -1 : (DELTA ? a.order[2 + 2 * t] : t);
            task_prev = (!stop && DELTA) ? a.order[3 + 2 * t] : -1;
        }
        __syncthreads();
        const int ti = task, prev = task_prev;
        if (ti < 0) break;
        const int4 tk = a.tasks[ti];
        const int s = tk.x, cb = tk.y, nc = tk.z;
        const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s];
        const int64_t fb = p.sn_rowptr[s];
        const int R0 = cb * CR, R1 = min(m, (cb + nc) * CR), Rs = max(R0, ns);
        if (tid == 0) {
            uint32_t bytes = 0;
            for (int k = 0; k < nc; ++k) bytes += (uint32_t)(ns * even(chunk_rows(m, cb + k))) * 8u;
            tc::mbar_arrive_expect_tx(&bar, bytes);
            for (int k = 0; k < nc; ++k)
                tc::bulk_load(dat + k * kChunk, a.at + a.at_ptr[s] + (int64_t)(cb + k) * CR * ns,
                              (uint32_t)(ns * even(chunk_rows(m, cb + k))) * 8u, &bar);
        }
        if (!inputs_ready) {
            wait_predecessor();
            inputs_ready = true;
        }
        // thread t < 64: column row t (W); thread 64 + i: structure row Rs + i of the task
        const int row = tid < kMaxWidth ? (tid < ns ? tid : -1)
                                        : (Rs + tid - kMaxWidth < R1 ? Rs + tid - kMaxWidth : -1);
        if (row >= 0) {
            RowGather g;
            gather_open<DELTA>(a, fb + row, g);
            const double rhs = tid < kMaxWidth ? (DELTA ? (c0 + row == se ? 1.0 : 0.0) : a.R[c0 + row]) : 0.0;
            const double sum = gather_sum<DELTA>(a, g, prev);
            if (tid < kMaxWidth) W[row] = rhs - sum;
            else gs[row - R0] = sum;
        }
        __syncthreads();
        wait_copies(&bar, parity, a.err);
        parity ^= 1u;
        for (int k = 0; k < nc; ++k) {
            const int rc = chunk_rows(m, cb + k);
            rows_times(dat + k * kChunk, rc, even(rc), ns, W, red);
            __syncthreads();
            if (tid < rc) {
                const int R = (cb + k) * CR + tid;
                const double x = row_sum(red, tid);
                if (R < ns) a.B[c0 + R] = x;
                else a.U[a.uoff[s] + R - ns] = x + gs[R - R0];
            }
            __syncthreads();
        }
    }
}

// Backward tasks: X (pending on entry) = the solution, from the forward result B.
__global__ void __launch_bounds__(NTN, 2) k_bwd_tasks(NarrowArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double* dat = reinterpret_cast<double*>(smraw);  // the task's column strips, chunk after chunk
    double* v = dat + kTaskDoubles;                   // [y_s; -X_r], max_m entries
    __shared__ uint64_t bar;
    __shared__ int task;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const DevPlan& p = a.p;
    allow_dependents();
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    uint32_t parity = 0;
    bool inputs_ready = false;  // the previous kernel's results (forward result) are visible
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(a.ticket, 1);
            task = (t >= a.ntasks || given_up(a.err)) ? -1 : t;
        }
        __syncthreads();
        const int ti = task;
        if (ti < 0) break;
        const int4 tk = a.tasks[ti];
        const int s = tk.x, j0 = tk.y, nj = tk.z - tk.y;
        const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], mp = even(m);
        const int32_t* rows = p.rows + p.sn_rowptr[s];
        if (tid == 0) {  // the strip: columns [j0, j0 + nj) over all rows, contiguous
            const uint32_t bytes = (uint32_t)(nj * mp) * 8u;
            tc::mbar_arrive_expect_tx(&bar, bytes);
            tc::bulk_load(dat, a.at + a.at_ptr[s] + (int64_t)j0 * mp, bytes, &bar);
        }
        if (!inputs_ready) {
            wait_predecessor();
            inputs_ready = true;
        }
        // The parent's columns come first among the structure rows (its first column is the
        // smallest structure row) and are written last, just before this task can run: warp 0
        // polls them with a short back-off. The other ancestors' entries, written earlier,
        // are polled by the other warps with a long one, so few requests reach the L2 slices
        // that hold the entries being produced.
        {
            const int par = p.sn_parent[s];
            const int pend = par >= 0 ? p.sn_c0[par + 1] : 0;  // one past the parent's last column
            if (warp == 0) {
                for (int R = ns + lane; R < min(m, ns + kMaxWidth); R += 32)
                    if (rows[R] < pend) v[R] = -read_one(a.X + rows[R], a.err, 32);
            } else {
                for (int R = tid - 32; R < m; R += NTN - 32) {
                    if (R < ns) v[R] = __ldcg(a.B + c0 + R);
                    else if (rows[R] >= pend) v[R] = -read_one(a.X + rows[R], a.err, 256);
                }
            }
        }
        __syncthreads();
        wait_copies(&bar, parity, a.err);
        parity ^= 1u;
        // warp w owns the strip's columns w + 8 jj; lanes walk the rows
        double acc[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) acc[jj] = 0.0;
        for (int R = lane; R < m; R += 32) {
            const double xv = v[R];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const int jl = warp + 8 * jj;
                if (jl < nj) acc[jj] = fma(dat[jl * mp + R], xv, acc[jj]);
            }
        }
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            double xs = acc[jj];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) xs += __shfl_xor_sync(0xffffffffu, xs, o);
            const int jl = warp + 8 * jj;
            if (lane == 0 && jl < nj) a.X[c0 + j0 + jl] = xs;
        }
        __syncthreads();  // v and the strips are free for the next task
    }
}

// The source's field in the caller's vertex order, shifted so the source is at zero.
__global__ void k_field_out_one(int32_t n, const double* __restrict__ Y, const int32_t* __restrict__ src_elim,
                                const int32_t* __restrict__ iperm, double* __restrict__ out) {
    const int se = *src_elim;
    if (se < 0) return;
    const double y0 = Y[se];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = Y[iperm[i]] - y0;
}

size_t fwd_bytes() { return (size_t)(kTaskDoubles + kMaxWidth + FC * CR + 4 * CR) * sizeof(double); }
size_t bwd_bytes(int max_m) { return (size_t)(kTaskDoubles + even(max_m)) * sizeof(double); }

}  // namespace

int64_t narrow_layout(const int32_t* sn_c0, const int32_t* sn_m, int32_t nsuper, int64_t* at_ptr) {
    int64_t off = 0;
    for (int32_t s = 0; s < nsuper; ++s) {
        const int64_t ns = sn_c0[s + 1] - sn_c0[s], m = sn_m[s];
        const int64_t nch = (m + CR - 1) / CR, last = m - CR * (nch - 1);
        at_ptr[s] = off;
        off += CR * ns * (nch - 1) + ns * even((int)last);
    }
    at_ptr[nsuper] = off;
    return off;
}

void narrow_tasks(const int32_t* sn_c0, const int32_t* sn_m, int32_t nsuper, const int32_t* level_nodes,
                  std::vector<int4>& fwd, std::vector<int32_t>& fwd_first, std::vector<int32_t>& nfwd,
                  std::vector<int4>& bwd, std::vector<int32_t>& nbwd) {
    fwd.clear();
    bwd.clear();
    fwd_first.assign((size_t)nsuper, 0);
    nfwd.assign((size_t)nsuper, 0);
    nbwd.assign((size_t)nsuper, 0);
    for (int32_t q = 0; q < nsuper; ++q) {  // level order: leaves first
        const int32_t s = level_nodes[q], m = sn_m[s];
        const int32_t nch = (m + CR - 1) / CR, per = fwd_chunks_per_task(m);
        fwd_first[s] = (int32_t)fwd.size();
        for (int32_t c = 0; c < nch; c += per) fwd.push_back(make_int4(s, c, std::min(per, nch - c), 0));
        nfwd[s] = (int32_t)fwd.size() - fwd_first[s];
    }
    for (int32_t q = nsuper - 1; q >= 0; --q) {  // reversed level order: root first
        const int32_t s = level_nodes[q], ns = sn_c0[s + 1] - sn_c0[s], m = sn_m[s];
        const int32_t w = bwd_strip_width(ns, m);
        for (int32_t j = 0; j < ns; j += w) bwd.push_back(make_int4(s, j, std::min(ns, j + w), 0));
        nbwd[s] = (ns + w - 1) / w;
    }
}

void launch_build_narrow(const DevPlan& p, const double* val, const double* inv, const int64_t* at_ptr,
                         double* at_f, double* at_b, cudaStream_t st) {
    if (p.nsuper > 0) k_build_narrow<<<p.nsuper, 256, 0, st>>>(p, val, inv, at_ptr, at_f, at_b);
}

cudaError_t configure_narrow_kernels(int max_m, int num_sms, NarrowLaunch* L) {
    if (max_m > kTaskDoubles) return cudaErrorInvalidValue;  // a backward strip must hold one column
    L->fwd_smem = fwd_bytes();
    L->bwd_smem = bwd_bytes(max_m);
    if (L->bwd_smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_fwd_tasks<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)L->fwd_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fwd_tasks<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->fwd_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_bwd_tasks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->bwd_smem);
    int per_sm = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fwd_tasks<false>, NTN, L->fwd_smem);
    L->grid_fwd = std::max(1, per_sm) * num_sms;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bwd_tasks, NTN, L->bwd_smem);
    L->grid_bwd = std::max(1, per_sm) * num_sms;
    return e;
}

namespace {
// overlap: launched as a programmatic dependent of the stream's previous kernel
template <typename Kern>
void launch_sweep(Kern kern, int grid, size_t smem, bool overlap, const NarrowArgs& a, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NTN);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = overlap ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, a);
}
}  // namespace

void launch_fwd_narrow(const NarrowArgs& a, bool delta, bool overlap, const NarrowLaunch& L, cudaStream_t st) {
    if (delta) launch_sweep(k_fwd_tasks<true>, L.grid_fwd, L.fwd_smem, overlap, a, st);
    else launch_sweep(k_fwd_tasks<false>, L.grid_fwd, L.fwd_smem, overlap, a, st);
}
void launch_bwd_narrow(const NarrowArgs& a, bool overlap, const NarrowLaunch& L, cudaStream_t st) {
    launch_sweep(k_bwd_tasks, L.grid_bwd, L.bwd_smem, overlap, a, st);
}
void launch_field_out_one(int32_t n, const double* Y, const int32_t* src_elim, const int32_t* iperm, double* out,
                          int num_sms, cudaStream_t st) {
    k_field_out_one<<<num_sms * 2, 256, 0, st>>>(n, Y, src_elim, iperm, out);
}

}  // namespace fcw
