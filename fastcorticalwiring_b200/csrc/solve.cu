// Multi-right-hand-side supernodal triangular solves, one etree level per launch.
//
// Right-hand sides R and results B are n x K row-major (a vertex row holds K
// contiguous right-hand sides). The forward sweep reads R and writes the
// forward result into B; the backward sweep turns B into the solution in
// place. R is never written, because several CTAs of one supernode (its row
// chunks) each rebuild that supernode's right-hand side. A CTA
// owns one task of one supernode and a 64-column tile of the right-hand sides;
// all dense work is 64 x 64 register-tiled products staged in shared memory
// (256 threads, 4 x 4 outputs per thread).
//
// Forward (leaves -> root), multifrontal: supernode s forms
//   W   = b_s - sum of the children's update rows that land on s's columns
//   X_s = inv(L_ss) W                                   (written to B)
//   U_s = (children's update rows that land on s's structure) + L_rs X_s
// and leaves U_s (nr x K) for its parent. Children are gathered through a
// per-front-row list in ascending child order, so results are deterministic.
// A supernode with a long structure is split into 64-row tasks that each
// recompute X_s (cheap) and write their own rows of U_s.
//
// Backward (root -> leaves): C = y_s - L_rs^T X_r (gather of the structure
// rows, which belong to ancestors and are final), X_s = inv(L_ss)^T C. Long
// structures are split over several CTAs (split-K); each writes a partial sum,
// and the CTA that arrives last (atomic ticket, no waiting) adds the partials in
// split order and finishes the supernode.
//
// Heat right-hand sides are columns of the identity: the forward sweep builds
// them from the source list, and only supernodes on a source's path to the
// root (`reach`) are solved; the others' forward results are zero.
#include "kernels.cuh"

namespace fcw {

namespace {

constexpr int TR = kMaxWidth;   // rows of a tile (= widest supernode)
constexpr int KT = kRhsTile;    // right-hand sides per CTA
constexpr int LDS = KT + 1;
constexpr int LDP = TR + 1;
constexpr int RC = 32;          // structure rows per staged chunk in the backward gather
constexpr int kGatherStage = 1024;  // gather entries staged in shared memory per forward task

template <typename T>
__device__ __forceinline__ void zero(T (&acc)[4][4]) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
}

// acc[a][b] += sum_{j<depth} A[(ty+16a)*lda + j] * Bm[j*ldb + tx+16b]   (A rows, B rows in smem)
template <typename T>
__device__ __forceinline__ void mma_rows(T (&acc)[4][4], const T* A, int lda, const T* Bm, int ldb, int depth,
                                         int ty, int tx) {
    for (int j = 0; j < depth; ++j) {
        T w[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) w[b] = Bm[j * ldb + tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const T l = A[(ty + 16 * a) * lda + j];
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] += l * w[b];
        }
    }
}

// acc[a][b] += sum_{j<depth} A[j*lda + ty+16a] * Bm[j*ldb + tx+16b]   (A transposed)
template <typename T>
__device__ __forceinline__ void mma_cols(T (&acc)[4][4], const T* A, int lda, const T* Bm, int ldb, int depth,
                                         int ty, int tx) {
    for (int j = 0; j < depth; ++j) {
        T w[4], l[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) w[b] = Bm[j * ldb + tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a) l[a] = A[j * lda + ty + 16 * a];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] += l[a] * w[b];
    }
}

// rows [f0, f0+nf) of supernode s's front (fb = its first front row): out[r][c] =
// init(r, k) + sign * sum of the children's update rows listed for front row f0+r,
// for this CTA's 64 columns. Entries are staged in shared memory when they fit;
// each thread owns one column and every 4th row, so its loads are independent.
template <typename T, typename Init>
__device__ __forceinline__ void gather_rows(const SolveArgs<T>& a, int64_t fb, int f0, int nrows, T* out, Init init,
                                            T sign, int* gsrc, int* gchild, int* grs) {
    const int tid = threadIdx.x;
    const int K = a.K, k0 = blockIdx.y * KT;
    const int eb = a.gm_ptr[fb + f0];
    const int E = a.gm_ptr[fb + f0 + nrows] - eb;
    const bool staged = E <= kGatherStage;
    for (int r = tid; r <= nrows; r += 256) grs[r] = a.gm_ptr[fb + f0 + r] - eb;
    if (staged)
        for (int e = tid; e < E; e += 256) {
            gsrc[e] = a.gm_src[eb + e];
            gchild[e] = a.gm_child[eb + e];
        }
    __syncthreads();
    const int c = tid & (KT - 1), k = k0 + c;
    for (int r = tid / KT; r < nrows; r += 256 / KT) {
        T v = init(r, k);
        const int e0 = grs[r], e1 = grs[r + 1];
        for (int e = e0; e < e1; ++e) {
            const int src = staged ? gsrc[e] : a.gm_src[eb + e];
            const int ch = staged ? gchild[e] : a.gm_child[eb + e];
            if (a.reach && !a.reach[ch]) continue;
            v += sign * a.U[(int64_t)src * K + k];
        }
        out[r * LDS + c] = v;
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwd(SolveArgs<T> a, int32_t t0) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* Ws = reinterpret_cast<T*>(smraw);   // TR x LDS
    T* Xs = Ws + TR * LDS;                  // TR x LDS
    T* Ms = Xs + TR * LDS;                  // TR x LDP
    __shared__ int gsrc[kGatherStage], gchild[kGatherStage], grs[TR + 1];
    const int2 task = a.tasks[t0 + blockIdx.x];
    const int s = task.x, chunk = task.y;
    if (a.reach && !a.reach[s]) return;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ty = tid >> 4, tx = tid & 15;
    const int K = a.K, k0 = blockIdx.y * KT;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], nr = m - ns;
    const int64_t fb = p.sn_rowptr[s];

    // W = right-hand side of s's columns minus the children's updates on them.
    // The gather entries of these rows are contiguous; stage them in shared memory
    // so every (row, column) accumulation issues independent, coalesced loads.
    gather_rows<T>(a, fb, 0, ns, Ws, [&](int f, int k) -> T {
        if (a.delta_src) return (a.delta_src[k] == c0 + f) ? T(1) : T(0);
        return a.R[(int64_t)(c0 + f) * K + k];
    }, T(-1), gsrc, gchild, grs);
    const T* inv = a.inv + p.sn_invptr[s];
    for (int e = tid; e < ns * ns; e += 256) {
        const int i = e / ns, j = e - i * ns;
        Ms[i * LDP + j] = inv[e];
    }
    __syncthreads();
    T acc[4][4];
    zero(acc);
    mma_rows(acc, Ms, LDP, Ws, LDS, ns, ty, tx);
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int t = ty + 16 * aa;
        if (t < ns)
#pragma unroll
            for (int b = 0; b < 4; ++b) Xs[t * LDS + tx + 16 * b] = acc[aa][b];
    }
    __syncthreads();
    if (chunk == 0) {
        for (int t = warp; t < ns; t += 8) {
            a.B[(int64_t)(c0 + t) * K + k0 + lane] = Xs[t * LDS + lane];
            a.B[(int64_t)(c0 + t) * K + k0 + lane + 32] = Xs[t * LDS + lane + 32];
        }
    }
    if (nr == 0) return;
    const int q0 = chunk * TR;
    const int nq = min(TR, nr - q0);
    const T* P = a.val + p.sn_valptr[s] + (int64_t)(ns + q0) * ns;
    for (int e = tid; e < nq * ns; e += 256) {
        const int r = e / ns, j = e - r * ns;
        Ms[r * LDP + j] = P[e];
    }
    __syncthreads();
    zero(acc);
    mma_rows(acc, Ms, LDP, Xs, LDS, ns, ty, tx);
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int r = ty + 16 * aa;
        if (r < nq)
#pragma unroll
            for (int b = 0; b < 4; ++b) Ws[r * LDS + tx + 16 * b] = acc[aa][b];
    }
    __syncthreads();
    // U_s rows of this chunk = L_rs X_s (in Ws) + the children's updates landing on them
    gather_rows<T>(a, fb, ns + q0, nq, Ws, [&](int r, int k) -> T { return Ws[r * LDS + (k - k0)]; }, T(1), gsrc,
                   gchild, grs);
    T* Us = a.U + (a.uoff[s] + q0) * (int64_t)K;
    for (int e = tid; e < nq * KT; e += 256) {
        const int r = e / KT, c = e - r * KT;
        Us[(int64_t)r * K + k0 + c] = Ws[r * LDS + c];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_bwd(SolveArgs<T> a, int32_t t0) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* Ps = reinterpret_cast<T*>(smraw);   // RC x LDP  panel rows of the chunk
    T* Xg = Ps + RC * LDP;                  // RC x LDS  gathered solution rows
    T* Cs = Xg + RC * LDS;                  // TR x LDS
    T* Ms = Ps;                             // TR x LDP  inverse diagonal block, after the gather
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

    T acc[4][4];
    zero(acc);
    for (int qq = q0; qq < q1; qq += RC) {
        const int nc = min(RC, q1 - qq);
        for (int e = tid; e < nc * ns; e += 256) {
            const int r = e / ns, j = e - r * ns;
            Ps[r * LDP + j] = P[(int64_t)(ns + qq + r) * ns + j];
        }
        for (int e = tid; e < nc * KT; e += 256) {
            const int r = e / KT, c = e - r * KT;
            Xg[r * LDS + c] = a.B[(int64_t)rows[ns + qq + r] * K + k0 + c];
        }
        __syncthreads();
        mma_cols(acc, Ps, LDP, Xg, LDS, nc, ty, tx);
        __syncthreads();
    }

    const bool zero_y = a.reach && !a.reach[s];
    if (nspl > 1) {
        T* part = a.part + a.poff[s] * (int64_t)TR * K;
#pragma unroll
        for (int aa = 0; aa < 4; ++aa) {
            const int t = ty + 16 * aa;
            if (t < ns)
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    part[((int64_t)split * TR + t) * K + k0 + tx + 16 * b] = acc[aa][b];
        }
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
                for (int b = 0; b < 4; ++b) {
                    T sum = T(0);
                    for (int sp = 0; sp < nspl; ++sp)
                        sum += __ldcg(&part[((int64_t)sp * TR + t) * K + k0 + tx + 16 * b]);
                    acc[aa][b] = sum;
                }
        }
        if (tid == 0) a.counters[(int64_t)s * a.ktiles + blockIdx.y] = 0;
    }
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int t = ty + 16 * aa;
        if (t < ns)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int c = tx + 16 * b;
                const T y = zero_y ? T(0) : a.B[(int64_t)(c0 + t) * K + k0 + c];
                Cs[t * LDS + c] = y - acc[aa][b];
            }
    }
    const T* inv = a.inv + p.sn_invptr[s];
    for (int e = tid; e < ns * ns; e += 256) {
        const int i = e / ns, j = e - i * ns;
        Ms[i * LDP + j] = inv[e];
    }
    __syncthreads();
    zero(acc);
    mma_cols(acc, Ms, LDP, Cs, LDS, ns, ty, tx);
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int t = ty + 16 * aa;
        if (t < ns)
#pragma unroll
            for (int b = 0; b < 4; ++b) a.B[(int64_t)(c0 + t) * K + k0 + tx + 16 * b] = acc[aa][b];
    }
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

template <typename T>
constexpr size_t fwd_smem() { return (size_t)(2 * TR * LDS + TR * LDP) * sizeof(T); }
template <typename T>
constexpr size_t bwd_smem() { return (size_t)(RC * LDP + RC * LDS + TR * LDS) * sizeof(T); }
static_assert(RC * LDP + RC * LDS >= TR * LDP, "the inverse tile aliases the gather staging area");

}  // namespace

cudaError_t configure_solve_kernels() {
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_fwd<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem<double>())))
        return e;
    if ((e = cudaFuncSetAttribute(k_fwd<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem<float>())))
        return e;
    if ((e = cudaFuncSetAttribute(k_bwd<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bwd_smem<double>())))
        return e;
    return cudaFuncSetAttribute(k_bwd<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bwd_smem<float>());
}

template <typename T>
void launch_fwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    k_fwd<T><<<dim3(ntasks, a.K / KT), 256, fwd_smem<T>(), st>>>(a, t0);
}

template <typename T>
void launch_bwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    k_bwd<T><<<dim3(ntasks, a.K / KT), 256, bwd_smem<T>(), st>>>(a, t0);
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
