// Multi-right-hand-side supernodal triangular solves, one etree level per launch.
//
// Right-hand sides R and results B are n x K row-major (a vertex row holds K
// contiguous right-hand sides). The forward sweep reads R and writes the
// forward result into B; the backward sweep turns B into the solution in
// place. R is never written, because several CTAs of one supernode (its row
// chunks) each rebuild that supernode's right-hand side. A CTA
// owns one task of one supernode and a 64-column tile of the right-hand sides;
// all dense work is register-tiled products staged in shared memory (256
// threads; a thread owns 4 rows x KT/16 columns). Column tiles are 64 wide in
// FP64 and 128 wide in FP32; the inverse diagonal block and the panel chunk of
// a forward task arrive by cp.async while the children's updates are gathered.
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
constexpr int LDP = TR + 1;     // leading dimension of panel / inverse tiles
constexpr int RC = 32;          // structure rows per staged chunk in the backward gather
constexpr int kGatherStage = 1024;  // gather entries staged in shared memory per forward task

template <typename T, int NB>
__device__ __forceinline__ void zero(T (&acc)[4][NB]) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[a][b] = T(0);
}

// acc[a][b] += sum_{j<depth} A[(ty+16a)*lda + j] * Bm[j*ldb + tx+16b]
template <typename T, int NB>
__device__ __forceinline__ void mma_rows(T (&acc)[4][NB], const T* A, int lda, const T* Bm, int ldb, int depth,
                                         int ty, int tx) {
    for (int j = 0; j < depth; ++j) {
        T w[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) w[b] = Bm[j * ldb + tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const T l = A[(ty + 16 * a) * lda + j];
#pragma unroll
            for (int b = 0; b < NB; ++b) acc[a][b] += l * w[b];
        }
    }
}

// acc[a][b] += sum_{j<depth} A[j*lda + ty+16a] * Bm[j*ldb + tx+16b]   (A transposed)
template <typename T, int NB>
__device__ __forceinline__ void mma_cols(T (&acc)[4][NB], const T* A, int lda, const T* Bm, int ldb, int depth,
                                         int ty, int tx) {
    for (int j = 0; j < depth; ++j) {
        T w[NB], l[4];
#pragma unroll
        for (int b = 0; b < NB; ++b) w[b] = Bm[j * ldb + tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a) l[a] = A[j * lda + ty + 16 * a];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < NB; ++b) acc[a][b] += l[a] * w[b];
    }
}

// Asynchronous global -> shared copy of one element (cp.async, L1-allocating).
template <typename T>
__device__ __forceinline__ void copy_async(T* smem, const T* gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Gather lists of front rows [f0, f0+nrows) of the supernode whose first front row
// is fb: each front row lists the children's update rows that land on it. The
// entries of consecutive rows are contiguous; they are staged in shared memory
// when they fit (staged = true), otherwise read from global memory.
struct Gather {
    int eb;
    bool staged;
};

template <typename T>
__device__ __forceinline__ Gather stage_entries(const SolveArgs<T>& a, int64_t fb, int f0, int nrows, int* gsrc,
                                                int* gchild, int* grs) {
    const int tid = threadIdx.x;
    Gather g;
    g.eb = a.gm_ptr[fb + f0];
    const int E = a.gm_ptr[fb + f0 + nrows] - g.eb;
    g.staged = E <= kGatherStage;
    for (int r = tid; r <= nrows; r += 256) grs[r] = a.gm_ptr[fb + f0 + r] - g.eb;
    if (g.staged)
        for (int e = tid; e < E; e += 256) {
            gsrc[e] = a.gm_src[g.eb + e];
            gchild[e] = a.gm_child[g.eb + e];
        }
    __syncthreads();
    return g;
}

// Sum of the listed children's update rows for front row r (relative), column k.
template <typename T>
__device__ __forceinline__ T gathered(const SolveArgs<T>& a, const Gather& g, int r, int k, const int* gsrc,
                                      const int* gchild, const int* grs) {
    T v = T(0);
    for (int e = grs[r]; e < grs[r + 1]; ++e) {
        const int src = g.staged ? gsrc[e] : a.gm_src[g.eb + e];
        const int ch = g.staged ? gchild[e] : a.gm_child[g.eb + e];
        if (a.reach && !a.reach[ch]) continue;
        v += a.U[(int64_t)src * a.K + k];
    }
    return v;
}

template <typename T, int KTT>
__global__ void __launch_bounds__(256) k_fwd(SolveArgs<T> a, int32_t t0) {
    constexpr int NB = KTT / 16, LDW = KTT + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* Wt = reinterpret_cast<T*>(smraw);   // TR x LDW: W, then X
    T* Li = Wt + TR * LDW;                  // TR x LDP: inverse diagonal block
    T* Pn = Li + TR * LDP;                  // TR x LDP: panel rows of this chunk
    __shared__ int gsrc[kGatherStage], gchild[kGatherStage], grs[TR + 1];
    const int2 task = a.tasks[t0 + blockIdx.x];
    const int s = task.x, chunk = task.y;
    if (a.reach && !a.reach[s]) return;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;
    const int K = a.K, k0 = blockIdx.y * KTT;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], nr = m - ns;
    const int64_t fb = p.sn_rowptr[s];
    const int q0 = chunk * TR;
    const int nq = nr > 0 ? min(TR, nr - q0) : 0;

    // the inverse block and this chunk's panel rows stream in while the gather runs
    const T* inv = a.inv + p.sn_invptr[s];
    for (int e = tid; e < ns * ns; e += 256) {
        const int i = e / ns, j = e - i * ns;
        copy_async(&Li[i * LDP + j], inv + e);
    }
    const T* P = a.val + p.sn_valptr[s] + (int64_t)(ns + q0) * ns;
    for (int e = tid; e < nq * ns; e += 256) {
        const int r = e / ns, j = e - r * ns;
        copy_async(&Pn[r * LDP + j], P + e);
    }

    // W = right-hand side of s's columns (identity columns are built in place,
    // stored ones arrive by cp.async with the blocks above), then minus the
    // children's updates on them
    if (a.delta_src) {
        for (int e = tid; e < ns * KTT; e += 256) {
            const int f = e / KTT, c = e - f * KTT;
            Wt[f * LDW + c] = (a.delta_src[k0 + c] == c0 + f) ? T(1) : T(0);
        }
    } else {
        for (int e = tid; e < ns * KTT; e += 256) {
            const int f = e / KTT, c = e - f * KTT;
            copy_async(&Wt[f * LDW + c], a.R + (int64_t)(c0 + f) * K + k0 + c);
        }
    }
    copy_async_commit();
    {
        const Gather g = stage_entries(a, fb, 0, ns, gsrc, gchild, grs);  // ends with a barrier
        copy_async_wait();
        __syncthreads();
        if (grs[ns] > 0) {  // some child update lands on these rows
            const int c = tid % KTT, k = k0 + c;
            for (int f = tid / KTT; f < ns; f += 256 / KTT)
                if (grs[f + 1] > grs[f]) Wt[f * LDW + c] -= gathered(a, g, f, k, gsrc, gchild, grs);
            __syncthreads();
        }
    }
    // X = inv(L_ss) W, written over W
    T acc[4][NB];
    zero(acc);
    mma_rows(acc, Li, LDP, Wt, LDW, ns, ty, tx);
    __syncthreads();
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int t = ty + 16 * aa;
        if (t < ns)
#pragma unroll
            for (int b = 0; b < NB; ++b) Wt[t * LDW + tx + 16 * b] = acc[aa][b];
    }
    __syncthreads();
    if (chunk == 0)
        for (int e = tid; e < ns * KTT; e += 256) {
            const int t = e / KTT, c = e - t * KTT;
            a.B[(int64_t)(c0 + t) * K + k0 + c] = Wt[t * LDW + c];
        }
    if (nq <= 0) return;
    // U_s rows of this chunk = L_rs X + the children's updates landing on them
    const Gather g = stage_entries(a, fb, ns + q0, nq, gsrc, gchild, grs);
    zero(acc);
    mma_rows(acc, Pn, LDP, Wt, LDW, ns, ty, tx);
    T* Us = a.U + (a.uoff[s] + q0) * (int64_t)K;
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int r = ty + 16 * aa;
        if (r < nq)
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int k = k0 + tx + 16 * b;
                Us[(int64_t)r * K + k] = acc[aa][b] + gathered(a, g, r, k, gsrc, gchild, grs);
            }
    }
}

template <typename T, int KTT>
__global__ void __launch_bounds__(256) k_bwd(SolveArgs<T> a, int32_t t0) {
    constexpr int NB = KTT / 16, LDW = KTT + 1;
    static_assert(RC * LDP + RC * LDW >= TR * LDP, "the inverse tile aliases the gather staging area");
    extern __shared__ __align__(16) unsigned char smraw[];
    T* Ps = reinterpret_cast<T*>(smraw);   // RC x LDP  panel rows of the chunk
    T* Xg = Ps + RC * LDP;                  // RC x LDW  gathered solution rows
    T* Cs = Xg + RC * LDW;                  // TR x LDW
    T* Ms = Ps;                             // TR x LDP  inverse diagonal block, after the gather
    __shared__ int last_arrival;
    __shared__ int rsh[RC];
    const int2 task = a.tasks[t0 + blockIdx.x];
    const int s = task.x, split = task.y;
    const DevPlan& p = a.p;
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;
    const int K = a.K, k0 = blockIdx.y * KTT;
    const int c0 = p.sn_c0[s], ns = p.sn_c0[s + 1] - c0, m = p.sn_m[s], nr = m - ns;
    const int nspl = a.nsplit[s];
    const int q0 = split * kSplitRows, q1 = min(nr, q0 + kSplitRows);
    const T* P = a.val + p.sn_valptr[s];
    const int32_t* rows = p.rows + p.sn_rowptr[s];

    T acc[4][NB];
    zero(acc);
    for (int qq = q0; qq < q1; qq += RC) {
        const int nc = min(RC, q1 - qq);
        if (tid < nc) rsh[tid] = rows[ns + qq + tid];
        for (int e = tid; e < nc * ns; e += 256) {
            const int r = e / ns, j = e - r * ns;
            copy_async(&Ps[r * LDP + j], P + (int64_t)(ns + qq + r) * ns + j);
        }
        __syncthreads();
        for (int e = tid; e < nc * KTT; e += 256) {
            const int r = e / KTT, c = e - r * KTT;
            copy_async(&Xg[r * LDW + c], a.B + (int64_t)rsh[r] * K + k0 + c);
        }
        copy_async_commit();
        copy_async_wait();
        __syncthreads();
        mma_cols(acc, Ps, LDP, Xg, LDW, nc, ty, tx);
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
                for (int b = 0; b < NB; ++b)
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
                for (int b = 0; b < NB; ++b) {
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
            for (int b = 0; b < NB; ++b) {
                const int c = tx + 16 * b;
                const T y = zero_y ? T(0) : a.B[(int64_t)(c0 + t) * K + k0 + c];
                Cs[t * LDW + c] = y - acc[aa][b];
            }
    }
    const T* inv = a.inv + p.sn_invptr[s];
    for (int e = tid; e < ns * ns; e += 256) {
        const int i = e / ns, j = e - i * ns;
        Ms[i * LDP + j] = inv[e];
    }
    __syncthreads();
    zero(acc);
    mma_cols(acc, Ms, LDP, Cs, LDW, ns, ty, tx);
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
        const int t = ty + 16 * aa;
        if (t < ns)
#pragma unroll
            for (int b = 0; b < NB; ++b) a.B[(int64_t)(c0 + t) * K + k0 + tx + 16 * b] = acc[aa][b];
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

template <typename T, int KTT>
constexpr size_t fwd_smem() { return (size_t)(TR * (KTT + 1) + 2 * TR * LDP) * sizeof(T); }
template <typename T, int KTT>
constexpr size_t bwd_smem() { return (size_t)(RC * LDP + RC * (KTT + 1) + TR * (KTT + 1)) * sizeof(T); }

// Widest column tile each precision uses when K allows it.
template <typename T>
constexpr int wide_tile() { return sizeof(T) == 4 ? 128 : 64; }

template <typename T, int KTT>
cudaError_t set_smem() {
    cudaError_t e = cudaFuncSetAttribute(k_fwd<T, KTT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fwd_smem<T, KTT>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_bwd<T, KTT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bwd_smem<T, KTT>());
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
        k_fwd<T, W><<<dim3(ntasks, a.K / W), 256, fwd_smem<T, W>(), st>>>(a, t0);
    else
        k_fwd<T, 64><<<dim3(ntasks, a.K / 64), 256, fwd_smem<T, 64>(), st>>>(a, t0);
}

template <typename T>
void launch_bwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, cudaStream_t st) {
    if (ntasks <= 0 || a.K <= 0) return;
    constexpr int W = wide_tile<T>();
    if (W != 64 && a.K % W == 0)
        k_bwd<T, W><<<dim3(ntasks, a.K / W), 256, bwd_smem<T, W>(), st>>>(a, t0);
    else
        k_bwd<T, 64><<<dim3(ntasks, a.K / 64), 256, bwd_smem<T, 64>(), st>>>(a, t0);
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
