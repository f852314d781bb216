// Multi-right-hand-side supernodal triangular solves, one etree level per launch.
//
// B is n x K row-major (one vertex row holds K contiguous right-hand sides),
// updated in place: right-hand side -> forward result -> solution. A CTA owns
// one (supernode, 32-column slice) pair; lane = right-hand side, so every
// vertex row access is a coalesced 32-element segment.
//
// Forward (leaves -> root), "pull" form: row t of supernode p first subtracts
// the contributions of every already-solved descendant d whose structure
// contains it (the per-row segment list, in ascending d: deterministic), then
// X_p = inv(L_pp) * B_p. No two CTAs write the same row, so no atomics.
// Backward (root -> leaves): B_s -= L_rs^T X_r (gather over the structure
// rows, which belong to ancestors and are final), then X_s = inv(L_pp)^T B_s.
//
// Heat right-hand sides are columns of the identity: the forward sweep builds
// them in registers from the source list, and only supernodes on a source's
// path to the root (`reach`) are solved; the rest of the forward result is
// known to be zero and is never read.
#include "kernels.cuh"

namespace fcw {

namespace {

constexpr int kWarps = 8;

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_level(DevPlan p, int32_t l0, const T* __restrict__ val,
                                                   const T* __restrict__ inv, T* __restrict__ B, int32_t K,
                                                   const int32_t* __restrict__ delta_src,
                                                   const uint8_t* __restrict__ reach) {
    __shared__ T Bs[kMaxWidth][kSlice + 1];
    const int node = p.level_nodes[l0 + blockIdx.x];
    if (reach && !reach[node]) return;
    const int k0 = blockIdx.y * kSlice;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = p.sn_c0[node];
    const int ns = p.sn_c0[node + 1] - c0;
    const int col = k0 + lane;
    for (int t = warp; t < ns; t += kWarps) {
        const int row = c0 + t;
        T b;
        if (delta_src) b = (delta_src[col] == row) ? T(1) : T(0);
        else b = B[(int64_t)row * K + col];
        T acc = T(0);
        for (int64_t q = p.seg_ptr[row]; q < p.seg_ptr[row + 1]; ++q) {
            const int d = p.seg_sn[q];
            if (reach && !reach[d]) continue;
            const int cd = p.sn_c0[d];
            const int nsd = p.sn_c0[d + 1] - cd;
            const T* Lr = val + p.sn_valptr[d] + (int64_t)p.seg_pos[q] * nsd;
            const T* X = B + (int64_t)cd * K + col;
            int j = 0;
            for (; j + 4 <= nsd; j += 4) {
                const T x0 = X[(int64_t)(j + 0) * K], x1 = X[(int64_t)(j + 1) * K];
                const T x2 = X[(int64_t)(j + 2) * K], x3 = X[(int64_t)(j + 3) * K];
                acc += Lr[j] * x0 + Lr[j + 1] * x1 + Lr[j + 2] * x2 + Lr[j + 3] * x3;
            }
            for (; j < nsd; ++j) acc += Lr[j] * X[(int64_t)j * K];
        }
        Bs[t][lane] = b - acc;
    }
    __syncthreads();
    const T* Inv = inv + p.sn_invptr[node];
    for (int t = warp; t < ns; t += kWarps) {
        const T* Lr = Inv + (int64_t)t * ns;
        T acc = T(0);
        for (int j = 0; j <= t; ++j) acc += Lr[j] * Bs[j][lane];
        B[(int64_t)(c0 + t) * K + col] = acc;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_bwd_level(DevPlan p, int32_t l0, const T* __restrict__ val,
                                                   const T* __restrict__ inv, T* __restrict__ B, int32_t K,
                                                   const uint8_t* __restrict__ reach) {
    __shared__ T Bs[kMaxWidth][kSlice + 1];
    const int node = p.level_nodes[l0 + blockIdx.x];
    const int k0 = blockIdx.y * kSlice;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = p.sn_c0[node];
    const int ns = p.sn_c0[node + 1] - c0;
    const int m = p.sn_m[node];
    const int col = k0 + lane;
    const bool zero_y = reach && !reach[node];
    for (int t = warp; t < ns; t += kWarps) Bs[t][lane] = zero_y ? T(0) : B[(int64_t)(c0 + t) * K + col];
    __syncthreads();
    const T* P = val + p.sn_valptr[node];
    const int32_t* rows = p.rows + p.sn_rowptr[node];
    T acc[kMaxWidth / kWarps];
#pragma unroll
    for (int q = 0; q < kMaxWidth / kWarps; ++q) acc[q] = T(0);
    for (int pos = ns; pos < m; ++pos) {
        const T x = B[(int64_t)rows[pos] * K + col];
        const T* Pr = P + (int64_t)pos * ns;
#pragma unroll
        for (int q = 0; q < kMaxWidth / kWarps; ++q) {
            const int j = warp + kWarps * q;
            if (j < ns) acc[q] += Pr[j] * x;
        }
    }
#pragma unroll
    for (int q = 0; q < kMaxWidth / kWarps; ++q) {
        const int j = warp + kWarps * q;
        if (j < ns) Bs[j][lane] -= acc[q];
    }
    __syncthreads();
    const T* Inv = inv + p.sn_invptr[node];
    for (int t = warp; t < ns; t += kWarps) {
        T a = T(0);
        for (int j = t; j < ns; ++j) a += Inv[(int64_t)j * ns + t] * Bs[j][lane];
        B[(int64_t)(c0 + t) * K + col] = a;
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

}  // namespace

template <typename T>
void launch_fwd_level(const DevPlan& p, int32_t l0, int32_t count, const T* val, const T* inv, T* B, int32_t K,
                      const int32_t* delta_src, const uint8_t* reach, cudaStream_t st) {
    if (count <= 0 || K <= 0) return;
    k_fwd_level<T><<<dim3(count, K / kSlice), 256, 0, st>>>(p, l0, val, inv, B, K, delta_src, reach);
}

template <typename T>
void launch_bwd_level(const DevPlan& p, int32_t l0, int32_t count, const T* val, const T* inv, T* B, int32_t K,
                      const uint8_t* reach, cudaStream_t st) {
    if (count <= 0 || K <= 0) return;
    k_bwd_level<T><<<dim3(count, K / kSlice), 256, 0, st>>>(p, l0, val, inv, B, K, reach);
}

void launch_reach(const DevPlan& p, const int32_t* src, int32_t K, uint8_t* reach, cudaStream_t st) {
    cudaMemsetAsync(reach, 0, (size_t)p.nsuper, st);
    k_reach<<<(K + 127) / 128, 128, 0, st>>>(p.col_sn, p.sn_parent, src, K, p.nlevels, reach);
}

template void launch_fwd_level<double>(const DevPlan&, int32_t, int32_t, const double*, const double*, double*,
                                       int32_t, const int32_t*, const uint8_t*, cudaStream_t);
template void launch_fwd_level<float>(const DevPlan&, int32_t, int32_t, const float*, const float*, float*,
                                      int32_t, const int32_t*, const uint8_t*, cudaStream_t);
template void launch_bwd_level<double>(const DevPlan&, int32_t, int32_t, const double*, const double*, double*,
                                       int32_t, const uint8_t*, cudaStream_t);
template void launch_bwd_level<float>(const DevPlan&, int32_t, int32_t, const float*, const float*, float*,
                                      int32_t, const uint8_t*, cudaStream_t);

}  // namespace fcw
