// Multifrontal supernodal Cholesky factorisation in FP64, one etree level per launch.
//
// Storage (offsets from the symbolic analysis):
//   panel  P_s : m x ns row-major  -- after factorisation [L11; L21]
//   inverse    : ns x ns row-major  -- L11^{-1} (lower), used by the solves
//   update U_s : nr x nr row-major  -- F22 - L21 L21^T, consumed by the parent
// A's lower entries are scattered into the panels first; each front then adds
// its children's update matrices (extend-add, children in a fixed order, so the
// result is deterministic), factors the dense ns x ns block in shared memory,
// inverts it, forms L21 = F21 L11^{-T}, and a second launch per level subtracts
// L21 L21^T from U_s in 32 x 32 tiles. Once every level is factored, a last
// launch replaces each L21 by Q = L21 L11^{-1}: with it the solves form update
// rows (forward) and corrections (backward) straight from the right-hand side,
// without waiting for X_s = L11^{-1} (...).
#include "kernels.cuh"

namespace fcw {

namespace {

constexpr int kLd = kMaxWidth + 1;  // padded leading dimension of shared tiles

__global__ void k_scatter_a(int64_t nnz, const int64_t* __restrict__ dst, const double* __restrict__ aval,
                            double* __restrict__ val) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        val[dst[e]] = aval[e];
}

__global__ void k_to_float(int64_t n, const double* __restrict__ s, float* __restrict__ d) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        d[e] = (float)s[e];
}

__global__ void __launch_bounds__(256) k_factor_front(DevPlan p, int32_t l0, double* __restrict__ val,
                                                      double* __restrict__ inv, double* __restrict__ upd,
                                                      int* __restrict__ err) {
    extern __shared__ double sm[];
    double* D = sm;               // ns x ns lower factor
    double* Li = sm + kMaxWidth * kLd;  // its inverse
    const int s = p.level_nodes[l0 + blockIdx.x];
    const int c0 = p.sn_c0[s];
    const int ns = p.sn_c0[s + 1] - c0;
    const int m = p.sn_m[s];
    const int nr = m - ns;
    double* P = val + p.sn_valptr[s];
    double* U = upd + p.sn_updptr[s];
    const int tid = threadIdx.x, bs = blockDim.x;
    if (ns > kMaxWidth) {
        if (tid == 0) atomicOr(err, KERR_ARGS);
        return;
    }

    // 1. extend-add the children's update matrices, one child at a time
    for (int q = p.child_ptr[s]; q < p.child_ptr[s + 1]; ++q) {
        const int c = p.child_list[q];
        const int nsc = p.sn_c0[c + 1] - p.sn_c0[c];
        const int nrc = p.sn_m[c] - nsc;
        const double* Uc = upd + p.sn_updptr[c];
        const int32_t* rel = p.relind + p.sn_rowptr[c] + nsc;
        const int64_t tot = (int64_t)nrc * nrc;
        for (int64_t e = tid; e < tot; e += bs) {
            const int ia = (int)(e / nrc), ib = (int)(e - (int64_t)ia * nrc);
            if (ib > ia) continue;
            const int ra = rel[ia], rb = rel[ib];
            const double v = Uc[e];
            if (rb < ns) P[(int64_t)ra * ns + rb] += v;
            else U[(int64_t)(ra - ns) * nr + (rb - ns)] += v;
        }
        __syncthreads();
    }

    // 2. dense Cholesky of the diagonal block
    for (int e = tid; e < ns * ns; e += bs) {
        const int i = e / ns, j = e - i * ns;
        D[i * kLd + j] = (j <= i) ? P[(int64_t)i * ns + j] : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < ns; ++k) {
        if (tid == 0) {
            double piv = D[k * kLd + k];
            if (!(piv > 0.0)) {
                atomicOr(err, KERR_NOT_SPD);
                piv = 1.0;
            }
            D[k * kLd + k] = sqrt(piv);
        }
        __syncthreads();
        const double dk = D[k * kLd + k];
        for (int i = k + 1 + tid; i < ns; i += bs) D[i * kLd + k] /= dk;
        __syncthreads();
        const int r = ns - k - 1;
        for (int e = tid; e < r * r; e += bs) {
            const int i = k + 1 + e / r, j = k + 1 + e % r;
            if (j <= i) D[i * kLd + j] -= D[i * kLd + k] * D[j * kLd + k];
        }
        __syncthreads();
    }

    // 3. inverse of the lower-triangular block, one column per thread
    for (int j = tid; j < ns; j += bs) {
        for (int i = 0; i < ns; ++i) Li[i * kLd + j] = 0.0;
        Li[j * kLd + j] = 1.0 / D[j * kLd + j];
        for (int i = j + 1; i < ns; ++i) {
            double acc = 0.0;
            for (int k = j; k < i; ++k) acc += D[i * kLd + k] * Li[k * kLd + j];
            Li[i * kLd + j] = -acc / D[i * kLd + i];
        }
    }
    __syncthreads();
    double* Inv = inv + p.sn_invptr[s];
    for (int e = tid; e < ns * ns; e += bs) {
        const int i = e / ns, j = e - i * ns;
        P[(int64_t)i * ns + j] = (j <= i) ? D[i * kLd + j] : 0.0;
        Inv[e] = (j <= i) ? Li[i * kLd + j] : 0.0;
    }

    // 4. L21 = F21 L11^{-T}: row p of L21 is sum_k F21[p][k] Li[j][k], one warp per row
    const int lane = tid & 31, warp = tid >> 5, nwarps = bs >> 5;
    for (int row = ns + warp; row < m; row += nwarps) {
        double* R = P + (int64_t)row * ns;
        const double f0 = lane < ns ? R[lane] : 0.0;
        const double f1 = lane + 32 < ns ? R[lane + 32] : 0.0;
        double o0 = 0.0, o1 = 0.0;
        for (int k = 0; k < ns; ++k) {
            const double fk = __shfl_sync(0xffffffffu, k < 32 ? f0 : f1, k & 31);
            if (k <= lane && lane < ns) o0 += fk * Li[lane * kLd + k];
            if (k <= lane + 32 && lane + 32 < ns) o1 += fk * Li[(lane + 32) * kLd + k];
        }
        __syncwarp();
        if (lane < ns) R[lane] = o0;
        if (lane + 32 < ns) R[lane + 32] = o1;
    }
}

__global__ void __launch_bounds__(256) k_factor_update(DevPlan p, int32_t l0, const double* __restrict__ val,
                                                       double* __restrict__ upd) {
    __shared__ double A[32][kLd];
    __shared__ double B[32][kLd];
    const int s = p.level_nodes[l0 + blockIdx.x];
    const int ns = p.sn_c0[s + 1] - p.sn_c0[s];
    const int m = p.sn_m[s];
    const int nr = m - ns;
    if (nr == 0 || ns > kMaxWidth) return;
    const double* P = val + p.sn_valptr[s];
    double* U = upd + p.sn_updptr[s];
    const int nt = (nr + 31) / 32;
    const int64_t ntl = (int64_t)nt * (nt + 1) / 2;
    const int tid = threadIdx.x;
    const int r = tid >> 3, cb = tid & 7;
    for (int64_t t = blockIdx.y; t < ntl; t += gridDim.y) {
        int ta = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((int64_t)(ta + 1) * (ta + 2) / 2 <= t) ++ta;
        while ((int64_t)ta * (ta + 1) / 2 > t) --ta;
        const int tb = (int)(t - (int64_t)ta * (ta + 1) / 2);
        __syncthreads();
        for (int e = tid; e < 32 * ns; e += blockDim.x) {
            const int rr = e / ns, k = e - rr * ns;
            const int ga = ta * 32 + rr, gb2 = tb * 32 + rr;
            A[rr][k] = ga < nr ? P[(int64_t)(ns + ga) * ns + k] : 0.0;
            B[rr][k] = gb2 < nr ? P[(int64_t)(ns + gb2) * ns + k] : 0.0;
        }
        __syncthreads();
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < ns; ++k) {
            const double a = A[r][k];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] += a * B[cb + 8 * q][k];
        }
        const int ga = ta * 32 + r;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int gb2 = tb * 32 + cb + 8 * q;
            if (ga < nr && gb2 < nr && gb2 <= ga) U[(int64_t)ga * nr + gb2] -= acc[q];
        }
    }
}

// Row p of the panel becomes sum_{k >= j} L21[p][k] Li[k][j] (Li = L11^{-1}, lower).
__global__ void __launch_bounds__(256) k_panel_inverse(DevPlan p, double* __restrict__ val,
                                                       const double* __restrict__ inv) {
    __shared__ double Li[kMaxWidth * kLd];
    const int s = blockIdx.x;
    const int ns = p.sn_c0[s + 1] - p.sn_c0[s];
    const int m = p.sn_m[s];
    if (m == ns || ns > kMaxWidth) return;
    const double* I = inv + p.sn_invptr[s];
    const int tid = threadIdx.x;
    for (int e = tid; e < ns * ns; e += blockDim.x) {
        const int i = e / ns, j = e - i * ns;
        Li[i * kLd + j] = I[e];
    }
    __syncthreads();
    double* P = val + p.sn_valptr[s];
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int row = ns + warp; row < m; row += nwarps) {
        double* Rw = P + (int64_t)row * ns;
        const double f0 = lane < ns ? Rw[lane] : 0.0;
        const double f1 = lane + 32 < ns ? Rw[lane + 32] : 0.0;
        double o0 = 0.0, o1 = 0.0;
        for (int k = 0; k < ns; ++k) {
            const double fk = __shfl_sync(0xffffffffu, k < 32 ? f0 : f1, k & 31);
            if (lane <= k && lane < ns) o0 += fk * Li[k * kLd + lane];
            if (lane + 32 <= k && lane + 32 < ns) o1 += fk * Li[k * kLd + lane + 32];
        }
        __syncwarp();
        if (lane < ns) Rw[lane] = o0;
        if (lane + 32 < ns) Rw[lane + 32] = o1;
    }
}

}  // namespace

cudaError_t configure_kernels() {
    const int smem = (int)(2 * kMaxWidth * kLd * sizeof(double));
    return cudaFuncSetAttribute(k_factor_front, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

void launch_scatter_a(int64_t nnz, const int64_t* dst, const double* aval, double* val, cudaStream_t st) {
    if (nnz <= 0) return;
    int blocks = (int)((nnz + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_scatter_a<<<blocks, 256, 0, st>>>(nnz, dst, aval, val);
}

void launch_to_float(int64_t n, const double* src, float* dst, cudaStream_t st) {
    if (n <= 0) return;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_to_float<<<blocks, 256, 0, st>>>(n, src, dst);
}

void launch_factor_front(const DevPlan& p, int32_t l0, int32_t count, double* val, double* inv, double* upd,
                         int* err, cudaStream_t st) {
    if (count <= 0) return;
    const size_t smem = 2 * kMaxWidth * kLd * sizeof(double);
    k_factor_front<<<count, 256, smem, st>>>(p, l0, val, inv, upd, err);
}

void launch_panel_inverse(const DevPlan& p, double* val, const double* inv, cudaStream_t st) {
    if (p.nsuper <= 0) return;
    k_panel_inverse<<<p.nsuper, 256, 0, st>>>(p, val, inv);
}

void launch_factor_update(const DevPlan& p, int32_t l0, int32_t count, int32_t max_tiles, const double* val,
                          double* upd, cudaStream_t st) {
    if (count <= 0) return;
    int y = max_tiles < 1 ? 1 : (max_tiles > 512 ? 512 : max_tiles);
    k_factor_update<<<dim3(count, y), 256, 0, st>>>(p, l0, val, upd);
}

}  // namespace fcw
