// Iterative refinement of the mixed form's FP32 Poisson solve (fcw_params.refine).
//
// The grounded system L_g phi = b is solved with the FP32 factor; its error is the FP32
// factor's, about cond(L_g) times the FP32 rounding. One refinement step computes the
// residual r = b - L_g phi in FP64 (phi and b are FP32 values, exact in FP64, and L_g is
// the FP64 operator the factor came from, so r is the true residual rounded once to
// FP32), solves L_g d = r with the same FP32 factor and adds d: the error shrinks by about
// the factor's relative error, to the FP32 storage of phi.
#include "kernels.cuh"

namespace fcw {

namespace {

// r = b - A x for n x K row-major FP32 blocks, accumulated in FP64. One warp per row,
// four columns per lane (16-byte loads), the row's entries in CSR order.
__global__ void __launch_bounds__(256) k_residual(int32_t n, int32_t K, const int64_t* __restrict__ rp,
                                                  const int32_t* __restrict__ ci, const double* __restrict__ av,
                                                  const float* __restrict__ b, const float* __restrict__ x,
                                                  float* __restrict__ r) {
    const int lane = threadIdx.x & 31;
    const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (row >= n) return;
    const int64_t k0 = rp[row], k1 = rp[row + 1];
    for (int c = 4 * lane; c < K; c += 128) {
        const float4 bb = *reinterpret_cast<const float4*>(b + row * K + c);
        double a0 = bb.x, a1 = bb.y, a2 = bb.z, a3 = bb.w;
        for (int64_t k = k0; k < k1; ++k) {
            const double v = av[k];
            const float4 xx = *reinterpret_cast<const float4*>(x + (int64_t)ci[k] * K + c);
            a0 = fma(-v, (double)xx.x, a0);
            a1 = fma(-v, (double)xx.y, a1);
            a2 = fma(-v, (double)xx.z, a2);
            a3 = fma(-v, (double)xx.w, a3);
        }
        *reinterpret_cast<float4*>(r + row * K + c) = make_float4((float)a0, (float)a1, (float)a2, (float)a3);
    }
}

__global__ void k_add(int64_t n4, float4* __restrict__ y, const float4* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = y[i], e = d[i];
        y[i] = make_float4(a.x + e.x, a.y + e.y, a.z + e.z, a.w + e.w);
    }
}

}  // namespace

void launch_residual(const CsrOperator& A, int32_t K, const float* b, const float* x, float* r, cudaStream_t st) {
    if (A.n <= 0 || K <= 0) return;
    const int64_t threads = (int64_t)A.n * 32;
    k_residual<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(A.n, K, A.rp, A.ci, A.av, b, x, r);
}

void launch_add(int64_t count, float* y, const float* d, int num_sms, cudaStream_t st) {
    if (count <= 0) return;
    k_add<<<num_sms * 8, 256, 0, st>>>(count / 4, reinterpret_cast<float4*>(y), reinterpret_cast<const float4*>(d));
}

}  // namespace fcw
