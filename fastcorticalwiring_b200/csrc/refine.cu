// Iterative refinement of the mixed form's FP32 Poisson solve (fcw_params.refine).
//
// The grounded system L_g phi = b is solved with the FP32 factor; its error is the FP32
// factor's, about cond(L_g) times the FP32 rounding. One refinement step computes the
// residual r = b - L_g phi in FP64 (phi and b are FP32 values, exact in FP64, and L_g is
// the FP64 operator the factor came from, so r is the true residual rounded once to
// FP32), solves L_g d = r with the same FP32 factor and adds d: the error shrinks by about
// the factor's relative error, to the FP32 storage of phi.
//
// On a submesh of several connected components, L is singular once per component and the
// grounded operator fixes one vertex of each at zero. The FP64 form's L + shift*M instead
// leaves phi with zero M-weighted mean on the source's component (1^T div X = 0 there) and
// zero on the others (no heat reaches them), so after the shift phi - phi(s) the vertices of
// other components sit at the mean distance over the source's component. The component level
// gives the grounded solution the same values off the source's component; on it the shift
// removes the difference.
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

constexpr int kCompVTile = 256;  // vertex rows per CTA: 8 warps x 32 rows

// part[tile][k] = sum over the tile's vertices v in the component of src[k] of mass[v] phi[v][k].
// 64 sources per CTA: lane l holds columns 2l, 2l+1 (each warp reads 256 contiguous bytes of a
// row), each warp 32 rows with four rows' loads in flight; the sums are taken in a fixed order.
__global__ void __launch_bounds__(256) k_comp_partial(int32_t n, int32_t K, const int32_t* __restrict__ src,
                                                      const int32_t* __restrict__ comp,
                                                      const double* __restrict__ mass, const float* __restrict__ phi,
                                                      double* __restrict__ part) {
    __shared__ double red[8][64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k = blockIdx.y * 64 + 2 * lane;
    const int s0 = src[k], s1 = src[k + 1];
    const int c0 = s0 >= 0 ? comp[s0] : -1, c1 = s1 >= 0 ? comp[s1] : -1;
    const int v0 = blockIdx.x * kCompVTile + warp * 32;
    const int v1 = min(n, v0 + 32);
    double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
    for (int v = v0; v < v1; ++v) {
        const int cv = comp[v];
        const double mv = mass[v];
        const float2 p = *reinterpret_cast<const float2*>(phi + (int64_t)v * K + k);
        if (cv == c0) a0 = fma(mv, (double)p.x, a0);
        if (cv == c1) a1 = fma(mv, (double)p.y, a1);
    }
    red[warp][2 * lane] = a0;
    red[warp][2 * lane + 1] = a1;
    __syncthreads();
    if (threadIdx.x < 64) {
        double t = 0.0;
        for (int j = 0; j < 8; ++j) t += red[j][threadIdx.x];
        part[(int64_t)blockIdx.x * K + blockIdx.y * 64 + threadIdx.x] = t;
    }
}

// level[k] = sum over tiles of part[tile][k] / area of src[k]'s component, in a fixed order
// (the same levels on every run).
__global__ void __launch_bounds__(256) k_comp_mean(int32_t ntiles, int32_t K, const int32_t* __restrict__ src,
                                                   const int32_t* __restrict__ comp,
                                                   const double* __restrict__ area,
                                                   const double* __restrict__ part, double* __restrict__ level) {
    __shared__ double red[8][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int k = blockIdx.x * 32 + tx;
    double acc = 0.0;
    for (int t = ty; t < ntiles; t += 8) acc += part[(int64_t)t * K + k];
    red[ty][tx] = acc;
    __syncthreads();
    if (ty == 0) {
        double t = 0.0;
        for (int j = 0; j < 8; ++j) t += red[j][tx];
        const int s = src[k];
        level[k] = s >= 0 ? t / area[comp[s]] : 0.0;
    }
}

// phi[v][k] = level[k] for v off src[k]'s component (the layout of k_comp_partial)
__global__ void __launch_bounds__(256) k_comp_fill(int32_t n, int32_t K, const int32_t* __restrict__ src,
                                                   const int32_t* __restrict__ comp,
                                                   const double* __restrict__ level, float* __restrict__ phi) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k = blockIdx.y * 64 + 2 * lane;
    const int s0 = src[k], s1 = src[k + 1];
    const int c0 = s0 >= 0 ? comp[s0] : -1, c1 = s1 >= 0 ? comp[s1] : -1;
    const float l0 = (float)level[k], l1 = (float)level[k + 1];
    const int v0 = blockIdx.x * kCompVTile + warp * 32;
    const int v1 = min(n, v0 + 32);
    for (int v = v0; v < v1; ++v) {
        const int cv = comp[v];
        if (c0 >= 0 && cv != c0) phi[(int64_t)v * K + k] = l0;
        if (c1 >= 0 && cv != c1) phi[(int64_t)v * K + k + 1] = l1;
    }
}

}  // namespace

int64_t component_tiles(int64_t n) { return (n + kCompVTile - 1) / kCompVTile; }

void launch_component_level(const ComponentLevel& c, int32_t K, const int32_t* src, float* phi, double* scratch,
                            cudaStream_t st) {
    if (c.n <= 0 || K <= 0) return;
    const int64_t nt = component_tiles(c.n);
    double* level = scratch + nt * K;
    const dim3 grid((unsigned)nt, (unsigned)(K / 64));  // K is a multiple of 64
    k_comp_partial<<<grid, 256, 0, st>>>(c.n, K, src, c.comp, c.mass, phi, scratch);
    k_comp_mean<<<K / 32, dim3(32, 8), 0, st>>>((int32_t)nt, K, src, c.comp, c.area, scratch, level);
    k_comp_fill<<<grid, 256, 0, st>>>(c.n, K, src, c.comp, level, phi);
}

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
