// Fused gradient -> normalise -> divergence over faces (fastcw_lean.py:416-442).
//
// Vertex-centric gather: warp = one vertex, lane = one right-hand side. Each
// vertex walks its incident faces in ascending face order and recomputes the
// face's unit gradient, so every output element is written exactly once, by
// one thread, with the per-vertex summation order of the reference's face loop
// (no atomics, deterministic).
//
// FP64 form: the reference's 3-vector arithmetic, operation for operation,
// with explicit round-to-nearest intrinsics so the compiler cannot contract
// into FMAs: given the same u, the divergence is bit-identical.
//
// Mixed form: X = -grad u / |grad u| is invariant to scaling u's differences,
// so the two FP64 differences are rescaled by a power of two to O(1) (exact)
// and the rest runs in FP32 in the intrinsic form:
//   |g|^2 = du1^2 c11 + 2 du1 du2 c12 + du2^2 c22,  g . gb_c = du1 c1c + du2 c2c
// with c_ab = gb_a . gb_b. This keeps the direction accurate where u is far
// below FP32's range (u spans ~1e-130..1 on these meshes).
#include "kernels.cuh"

namespace fcw {

namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// The term of incidence q (a face of vertex v, at corner c) in column col of u (leading
// dimension K); false when the face's gradient vanishes (the face is skipped).
__device__ __forceinline__ bool face_term(const FaceData& fd, const double* __restrict__ u, int64_t K, int64_t col,
                                          int q, double& t) {
    const int f = fd.inc_face[q];
    const int c = fd.inc_corner[q];
    const int i0 = fd.fv[3 * f], i1 = fd.fv[3 * f + 1], i2 = fd.fv[3 * f + 2];
    const double* g = fd.gb + 9 * (int64_t)f;
    const double u0 = u[(int64_t)i0 * K + col];
    const double du1 = sub(u[(int64_t)i1 * K + col], u0);
    const double du2 = sub(u[(int64_t)i2 * K + col], u0);
    const double gx = add(mul(du1, g[3]), mul(du2, g[6]));
    const double gy = add(mul(du1, g[4]), mul(du2, g[7]));
    const double gz = add(mul(du1, g[5]), mul(du2, g[8]));
    const double nn = __dsqrt_rn(add(add(mul(gx, gx), mul(gy, gy)), mul(gz, gz)));
    if (!(nn > 1e-300)) return false;
    const double s = __ddiv_rn(-fd.garea[f], nn);
    const double* b = g + 3 * c;
    t = mul(s, add(add(mul(gx, b[0]), mul(gy, b[1])), mul(gz, b[2])));
    return true;
}

// The divergence at vertex v of column col of u: its faces' terms in incidence order.
__device__ __forceinline__ double div_at(const FaceData& fd, const double* __restrict__ u, int64_t K, int64_t col,
                                         int v) {
    double acc = 0.0;
    for (int q = fd.inc_ptr[v]; q < fd.inc_ptr[v + 1]; ++q) {
        double t;
        if (face_term(fd, u, K, col, q, t)) acc = add(acc, t);
    }
    return acc;
}

__global__ void __launch_bounds__(256) k_div_fp64(FaceData fd, const double* __restrict__ u,
                                                  double* __restrict__ div, int32_t K) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int v = blockIdx.x * 8 + warp;
    if (v >= fd.nv) return;
    const int col = blockIdx.y * kSlice + lane;
    div[(int64_t)v * K + col] = div_at(fd, u, K, col, v);
}

// One column: a thread per vertex (its face loop's loads are independent, so they overlap).
__global__ void __launch_bounds__(256) k_div_fp64_one(FaceData fd, const double* __restrict__ u,
                                                      double* __restrict__ div) {
    asm volatile("griddepcontrol.launch_dependents;");
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < fd.nv) div[v] = div_at(fd, u, 1, 0, v);
}

// 2^-e for the binary exponent e of |x| (x normal, nonzero): exact scaling to [1, 2).
__device__ __forceinline__ double unit_scale(double m) {
    const long long bits = __double_as_longlong(m);
    const int e = (int)((bits >> 52) & 0x7ff) - 1023;
    return __longlong_as_double((long long)(1023 - e) << 52);
}

// Mixed form, 64*NP columns per warp: lane l owns the column pairs {2l, 2l+1} + 64p,
// p < NP, of the warp's slice (one 16-byte load per pair and vertex row, 512
// contiguous bytes across the warp). The vertex's incidence records are read
// once, lane j holding the j-th, and broadcast face by face.
template <int NP>
__global__ void __launch_bounds__(256) k_div_mixed(FaceData fd, const double* __restrict__ u,
                                                   float* __restrict__ div, int32_t K,
                                                   const uint8_t* __restrict__ grounded) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int v = blockIdx.x * 8 + warp;
    if (v >= fd.nv) return;
    const int64_t c0 = (int64_t)blockIdx.y * 64 * NP + 2 * lane;
    float acc[2 * NP];
#pragma unroll
    for (int t = 0; t < 2 * NP; ++t) acc[t] = 0.0f;
    if (!grounded[v]) {
        const int q0 = fd.inc_ptr[v], deg = fd.inc_ptr[v + 1] - q0;
        for (int jb = 0; jb < deg; jb += 32) {
            const int nj = min(32, deg - jb);
            int4 rv = make_int4(0, 0, 0, 0);
            float4 rc = make_float4(0.f, 0.f, 0.f, 0.f);
            float2 rw = make_float2(0.f, 0.f);
            if (lane < nj) {
                rv = fd.inc_corners[q0 + jb + lane];
                rc = fd.inc_coef[q0 + jb + lane];
                rw = fd.inc_w[q0 + jb + lane];
            }
            for (int j = 0; j < nj; ++j) {
                const int i0 = __shfl_sync(0xffffffffu, rv.x, j);
                const int i1 = __shfl_sync(0xffffffffu, rv.y, j);
                const int i2 = __shfl_sync(0xffffffffu, rv.z, j);
                const double* p0 = u + (int64_t)i0 * K + c0;
                const double* p1 = u + (int64_t)i1 * K + c0;
                const double* p2 = u + (int64_t)i2 * K + c0;
                double u0[2 * NP], u1[2 * NP], u2[2 * NP];
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const double2 x0 = *reinterpret_cast<const double2*>(p0 + 64 * q);
                    const double2 x1 = *reinterpret_cast<const double2*>(p1 + 64 * q);
                    const double2 x2 = *reinterpret_cast<const double2*>(p2 + 64 * q);
                    u0[2 * q] = x0.x; u0[2 * q + 1] = x0.y;
                    u1[2 * q] = x1.x; u1[2 * q + 1] = x1.y;
                    u2[2 * q] = x2.x; u2[2 * q + 1] = x2.y;
                }
                const float c11 = __shfl_sync(0xffffffffu, rc.x, j);
                const float c12 = __shfl_sync(0xffffffffu, rc.y, j);
                const float c22 = __shfl_sync(0xffffffffu, rc.z, j);
                const float area = __shfl_sync(0xffffffffu, rc.w, j);
                const float w1 = __shfl_sync(0xffffffffu, rw.x, j);
                const float w2 = __shfl_sync(0xffffffffu, rw.y, j);
#pragma unroll
                for (int t = 0; t < 2 * NP; ++t) {
                    const double d1 = u1[t] - u0[t];
                    const double d2 = u2[t] - u0[t];
                    const double mx = fmax(fabs(d1), fabs(d2));
                    if (!(mx >= 2.2250738585072014e-308)) continue;  // zero (or subnormal) gradient
                    const double sc = unit_scale(mx);
                    const float x1 = (float)(d1 * sc), x2 = (float)(d2 * sc);
                    const float qn = x1 * x1 * c11 + 2.0f * x1 * x2 * c12 + x2 * x2 * c22;
                    if (!(qn > 0.0f)) continue;
                    acc[t] -= area * (x1 * w1 + x2 * w2) * rsqrtf(qn);
                }
            }
        }
    }
    float* o = div + (int64_t)v * K + c0;
#pragma unroll
    for (int q = 0; q < NP; ++q) *reinterpret_cast<float2*>(o + 64 * q) = make_float2(acc[2 * q], acc[2 * q + 1]);
}

}  // namespace

void launch_divergence_fp64(const FaceData& fd, const double* u, double* div, int32_t K, cudaStream_t st) {
    if (fd.nv <= 0 || K <= 0) return;
    k_div_fp64<<<dim3((fd.nv + 7) / 8, K / kSlice), 256, 0, st>>>(fd, u, div, K);
}

void launch_divergence_fp64_one(const FaceData& fd, const double* u, double* div, cudaStream_t st) {
    if (fd.nv > 0) k_div_fp64_one<<<(fd.nv + 255) / 256, 256, 0, st>>>(fd, u, div);
}

void launch_divergence_mixed(const FaceData& fd, const double* u, float* div, int32_t K, const uint8_t* grounded,
                             cudaStream_t st) {
    if (fd.nv <= 0 || K <= 0) return;
    if (K % 128 == 0)
        k_div_mixed<2><<<dim3((fd.nv + 7) / 8, K / 128), 256, 0, st>>>(fd, u, div, K, grounded);
    else  // K is a multiple of 64
        k_div_mixed<1><<<dim3((fd.nv + 7) / 8, K / 64), 256, 0, st>>>(fd, u, div, K, grounded);
}

}  // namespace fcw
