// One tensor-core product tile, exposed for checking the FP32 sweeps' arithmetic:
// C = A B (or P^T B) with A, B split into two TF32 terms each and the three
// significant cross products accumulated by tcgen05.mma in tensor memory. The
// operands go through the same shared-memory layouts and descriptors as the
// sweeps (tc.cuh), so a test of this entry point pins both the layouts and the
// accuracy of the split product against an FP64 product.
#include "fcw_b200.h"
#include "kernels.cuh"
#include "tc.cuh"

namespace fcw {
namespace {

constexpr int kCheckThreads = 256;

// One CTA. A: M x Kd row-major (trans = 0), or P: Kd x M row-major read as P^T
// (trans = 1). B: Kd x N row-major. C: M x N row-major. terms: 1 (hi x hi) or
// 3 (hi x hi + hi x lo + lo x hi); 0 and 2 are checks of the accumulator paths (see
// below). M <= 128, Kd <= 64, N in {64, 128}.
__global__ void __launch_bounds__(kCheckThreads) k_tc_product(const float* __restrict__ A,
                                                             const float* __restrict__ B, float* __restrict__ C,
                                                             int M, int Kd, int N, int terms, int trans,
                                                             float* __restrict__ raw, int* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint64_t done;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int MM = M <= 64 ? 64 : 128;          // instruction M
    const int Kp = (Kd + 7) / 8 * 8;            // depth padded to the instruction's K = 8
    const int kcores = Kp / 4;                  // 16-byte k-chunks per 8-row (8-column) group
    // both operands K-major, as in the sweeps: A (MM rows; trans: the transpose of P, made
    // when it is written) and B^T (N columns), split into TF32 hi and lo, zero outside
    const uint32_t a_bytes = (uint32_t)MM * Kp * 4u;
    const uint32_t b_bytes = (uint32_t)N * Kp * 4u;
    float* Ahi = reinterpret_cast<float*>(sm);
    float* Alo = reinterpret_cast<float*>(sm + a_bytes);
    float* Bhi = reinterpret_cast<float*>(sm + 2 * a_bytes);
    float* Blo = reinterpret_cast<float*>(sm + 2 * a_bytes + b_bytes);
    for (int e = tid; e < MM * Kp; e += kCheckThreads) {
        const int m = e / Kp, k = e - m * Kp;
        float x = 0.0f;
        if (m < M && k < Kd) x = trans ? A[k * M + m] : A[m * Kd + k];
        float hi, lo;
        tc::split_tf32(x, hi, lo);
        const uint32_t off = tc::core_offset(m, k, kcores) >> 2;
        Ahi[off] = hi;
        Alo[off] = lo;
    }
    for (int e = tid; e < Kp * N; e += kCheckThreads) {
        const int k = e / N, n = e - k * N;
        const float x = k < Kd ? B[k * N + n] : 0.0f;
        float hi, lo;
        tc::split_tf32(x, hi, lo);
        const uint32_t off = tc::core_offset(n, k, kcores) >> 2;
        Bhi[off] = hi;
        Blo[off] = lo;
    }
    tc::fence_async_smem();
    if (warp == 0) tc::tmem_alloc(&tbase, (uint32_t)N);
    if (tid == 0) {
        tc::mbar_init(&done, 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;
    // terms 0 / 2: lane l, column c of the accumulator first set to l * 1024 + c by tcgen05.st
    // (0: nothing else, a check of the accumulator's store and load paths; 2: the one-term
    // product is then added to it)
    if ((terms == 0 || terms == 2) && warp < 4) {
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            for (int j = 0; j < 16; ++j) v[j] = (float)((32 * warp + lane) * 1024 + c0 + j);
            tc::tmem_st16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0 && terms != 0) {
        const uint32_t idesc = tc::idesc_tf32(MM, N, false, false, false);
        const uint32_t sbo = (uint32_t)kcores * 128u;  // 8-row groups; k-chunks 128 bytes apart
        const uint32_t ah = tc::smem_u32(Ahi), al = tc::smem_u32(Alo), bh = tc::smem_u32(Bhi),
                       bl = tc::smem_u32(Blo);
        for (int s = 0; s < Kp / 8; ++s) {
            const uint32_t step = (uint32_t)s * 256u;
            const uint64_t dah = tc::sdesc(ah + step, 128u, sbo);
            const uint64_t dal = tc::sdesc(al + step, 128u, sbo);
            const uint64_t dbh = tc::sdesc(bh + step, 128u, sbo);
            const uint64_t dbl = tc::sdesc(bl + step, 128u, sbo);
            tc::mma_tf32(tmem, dah, dbh, idesc, (s > 0 || terms == 2) ? 1u : 0u);
            if (terms == 3) {
                tc::mma_tf32(tmem, dah, dbl, idesc, 1u);
                tc::mma_tf32(tmem, dal, dbh, idesc, 1u);
            }
        }
        tc::mma_commit(&done);
    }
    const bool ok = terms == 0 || tc::mbar_wait(&done, 0);
    if (!ok && lane == 0) atomicOr(status, KERR_TIMEOUT);
    tc::fence_after_sync();
    if (warp < 4 && ok) {
        const int lane0 = 32 * warp;
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + ((uint32_t)lane0 << 16) + (uint32_t)c0, v);
            const int L = lane0 + lane;  // this thread's TMEM lane
            if (raw)
                for (int j = 0; j < 16; ++j) raw[L * N + c0 + j] = v[j];
            // D row held by lane L: M = 128 -> L; M = 64 -> lanes 0-15 of each 32-lane quarter
            int row = -1;
            if (MM == 128) row = L;
            else if ((L & 31) < 16) row = (L & 15) + 16 * (L >> 5);
            if (row >= 0 && row < M)
                for (int j = 0; j < 16; ++j) C[row * N + c0 + j] = v[j];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, (uint32_t)N);
}

}  // namespace
}  // namespace fcw

extern "C" int fcw_tc_product_check(const float* a_dev, const float* b_dev, float* c_dev, int32_t m, int32_t k,
                                    int32_t n, int32_t terms, int32_t trans, float* raw_dev, int32_t* status_dev,
                                    void* stream) {
    if (!a_dev || !b_dev || !c_dev || !status_dev) return FCW_E_INVALID;
    if (m < 1 || m > 128 || k < 1 || k > 64 || (n != 64 && n != 128) || terms < 0 || terms > 3 ||
        (trans != 0 && trans != 1))
        return FCW_E_INVALID;
    const int MM = m <= 64 ? 64 : 128, Kp = (k + 7) / 8 * 8;
    const size_t a_bytes = (size_t)MM * Kp * 4;
    const size_t b_bytes = (size_t)Kp * n * 4;
    const size_t smem = 2 * a_bytes + 2 * b_bytes;
    cudaFuncSetAttribute(fcw::k_tc_product, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fcw::k_tc_product<<<1, fcw::kCheckThreads, smem, static_cast<cudaStream_t>(stream)>>>(
        a_dev, b_dev, c_dev, m, k, n, terms, trans, raw_dev, status_dev);
    return cudaGetLastError() == cudaSuccess ? FCW_OK : FCW_E_CUDA;
}
