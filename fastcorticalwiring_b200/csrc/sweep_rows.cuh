// Row-segment movement shared by the supernodal sweeps (solve.cu): 16-byte
// vectors, cp.async copies, tiles to n x K arrays, and the gather of children's
// update rows (see solve.cu for the algorithm).
#pragma once

#include "kernels.cuh"

namespace fcw {
namespace {

constexpr int NT = 256;  // threads per sweep CTA

template <typename T>
constexpr int vec() { return 16 / (int)sizeof(T); }  // elements per 16-byte vector

// One 16-byte vector (vec<T>() elements) between memory and registers.
template <typename T>
__device__ __forceinline__ void ldv(const T* p, T* w) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else {
        const double2 v = *reinterpret_cast<const double2*>(p);
        w[0] = v.x; w[1] = v.y;
    }
}

template <typename T>
__device__ __forceinline__ void stv(T* p, const T* w) {
    if constexpr (sizeof(T) == 4)
        *reinterpret_cast<float4*>(p) = make_float4(w[0], w[1], w[2], w[3]);
    else
        *reinterpret_cast<double2*>(p) = make_double2(w[0], w[1]);
}

// V adjacent elements (V * sizeof(T) is 8 or 16 bytes, aligned).
template <typename T, int V>
__device__ __forceinline__ void ld_n(const T* p, T* w) {
    if constexpr (V * sizeof(T) == 16) {
        ldv(p, w);
    } else {
        static_assert(V == 2 && sizeof(T) == 4, "8-byte groups are float pairs");
        const float2 v = *reinterpret_cast<const float2*>(p);
        w[0] = v.x; w[1] = v.y;
    }
}
template <typename T, int V>
__device__ __forceinline__ void st_n(T* p, const T* w) {
    if constexpr (V * sizeof(T) == 16) {
        stv(p, w);
    } else {
        static_assert(V == 2 && sizeof(T) == 4, "8-byte groups are float pairs");
        *reinterpret_cast<float2*>(p) = make_float2(w[0], w[1]);
    }
}

// Asynchronous global -> shared copies (cp.async): single elements through L1,
// 16-byte vectors around it.
template <typename T>
__device__ __forceinline__ void copy_async(T* smem, const T* gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy16_async(void* smem, const void* gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void copy_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Rows [0, nrows) of a KT-wide shared tile (row stride ld) to an n x K array
// (g = first row, first column).
template <typename T, int KT>
__device__ __forceinline__ void tile_rows_to_global(T* g, int64_t K, const T* D, int ld, int nrows) {
    constexpr int VPR = KT / vec<T>();
    for (int i = threadIdx.x; i < nrows * VPR; i += NT) {
        const int r = i / VPR, v = i - r * VPR;
        *reinterpret_cast<uint4*>(g + r * K + v * vec<T>()) =
            *reinterpret_cast<const uint4*>(D + r * ld + v * vec<T>());
    }
}

// ---------------------------------------------------------------------------
// Children's update rows of front rows [f0, f0+nrows): entries [eb, eb+E) of the
// gather lists; grs[r] .. grs[r+1] (relative to eb) are those of row r.
// ---------------------------------------------------------------------------
struct GatherRange {
    int eb, E;
};

template <typename T>
__device__ __forceinline__ GatherRange gather_open(const SolveArgs<T>& a, int64_t fb, int f0, int nrows, int* grs) {
    GatherRange g;
    g.eb = a.gm_ptr[fb + f0];
    g.E = a.gm_ptr[fb + f0 + nrows] - g.eb;
    for (int r = threadIdx.x; r <= nrows; r += NT) grs[r] = a.gm_ptr[fb + f0 + r] - g.eb;
    return g;
}

// Async copies of the staged chunk that starts at entry e0; live[e] = 0 for rows
// of children off the sources' paths (their update rows were never written).
template <typename T, int KT, int TR>
__device__ __forceinline__ void gather_issue(const SolveArgs<T>& a, const GatherRange& g, int e0, int k0, T* St,
                                             unsigned char* live) {
    constexpr int VPR = KT / vec<T>();
    const int ne = min(g.E - e0, a.stage);
    for (int i = threadIdx.x; i < ne * VPR; i += NT) {
        const int e = i / VPR, v = i - e * VPR;
        const int ge = g.eb + e0 + e;
        const bool on = !a.reach || a.reach[(int64_t)a.gm_child[ge] * a.reach_tiles + k0 / kReachCols];
        if (v == 0) live[e] = on;
        if (on) copy16_async(St + e * KT + v * vec<T>(), a.U + (int64_t)a.gm_src[ge] * a.K + k0 + v * vec<T>());
    }
}

// D rows (+ or -)= the staged entries [e0, e1) that belong to them, in entry order.
template <typename T, int KT, bool SUB>
__device__ __forceinline__ void gather_accumulate(T* D, int ld, const T* St, const unsigned char* live,
                                                  const int* grs, int nrows, int e0, int e1) {
    constexpr int G = vec<T>(), TPR = KT / G, RG = NT / TPR;  // threads per row (one vector each), rows in parallel
    const int c = G * (threadIdx.x % TPR);
    for (int r = threadIdx.x / TPR; r < nrows; r += RG) {
        const int lo = max(grs[r], e0), hi = min(grs[r + 1], e1);
        if (lo >= hi) continue;
        T v[G], u[G];
        ldv(D + r * ld + c, v);
        for (int e = lo; e < hi; ++e) {
            if (!live[e - e0]) continue;
            ldv(St + (e - e0) * KT + c, u);
#pragma unroll
            for (int q = 0; q < G; ++q) v[q] = SUB ? v[q] - u[q] : v[q] + u[q];
        }
        stv(D + r * ld + c, v);
    }
}

// Waits for every copy this CTA has in flight (the caller has issued the
// range's first chunk), then adds the range chunk by chunk.
template <typename T, int KT, int TR, bool SUB>
__device__ __forceinline__ void gather_finish(const SolveArgs<T>& a, const GatherRange& g, int k0, T* D, int ld,
                                              int nrows, T* St, unsigned char* live, const int* grs) {
    const int SG = a.stage;  // >= 1 whenever the level has gathers (g.E > 0)
    int e0 = 0;
    do {
        if (e0 > 0) {
            gather_issue<T, KT, TR>(a, g, e0, k0, St, live);
            copy_async_commit();
        }
        copy_async_wait();
        __syncthreads();
        if (g.E > 0) gather_accumulate<T, KT, SUB>(D, ld, St, live, grs, nrows, e0, min(g.E, e0 + SG));
        __syncthreads();
        e0 += SG;
    } while (e0 < g.E);
}

}  // namespace
}  // namespace fcw
