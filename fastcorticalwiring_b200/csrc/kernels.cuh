// Device kernels of the heat-method pipeline and their host launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace fcw {

// Error bits a kernel may raise (OR-ed into a device word read by the host).
enum : int {
    KERR_NOT_SPD = 1,         // non-positive pivot in the numeric factorisation
    KERR_HIST_OVERFLOW = 2,   // more distance bins than the geometry kernel holds
    KERR_SCRATCH = 4,         // per-source face list overflow
    KERR_ARGS = 8,            // inconsistent launch arguments
    KERR_TIMEOUT = 16,        // a bounded wait (mbarrier, tensor-core completion) expired
};

constexpr int kMaxWidth = 64;      // widest supernode the dense kernels accept
constexpr int kSlice = 32;         // right-hand sides per CTA column slice (one per lane)
constexpr int kMaxBins = 2048;     // distance bins per source held in shared memory
constexpr int kMaxTargets = 32;
constexpr int kMaxBetween = 8;

// Supernodal structure on the device (all pointers device memory).
struct DevPlan {
    int32_t n = 0, nsuper = 0, nlevels = 0;
    const int32_t* sn_c0 = nullptr;
    const int32_t* sn_m = nullptr;
    const int64_t* sn_rowptr = nullptr;
    const int32_t* rows = nullptr;
    const int64_t* sn_valptr = nullptr;
    const int64_t* sn_invptr = nullptr;
    const int64_t* sn_updptr = nullptr;
    const int32_t* sn_parent = nullptr;
    const int32_t* col_sn = nullptr;
    const int32_t* level_nodes = nullptr;
    const int32_t* child_ptr = nullptr;
    const int32_t* child_list = nullptr;
    const int32_t* relind = nullptr;
    const int64_t* seg_ptr = nullptr;
    const int32_t* seg_sn = nullptr;
    const int32_t* seg_pos = nullptr;
};

// ---- numeric factorisation (factor.cu) ----
// Per-device kernel attributes (large dynamic shared memory); call once per device.
cudaError_t configure_kernels();
void launch_scatter_a(int64_t nnz, const int64_t* dst, const double* aval, double* val, cudaStream_t st);
// one level: extend-add children, dense Cholesky of the diagonal block, its inverse, L21
void launch_factor_front(const DevPlan& p, int32_t l0, int32_t count, double* val, double* inv, double* upd,
                         int* err, cudaStream_t st);
// one level: update matrices U -= L21 L21^T
void launch_factor_update(const DevPlan& p, int32_t l0, int32_t count, int32_t max_tiles, const double* val,
                          double* upd, cudaStream_t st);
void launch_to_float(int64_t n, const double* src, float* dst, cudaStream_t st);
// after every level: each panel's L21 becomes Q = L21 L11^{-1} (what the solves read)
void launch_panel_inverse(const DevPlan& p, double* val, const double* inv, cudaStream_t st);

// ---- multi-RHS supernodal triangular solves (solve.cu) ----
constexpr int kRhsTile = 64;     // right-hand sides per solve CTA; K is a multiple of this
constexpr int kReachCols = 64;   // columns per tile of the heat solve's reach flags (its FP64 tile width)
constexpr int kSplitRows = 128;  // structure rows per backward split-K task

template <typename T>
struct SolveArgs {
    DevPlan p;
    const T* val = nullptr;          // panels: below the diagonal block, Q = L21 L11^{-1}
    const T* inv = nullptr;          // inverse diagonal blocks
    const T* R = nullptr;            // n x K right-hand sides (read only; unused with delta_src)
    T* B = nullptr;                  // n x K forward result, then solution (elimination order)
    int32_t K = 0;
    T* U = nullptr;                  // forward update rows, (sum nr) x K
    const int64_t* uoff = nullptr;   // first update row of each supernode
    const int32_t* gm_ptr = nullptr; // per front row (sn_rowptr-based index): update rows that land on it
    const int32_t* gm_src = nullptr;
    const int32_t* gm_child = nullptr;
    const int32_t* delta_src = nullptr;  // forward: identity columns for these sources (elimination order)
    const uint8_t* reach = nullptr;      // heat solve: reach[s * reach_tiles + t], supernode s on the path to the
                                         // root of some source of column tile t (kReachCols columns)
    int32_t reach_tiles = 0;
    const int2* tasks = nullptr;         // (supernode, row chunk | split)
    const int32_t* nsplit = nullptr;     // backward splits per supernode
    const int64_t* poff = nullptr;       // partial-sum slot of the first split (units of 64 x K)
    T* part = nullptr;
    int* counters = nullptr;             // per (supernode, column tile) arrival tickets, zero at rest
    int32_t ktiles = 0;                  // column tiles the counters were sized for
    int32_t stage = 0;                   // forward: children's update rows staged per chunk (set by the launcher)
    // FP32 tensor-core sweeps: per supernode the stacked [inv(L_ss); Q_s] split into TF32 hi and
    // lo terms, in core-matrix order (tc.cuh), ns8 = round_up(ns, 8) columns and ns8 +
    // round_up(nr, 32) rows (padding zero)
    const float* core_hi = nullptr;
    const float* core_lo = nullptr;
    const float* coreT_hi = nullptr;     // the transposes (backward products), 32-row chunks
    const float* coreT_lo = nullptr;
    const int64_t* core_ptr = nullptr;   // per supernode: offset (floats) of its core array
    int* err = nullptr;                  // error bits (bounded waits that expired)
};

cudaError_t configure_solve_kernels();
// Forward sweep of one level (tasks [t0, t0+ntasks) of the level's list);
// gathers: some supernode of the level has children (leaf levels have none and
// launch without a staging buffer, so more CTAs share an SM).
template <typename T>
void launch_fwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, bool gathers, cudaStream_t st);
// Backward sweep of one level; tile_rows is 32 when every supernode of the
// level is at most 32 wide, else 64.
template <typename T>
void launch_bwd_level(const SolveArgs<T>& a, int32_t t0, int32_t ntasks, int32_t tile_rows, cudaStream_t st);
void launch_reach(const DevPlan& p, const int32_t* src, int32_t K, uint8_t* reach, cudaStream_t st);

// FP32 sweeps on the tensor cores (tcgen05.mma kind::tf32, each operand split into two TF32
// terms, three products accumulated in tensor memory); K a multiple of 64, 64 columns per CTA.
// Forward tasks are (supernode, c): c = 0 forms X_s = inv(L_ss) W and update rows [0, 64),
// c >= 1 update rows [64 + 128 (c - 1), 64 + 128 c). Backward tasks are those of launch_bwd_level. rows_map is a tiled tensor
// map of the sweep's own-row input (forward: R, backward: B) made by make_rows_map.
constexpr int kTcCols = 64;
void launch_fwd_level_tc(const SolveArgs<float>& a, int32_t t0, int32_t ntasks, const CUtensorMap& rows_map,
                         cudaStream_t st);
void launch_bwd_level_tc(const SolveArgs<float>& a, int32_t t0, int32_t ntasks, const CUtensorMap& rows_map,
                         cudaStream_t st);
cudaError_t configure_tc_kernels();
// Tensor map of an n x K row-major FP32 array: boxes of 64 rows x 32 columns, 128-byte swizzle.
int make_rows_map(CUtensorMap* map, const float* base, int64_t n, int32_t K);
// The core arrays of the tensor-core sweeps from the FP64 panels and inverse blocks.
void launch_build_cores(const DevPlan& p, const double* val, const double* inv, const int64_t* core_ptr,
                        float* hi, float* lo, float* hiT, float* loT, cudaStream_t st);

// ---- one right-hand side: the single-source drop-in (solve_narrow.cu) ----
constexpr int kNarrowRows = 64;            // stacked rows per chunk of the narrow layout
constexpr int kNarrowTaskDoubles = 12288;  // panel data of one task (96 KB); fronts up to this many rows
struct NarrowArgs {
    DevPlan p;
    const double* at = nullptr;       // per supernode [inv(L_ss); Q_s]: forward, 64-row column-major chunks;
                                      // backward, column-major over all rows
    const int64_t* at_ptr = nullptr;  // per supernode: offset (doubles, even) in either layout
    const int4* tasks = nullptr;      // forward: (s, first chunk, chunks); backward: (s, j0, j1)
    int32_t ntasks = 0;
    // heat forward: the source's elimination index, the path's task count, then (task,
    // previous supernode on the path) pairs bottom-up
    const int32_t* order = nullptr;
    const double* R = nullptr;        // forward right-hand side (n)
    double* B = nullptr;              // forward result (n)
    double* X = nullptr;              // backward: the solution (n), pending on entry
    double* U = nullptr;              // forward update entries (sum nr), pending on entry
    const int64_t* uoff = nullptr;
    const int32_t* gm_ptr = nullptr;
    const int32_t* gm_src = nullptr;
    const int32_t* gm_child = nullptr;
    int* ticket = nullptr;            // zero when a sweep starts
    const int32_t* iperm = nullptr;
    int* err = nullptr;
};
struct NarrowLaunch {
    int grid_fwd = 0, grid_bwd = 0;
    size_t fwd_smem = 0, bwd_smem = 0;
};
// Chunk offsets of the narrow layout (nsuper + 1 entries); returns the doubles it holds.
int64_t narrow_layout(const int32_t* sn_c0, const int32_t* sn_m, int32_t nsuper, int64_t* at_ptr);
// Forward tasks in level order (supernode s's are the nfwd[s] from fwd_first[s]), backward
// tasks in reversed level order, and each supernode's task counts.
void narrow_tasks(const int32_t* sn_c0, const int32_t* sn_m, int32_t nsuper, const int32_t* level_nodes,
                  std::vector<int4>& fwd, std::vector<int32_t>& fwd_first, std::vector<int32_t>& nfwd,
                  std::vector<int4>& bwd, std::vector<int32_t>& nbwd);
void launch_build_narrow(const DevPlan& p, const double* val, const double* inv, const int64_t* at_ptr,
                         double* at_f, double* at_b, cudaStream_t st);
cudaError_t configure_narrow_kernels(int max_m, int num_sms, NarrowLaunch* L);
// Forward sweep (delta: the identity column of a.order's source over its path's tasks; B
// zero on entry), backward sweep.
// overlap: start while the stream's previous kernel finishes (programmatic dependent launch);
// that kernel's results are read only once it has completed.
void launch_fwd_narrow(const NarrowArgs& a, bool delta, bool overlap, const NarrowLaunch& L, cudaStream_t st);
void launch_bwd_narrow(const NarrowArgs& a, bool overlap, const NarrowLaunch& L, cudaStream_t st);
// out[i] = Y[iperm[i]] - Y[*src_elim] (caller's order, shifted to zero at the source)
void launch_field_out_one(int32_t n, const double* Y, const int32_t* src_elim, const int32_t* iperm, double* out,
                          int num_sms, cudaStream_t st);

// ---- iterative refinement of the mixed Poisson solve (refine.cu) ----
struct CsrOperator {
    int32_t n = 0;
    const int64_t* rp = nullptr;  // n + 1
    const int32_t* ci = nullptr;
    const double* av = nullptr;
};
// r = b - A x (n x K row-major FP32 blocks, K a multiple of 4), accumulated in FP64
void launch_residual(const CsrOperator& A, int32_t K, const float* b, const float* x, float* r, cudaStream_t st);
// y += d over count floats (a multiple of 4)
void launch_add(int64_t count, float* y, const float* d, int num_sms, cudaStream_t st);

// ---- the mixed form's level on a submesh of several connected components (refine.cu) ----
struct ComponentLevel {
    int32_t n = 0;
    int32_t* comp = nullptr;  // n: each vertex's component (elimination order)
    double* mass = nullptr;   // n: each vertex's lumped mass (elimination order)
    double* area = nullptr;   // each component's total lumped mass
};
// vertex tiles of the level's per-tile sums
int64_t component_tiles(int64_t n);
// Sets each column of phi (n x K FP32, row-major, zero off its source's component) off the
// component of its source src[k] (elimination order) to the M-weighted mean of phi over that
// component. scratch: (component_tiles(n) + 1) * K doubles. Three kernels.
void launch_component_level(const ComponentLevel& c, int32_t K, const int32_t* src, float* phi, double* scratch,
                            cudaStream_t st);

// ---- fused gradient -> normalise -> divergence (face.cu) ----
struct FaceData {
    int32_t nv = 0, nf = 0;
    const int32_t* fv = nullptr;        // nf*3, elimination-order vertex ids
    const double* gb = nullptr;         // nf*9 hat-function gradients (fastcw_lean.py:375-391)
    const double* garea = nullptr;      // nf
    const float* coef = nullptr;        // nf*4: c11, c12, c22, area (FP32 intrinsic form)
    const int32_t* inc_ptr = nullptr;   // nv+1, per elimination-order vertex
    const int32_t* inc_face = nullptr;  // incident faces in ascending face order
    const int8_t* inc_corner = nullptr; // which corner of the face the vertex is
    // the same incidences as records for the mixed form: the face's corners, its
    // FP32 intrinsic coefficients (c11, c12, c22, area) and the vertex's corner
    // weights (w1, w2), so a vertex reads its faces without an index chain
    const int4* inc_corners = nullptr;
    const float4* inc_coef = nullptr;
    const float2* inc_w = nullptr;
};
void launch_divergence_fp64(const FaceData& fd, const double* u, double* div, int32_t K, cudaStream_t st);
// One column (K = 1), the same arithmetic per vertex.
void launch_divergence_fp64_one(const FaceData& fd, const double* u, double* div, cudaStream_t st);
// grounded (elimination order): the ground vertices, whose divergence is zero
void launch_divergence_mixed(const FaceData& fd, const double* u, float* div, int32_t K, const uint8_t* grounded,
                             cudaStream_t st);

// ---- per-source kernels (metrics.cu) ----
template <typename Tin, typename Tout>
void launch_shift_transpose(int32_t n, int32_t K, const Tin* phi, const int32_t* src, Tout* dT, cudaStream_t st);
// out[out_idx[i]][c] = in[in_idx[i]][c] for i < n, c < cols (null index = identity)
void launch_permute_rows(int32_t n, int32_t cols, const double* in, int32_t in_ld, const int32_t* in_idx,
                         double* out, int32_t out_ld, const int32_t* out_idx, cudaStream_t st);

// A block's inputs in the pipelined metrics path, read on the device, so that the
// launch chain captured once per workspace serves every block.
struct BlockDesc {
    const int32_t* sources = nullptr;  // the block's sources (caller's order)
    int64_t n = 0;                     // sources in the block (<= K)
    double* out = nullptr;             // the block's records (n * stride)
};

struct MetricArgs {
    int32_t n = 0, nf = 0, nsrc = 0, stride = 0, n_targets = 0, n_between = 0, n_boundary = 0;
    const double* coords = nullptr;     // n*3, elimination order
    const double* vertex_area = nullptr;
    const int32_t* boundary = nullptr;  // elimination-order ids
    const int32_t* fv = nullptr;
    const int32_t* inc_ptr = nullptr;   // vertex -> incident faces (elimination order)
    const int32_t* inc_face = nullptr;
    const int8_t* inc_corner = nullptr;
    const int4* inc_rec = nullptr;      // per incidence (inc_face order): face, its three corners
    const long long* farea_fx = nullptr;  // lean face areas in fixed point (exact order-free sums)
    double area_unscale = 0.0;          // fixed point -> area
    double total_area = 0.0;            // sum of the lean face areas
    const double* farea = nullptr;      // lean face area, g11, g12, g22 (lean_geometry.py:44-63)
    const double* g11 = nullptr;
    const double* g12 = nullptr;
    const double* g22 = nullptr;
    double width = 0.0, health_h = 0.0, eps = 1e-6, rtol = 1e-10;
    int32_t max_iter = 60;
    double targets[kMaxTargets];
    double fracs[kMaxBetween];
    const int32_t* src = nullptr;       // elimination-order source per column
    int4* band = nullptr;               // nsrc * nf scratch: near faces (face, corners) sorted by sub-bin
    int32_t* longf = nullptr;           // nsrc * nf scratch: near long faces
    double* out = nullptr;              // nsrc * stride
    const BlockDesc* desc = nullptr;    // when set, the records go to desc->out instead
    int* err = nullptr;
    // shift + statistics (k_shift_stats) -> per-source kernel
    int32_t K = 0;                      // columns of the block (partials' leading dimension)
    int32_t ntiles = 0;                 // vertex tiles of kStatVTile vertices
    double* partials = nullptr;         // ntiles x K x 8 partial statistics
    double near_radius = 0.0;           // = near_bins * width
    int32_t near_bins = 0;
    int32_t first_bins = 0;             // cut of a source's first attempt (<= near_bins)
    int32_t* near_list = nullptr;       // K x n: vertices closer than near_radius, per source
    int32_t* near_count = nullptr;      // K
};
constexpr int kStatVTile = 1024;   // vertices per shift-statistics CTA

// ---- per-source sample assembly (samples.cu) ----
constexpr int kMaxSamples = kMaxTargets + (kMaxTargets - 1) * kMaxBetween;
struct SampleArgs {
    int64_t n = 0;                    // sources (records)
    int32_t n_targets = 0, n_between = 0, stride = 0, capacity = 0;
    double targets[kMaxTargets];
    double cap = 0.0;                 // boundary cap on the clipped disc fraction; NaN: none
    const double* records = nullptr;  // n x stride (fcw_compute_metrics layout)
    float* radii_out = nullptr;       // n x capacity
    float* areas_out = nullptr;       // n x capacity
    int32_t* count_out = nullptr;     // n
};
void launch_assemble_samples(const SampleArgs& a, cudaStream_t st);
// phi (n x K) -> dT (K x n) with phi[source] subtracted, plus per-tile health/MSD
// partials and the per-source near-vertex lists.
template <typename Tin, typename Tout>
void launch_shift_stats(const MetricArgs& a, int32_t K, const Tin* phi, Tout* dT, cudaStream_t st);
// The same for one field (K = 1): phi (n, elimination order) shifted at a.src[0] into d.
void launch_shift_stats_one(const MetricArgs& a, const double* phi, double* d, cudaStream_t st);
// Health, MSD, distance to boundary, radii, perimeters and samples of each source's field.
template <typename T>
void launch_source_metrics(const MetricArgs& a, const T* dT, cudaStream_t st);

}  // namespace fcw
