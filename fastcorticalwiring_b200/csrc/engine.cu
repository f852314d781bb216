// Engine lifecycle, factorisation sequence, the per-block pipeline and the C ABI.
//
// One engine = one cortical submesh on one GPU. Creation prepares the mesh on
// the host, runs the symbolic analysis, uploads the structure and factors the
// heat operator M + tL and the Poisson operator L + shift*M in FP64 on the
// device (plus, for the mixed form, the Poisson operator grounded at the last
// eliminated vertex of each connected component, rounded to FP32). A block of K
// sources then runs:
//   reach -> heat forward (delta RHS, pruned) -> heat backward -> divergence
//   -> Poisson forward/backward -> shift + transpose -> vertex stats -> geometry
// entirely on one stream.
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "fcw_b200.h"
#include "fcw_internal.h"
#include "kernels.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define FCW_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(FCW_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define FCW_TRY(expr)            \
    do {                         \
        int rc_ = (expr);        \
        if (rc_ != FCW_OK) return rc_; \
    } while (0)

// Triangle-inequality margin of the robust operators' mollified edge lengths, relative to
// the mean edge length (the default of Sharp & Crane's intrinsic mollification).
constexpr double kMollifyFactor = 1e-6;

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

__global__ void k_map_sources(int64_t n, const int32_t* __restrict__ sources, const int32_t* __restrict__ iperm,
                              int32_t nv, int32_t K, int32_t* __restrict__ out, int* __restrict__ err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    int v = -1;
    if (k < n) {
        const int s = sources[k];
        if (s >= 0 && s < nv) v = iperm[s];
        else atomicOr(err, fcw::KERR_ARGS);
    }
    out[k] = v;
}

// The block's inputs into its workspace descriptor (ahead of the block's launch chain).
__global__ void k_set_block(fcw::BlockDesc* d, const int32_t* sources, int64_t n, double* out) {
    d->sources = sources;
    d->n = n;
    d->out = out;
}

// k_map_sources with the block's sources from the descriptor.
__global__ void k_map_block_sources(const fcw::BlockDesc* __restrict__ d, const int32_t* __restrict__ iperm,
                                    int32_t nv, int32_t K, int32_t* __restrict__ out, int* __restrict__ err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    int v = -1;
    if (k < d->n) {
        const int s = d->sources[k];
        if (s >= 0 && s < nv) v = iperm[s];
        else atomicOr(err, fcw::KERR_ARGS);
    }
    out[k] = v;
}

// Rows [0, k) of dT (K x n, one field per source, elimination order) -> out (k x n, caller order).
template <typename T>
__global__ void k_fields_out(int32_t n, int32_t k, const T* __restrict__ dT, const int32_t* __restrict__ iperm,
                             double* __restrict__ out) {
    const int64_t total = (int64_t)k * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / n), i = (int)(e - (int64_t)r * n);
        out[e] = (double)dT[(int64_t)r * n + iperm[i]];
    }
}

// d (k rows, caller vertex order) -> Y (n x K vertex-major, elimination order); columns >= k are zero.
__global__ void k_fields_in(int32_t n, int32_t k, int32_t K, const double* __restrict__ d,
                            const int32_t* __restrict__ iperm, double* __restrict__ Y) {
    const int64_t total = (int64_t)K * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / n), i = (int)(e - (int64_t)r * n);
        Y[(int64_t)iperm[i] * K + r] = r < k ? d[(int64_t)r * n + i] : 0.0;
    }
}

}  // namespace

struct Workspace {
    int32_t K = 0;
    double* Bh = nullptr;
    double* Bp64 = nullptr;
    float* Bp32 = nullptr;
    double* Y = nullptr;        // Poisson solution (n x K doubles, or floats for the mixed form)
    double* dT64 = nullptr;
    float* dT32 = nullptr;
    int32_t* src = nullptr;
    uint8_t* reach = nullptr;
    int4* band = nullptr;
    int32_t* longf = nullptr;
    double* out = nullptr;
    int32_t out_stride = 0;
    double* U = nullptr;        // forward update rows, (sum nr) x K doubles (reused as floats)
    double* partials = nullptr; // per (vertex tile, source) health/MSD partial sums
    double* csum = nullptr;     // per (vertex tile, source) component sums, then the levels (several components)
    int32_t* near_list = nullptr;
    int32_t* near_count = nullptr;
    cudaStream_t stream = nullptr;  // this workspace's stream in the pipelined device path
    cudaEvent_t done = nullptr;
    std::vector<std::pair<int, cudaEvent_t>> marks;  // stage timeline on this workspace
    double* part = nullptr;     // backward split-K partial sums
    int* counters = nullptr;    // split-K arrival tickets, zero at rest
    fcw::BlockDesc* desc = nullptr;     // the current block's inputs (device)
    // the block's launch chain captured as CUDA graphs, one per set of arguments (a few)
    struct Graph {
        std::vector<double> key;
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;           // kernels in the graph
    };
    std::vector<Graph> graphs;
    void drop_graph() {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
};

// The single-source drop-in (fcw_compute_distance): the narrow panel layouts of the two FP64
// factors, the task lists, its own vectors and sweep state, and its launch chain; built on
// its first call.
struct NarrowState {
    bool ready = false;
    fcw::NarrowLaunch L;
    int64_t* at_ptr = nullptr;
    double *at_h = nullptr, *at_p = nullptr;    // forward layouts of the heat and Poisson factors
    double *atb_h = nullptr, *atb_p = nullptr;  // backward layouts
    int4 *ftasks = nullptr, *btasks = nullptr;
    int32_t n_ftasks = 0, n_btasks = 0;
    double *u = nullptr, *div = nullptr, *y = nullptr, *out = nullptr;
    double* pend = nullptr;       // entries a sweep's readers poll: heat and Poisson update entries, heat
                                  // and Poisson solutions (set pending at the start of each call)
    int* sync = nullptr;          // the four sweeps' ticket counters
    // the heat forward's work list, built on the host per call: the source's elimination
    // index, the path's task count, then (task, previous supernode on the path) pairs
    int32_t* order = nullptr;
    int32_t* horder = nullptr;    // pinned host staging of the list
    std::vector<int32_t> fwd_first, nfwd_h;  // per supernode: first forward task, count
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;         // kernels per call
};

struct fcw_engine {
    fcw_params prm{};
    int device = 0;
    fcw::MeshPrep mesh;
    fcw::Symbolic sym;
    double t_coef = 0.0, t = 0.0;
    // the grounded (mixed-form) Poisson operator: one ground vertex per connected component of
    // the submesh, its last eliminated vertex; flags in the caller's order (host) and in
    // elimination order (device)
    std::vector<uint8_t> grounded_old;
    uint8_t* grounded_d = nullptr;
    // with several components: each vertex's component and lumped mass (elimination order) and
    // each component's total mass, for the mixed form's level on the source's component
    int32_t ncomp = 1;
    std::vector<int32_t> comp_h;
    std::vector<double> cmass_h, carea_h;
    fcw::ComponentLevel clevel;
    cudaStream_t stream = nullptr;
    std::vector<std::pair<void*, size_t>> allocs;  // device allocations and their sizes
    int64_t bytes = 0;
    fcw::DevPlan plan;
    std::vector<int32_t> level_tiles;
    // solve schedule: per level, task ranges of the forward / backward task lists
    std::vector<int32_t> fwd_ptr, bwd_ptr;
    std::vector<int32_t> level_rows;  // backward tile rows per level: 32 if all its supernodes are <= 32 wide
    std::vector<uint8_t> level_gathers;  // some supernode of the level has children
    int2 *fwd_tasks = nullptr, *bwd_tasks = nullptr;
    int64_t* uoff_d = nullptr;
    int64_t* poff_d = nullptr;
    int32_t* nsplit_d = nullptr;
    int32_t *gm_ptr_d = nullptr, *gm_src_d = nullptr, *gm_child_d = nullptr;
    int64_t n_urows = 0, n_parts = 0;
    double *val_h = nullptr, *inv_h = nullptr, *val_p = nullptr, *inv_p = nullptr;
    float *val_g = nullptr, *inv_g = nullptr;
    fcw::CsrOperator lg;  // the grounded Poisson operator in FP64, elimination order (refinement residuals)
    // tensor-core FP32 sweeps: core arrays of the grounded factor and the forward task list
    float *core_hi = nullptr, *core_lo = nullptr, *coreT_hi = nullptr, *coreT_lo = nullptr;
    int64_t* core_ptr_d = nullptr;
    int2* tc_fwd_tasks = nullptr;
    std::vector<int32_t> tc_fwd_ptr;
    fcw::FaceData fd;
    int32_t* iperm_d = nullptr;
    int32_t* perm_d = nullptr;
    double *coords_d = nullptr, *varea_d = nullptr, *farea_d = nullptr, *g11_d = nullptr, *g12_d = nullptr,
           *g22_d = nullptr;
    int32_t* boundary_d = nullptr;
    int4* inc_rec_d = nullptr;        // per incidence: face, corners (elimination order)
    long long* farea_fx_d = nullptr;  // lean face areas in fixed point
    double area_unscale = 0.0;
    int* err_d = nullptr;
    std::vector<Workspace> pool;  // blocks in flight: workspace i runs on pool[i].stream
    size_t cur_ws = 0;
    Workspace& cw() { return pool[cur_ws]; }
    cudaEvent_t ev_in = nullptr;  // the caller's stream at the start of a pipelined call
    int32_t* hsrc_d = nullptr;    // staging for the host-buffer metrics API
    double* hout_d = nullptr;
    int64_t hcap_src = 0, hcap_out = 0;
    float *hsr_d = nullptr, *hsa_d = nullptr;  // staging for the host-buffer sample assembly
    int32_t* hcnt_d = nullptr;
    int64_t hcap_smp = 0, hcap_cnt = 0;
    double* hdist_d = nullptr;  // staging for the host-buffer distances API (caller order)
    int64_t hcap_dist = 0;
    double analyze_ms = 0.0, factor_ms = 0.0;
    double lean_total = 0.0;  // sum of the lean face areas (the prefix total of a finite field)
    // stage timeline (CUDA events on the working stream), off unless enabled
    bool prof_on = false;
    bool graphs_on = true;  // replay each workspace's captured launch chain
    std::vector<cudaEvent_t> event_pool;
    double stage_ms[FCW_N_STAGES] = {0};
    int64_t launches = 0;
    int32_t num_sms = 148;  // the device's multiprocessors (grid sizes of grid-stride kernels)
    int64_t n_flips = 0;    // intrinsic edge flips of the robust operators
    NarrowState nar;

    // Device memory is stream-ordered (the device's default pool): freeing it
    // waits for this engine's streams only, never for other engines' work, so
    // engines can come and go while others run (the serving loop relies on it).
    template <typename T>
    int dalloc(T** p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        void* q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, count * sizeof(T), stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // usable from any stream from here on
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(FCW_E_NOMEM, "allocation of " + std::to_string(count * sizeof(T)) + " bytes failed: " +
                                         cudaGetErrorString(e));
        }
        allocs.emplace_back(q, count * sizeof(T));
        bytes += (int64_t)(count * sizeof(T));
        *p = static_cast<T*>(q);
        return FCW_OK;
    }
    // Waits for all of this engine's streams (the work that may still read its buffers).
    void sync_streams() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& w : pool)
            if (w.stream) cudaStreamSynchronize(w.stream);
    }
    template <typename T>
    int upload(T** p, const std::vector<T>& h) {
        FCW_TRY(dalloc(p, h.size()));
        if (!h.empty()) FCW_CUDA(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
        return FCW_OK;
    }
    void release(void* p) {
        for (size_t i = 0; i < allocs.size(); ++i)
            if (allocs[i].first == p) {
                sync_streams();
                cudaFreeAsync(p, stream);
                bytes -= (int64_t)allocs[i].second;
                allocs.erase(allocs.begin() + (long)i);
                return;
            }
    }
    ~fcw_engine() {
        sync_streams();
        for (auto& a : allocs) cudaFreeAsync(a.first, stream);
        if (stream) cudaStreamSynchronize(stream);
        for (auto& w : pool) {
            w.drop_graph();
            for (auto& m : w.marks) cudaEventDestroy(m.second);
            if (w.done) cudaEventDestroy(w.done);
            if (w.stream) cudaStreamDestroy(w.stream);
        }
        if (ev_in) cudaEventDestroy(ev_in);
        if (nar.exec) cudaGraphExecDestroy(nar.exec);
        if (nar.horder) cudaFreeHost(nar.horder);
        for (cudaEvent_t ev : event_pool) cudaEventDestroy(ev);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int check_kernel_errors(fcw_engine* e, const char* where) {
    int h = 0;
    FCW_CUDA(cudaMemcpyAsync(&h, e->err_d, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    FCW_CUDA(cudaStreamSynchronize(e->stream));
    if (h) {
        FCW_CUDA(cudaMemsetAsync(e->err_d, 0, sizeof(int), e->stream));
        std::string what;
        if (h & fcw::KERR_NOT_SPD) what += " non-positive pivot (operator not SPD);";
        if (h & fcw::KERR_HIST_OVERFLOW) what += " too many distance bins for one source;";
        if (h & fcw::KERR_SCRATCH) what += " per-source face list overflow;";
        if (h & fcw::KERR_ARGS) what += " invalid source index or launch arguments;";
        if (h & fcw::KERR_TIMEOUT) what += " a bounded device wait expired;";
        const int code = (h & fcw::KERR_ARGS) ? FCW_E_INVALID : (h & fcw::KERR_TIMEOUT) ? FCW_E_TIMEOUT : FCW_E_NUMERIC;
        return fail(code, std::string(where) + ":" + what);
    }
    return FCW_OK;
}

// Record a stage boundary: the stage `stage` starts here (-1 = end of a block).
void mark(fcw_engine* e, cudaStream_t st, int stage) {
    if (!e->prof_on) return;
    cudaEvent_t ev;
    if (!e->event_pool.empty()) {
        ev = e->event_pool.back();
        e->event_pool.pop_back();
    } else if (cudaEventCreate(&ev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    cudaEventRecord(ev, st);
    e->cw().marks.push_back({stage, ev});
}

int collect_marks(fcw_engine* e) {
    for (auto& w : e->pool) {
        auto& marks = w.marks;
        if (marks.empty()) continue;
        FCW_CUDA(cudaEventSynchronize(marks.back().second));
        for (size_t j = 0; j + 1 < marks.size(); ++j) {
            const int stg = marks[j].first;
            if (stg < 0 || stg >= FCW_N_STAGES) continue;
            float ms = 0.0f;
            FCW_CUDA(cudaEventElapsedTime(&ms, marks[j].second, marks[j + 1].second));
            e->stage_ms[stg] += ms;
        }
        for (auto& m : marks) e->event_pool.push_back(m.second);
        marks.clear();
    }
    return FCW_OK;
}

int validate_params(const fcw_params* p) {
    if (!p) return fail(FCW_E_INVALID, "params is NULL");
    if (!std::isfinite(p->diffusion_length_mm) || p->diffusion_length_mm < 0.5)
        return fail(FCW_E_INVALID, "diffusion_length_mm must be finite and at least 0.5 mm.");
    if (!std::isfinite(p->poisson_shift) || p->poisson_shift < 0.0) return fail(FCW_E_INVALID, "invalid poisson_shift");
    if (p->block_k < 64 || p->block_k % 64 != 0 || p->block_k > 4096)
        return fail(FCW_E_INVALID, "block_k must be a multiple of 64 in [64, 4096]");
    if (p->leaf_size < 1 || p->max_width < 1 || p->max_width > fcw::kMaxWidth)
        return fail(FCW_E_INVALID, "max_width must be in [1, 64] and leaf_size >= 1");
    if (p->relax < 1 || p->relax > p->max_width) return fail(FCW_E_INVALID, "relax must be in [1, max_width]");
    if (p->pipeline_depth < 1 || p->pipeline_depth > 8) return fail(FCW_E_INVALID, "pipeline_depth must be in [1, 8]");
    if (p->tc_sweeps != 0 && p->tc_sweeps != 1) return fail(FCW_E_INVALID, "tc_sweeps must be 0 or 1");
    if (p->robust != 0 && p->robust != 1) return fail(FCW_E_INVALID, "robust must be 0 or 1");
    if (p->refine < 0 || p->refine > 4) return fail(FCW_E_INVALID, "refine must be in [0, 4]");
    return FCW_OK;
}

// Connected components of the submesh (union-find over its faces; core_analysis.py:1349-1381
// reports the same ones): comp[v] for each vertex v, numbered in order of first appearance in
// the elimination order perm. Returns their count.
int32_t mesh_components(const fcw::MeshPrep& m, const std::vector<int32_t>& perm, std::vector<int32_t>& comp) {
    const int64_t n = m.nv;
    std::vector<int32_t> up(n);
    for (int64_t i = 0; i < n; ++i) up[i] = (int32_t)i;
    auto find = [&](int32_t x) {
        while (up[x] != x) x = up[x] = up[up[x]];
        return x;
    };
    for (int64_t f = 0; f < m.nf; ++f)
        for (int c = 1; c < 3; ++c) {
            const int32_t a = find(m.F[3 * f]), b = find(m.F[3 * f + c]);
            if (a != b) up[std::max(a, b)] = std::min(a, b);
        }
    std::vector<int32_t> label(n, -1);
    comp.assign(n, -1);
    int32_t count = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int32_t v = perm[i], r = find(v);
        if (label[r] < 0) label[r] = count++;
        comp[v] = label[r];
    }
    return count;
}

// Values of A's lower entries in the symbolic analysis' order.
enum class Op { Heat, Poisson, Grounded };
std::vector<double> operator_values(const fcw_engine* e, Op op) {
    const auto& S = e->sym;
    const auto& m = e->mesh;
    std::vector<double> v(S.nnz_lower_a);
    for (int64_t q = 0; q < S.nnz_lower_a; ++q) {
        const int64_t k = S.a_src[q];
        const int32_t col = S.a_col[q], row = m.Li[k];
        const bool diag = row == col;
        const double L = m.Lx[k];
        switch (op) {
            case Op::Heat:  // M + t L (fastcw_lean.py:498)
                v[q] = diag ? m.mass[col] + e->t * L : e->t * L;
                break;
            case Op::Poisson:  // L + shift M (fastcw_lean.py:500)
                v[q] = diag ? L + e->prm.poisson_shift * m.mass[col] : L;
                break;
            case Op::Grounded:  // L with the ground vertices' rows and columns replaced by the identity
                v[q] = (e->grounded_old[row] || e->grounded_old[col]) ? (diag ? 1.0 : 0.0) : L;
                break;
        }
    }
    return v;
}

}  // namespace

// ---------------------------------------------------------------------------
// engine construction
// ---------------------------------------------------------------------------
namespace {

int build_engine(fcw_engine* e, const double* V, int64_t nv, const int32_t* F, int64_t nf) {
    std::string err;
    double t0 = now_ms();
    if (fcw::prepare_mesh(V, nv, F, nf, e->mesh, err)) return fail(FCW_E_INVALID, err);
    if (e->prm.robust && fcw::intrinsic_delaunay(e->mesh, kMollifyFactor, e->n_flips, err))
        return fail(FCW_E_INVALID, err);
    e->t_coef = std::pow(e->prm.diffusion_length_mm / e->mesh.mean_edge, 2.0);
    e->t = e->t_coef * e->mesh.mean_edge * e->mesh.mean_edge;
    if (fcw::build_symbolic(e->mesh, e->prm.leaf_size, e->prm.max_width, e->prm.relax, e->sym, err)) return fail(FCW_E_INVALID, err);
    e->analyze_ms = now_ms() - t0;
    const auto& S = e->sym;
    const auto& m = e->mesh;
    if (S.max_ns > fcw::kMaxWidth) return fail(FCW_E_INVALID, "supernode wider than the kernels support");
    {
        // each connected component grounded at its last eliminated vertex: L is singular once
        // per component
        std::vector<int32_t> comp;
        e->ncomp = mesh_components(m, S.perm, comp);
        std::vector<int32_t> last(e->ncomp, -1);
        for (int64_t i = 0; i < S.n; ++i) last[comp[S.perm[i]]] = (int32_t)i;  // ascending i: the last wins
        e->grounded_old.assign(S.n, 0);
        for (int32_t c = 0; c < e->ncomp; ++c) e->grounded_old[S.perm[last[c]]] = 1;
        if (e->ncomp > 1) {
            e->comp_h.resize(S.n);
            e->cmass_h.resize(S.n);
            e->carea_h.assign(e->ncomp, 0.0);
            for (int64_t i = 0; i < S.n; ++i) {
                e->comp_h[i] = comp[S.perm[i]];
                e->cmass_h[i] = m.mass[S.perm[i]];
                e->carea_h[e->comp_h[i]] += e->cmass_h[i];
            }
        }
    }

    FCW_CUDA(cudaSetDevice(e->device));
    FCW_CUDA(cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->device));
    FCW_CUDA(fcw::configure_kernels());
    FCW_CUDA(fcw::configure_solve_kernels());
    FCW_CUDA(fcw::configure_tc_kernels());
    FCW_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    FCW_CUDA(cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming));
    e->pool.resize((size_t)std::max(1, e->prm.pipeline_depth));
    for (auto& w : e->pool) {
        FCW_CUDA(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking));
        FCW_CUDA(cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming));
    }
    FCW_TRY(e->dalloc(&e->err_d, 1));
    FCW_CUDA(cudaMemset(e->err_d, 0, sizeof(int)));

    // structure
    int32_t *sn_c0, *sn_m, *rows, *sn_parent, *col_sn, *level_nodes, *child_ptr, *child_list, *relind, *seg_sn,
        *seg_pos;
    int64_t *sn_rowptr, *sn_valptr, *sn_invptr, *sn_updptr, *seg_ptr, *a_dst;
    FCW_TRY(e->upload(&sn_c0, S.sn_c0));
    FCW_TRY(e->upload(&sn_m, S.sn_m));
    FCW_TRY(e->upload(&sn_rowptr, S.sn_rowptr));
    FCW_TRY(e->upload(&rows, S.rows));
    FCW_TRY(e->upload(&sn_valptr, S.sn_valptr));
    FCW_TRY(e->upload(&sn_invptr, S.sn_invptr));
    FCW_TRY(e->upload(&sn_updptr, S.sn_updptr));
    FCW_TRY(e->upload(&sn_parent, S.sn_parent));
    FCW_TRY(e->upload(&col_sn, S.col_sn));
    FCW_TRY(e->upload(&level_nodes, S.level_nodes));
    FCW_TRY(e->upload(&child_ptr, S.child_ptr));
    FCW_TRY(e->upload(&child_list, S.child_list));
    FCW_TRY(e->upload(&relind, S.relind));
    FCW_TRY(e->upload(&seg_ptr, S.seg_ptr));
    FCW_TRY(e->upload(&seg_sn, S.seg_sn));
    FCW_TRY(e->upload(&seg_pos, S.seg_pos));
    FCW_TRY(e->upload(&a_dst, S.a_dst));
    fcw::DevPlan& P = e->plan;
    P.n = (int32_t)S.n;
    P.nsuper = S.nsuper;
    P.nlevels = S.nlevels;
    P.sn_c0 = sn_c0; P.sn_m = sn_m; P.sn_rowptr = sn_rowptr; P.rows = rows; P.sn_valptr = sn_valptr;
    P.sn_invptr = sn_invptr; P.sn_updptr = sn_updptr; P.sn_parent = sn_parent; P.col_sn = col_sn;
    P.level_nodes = level_nodes; P.child_ptr = child_ptr; P.child_list = child_list; P.relind = relind;
    P.seg_ptr = seg_ptr; P.seg_sn = seg_sn; P.seg_pos = seg_pos;
    e->level_tiles.assign(S.nlevels, 1);
    for (int32_t l = 0; l < S.nlevels; ++l) {
        int64_t mx = 1;
        for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
            const int32_t s = S.level_nodes[q];
            const int64_t nr = S.sn_m[s] - (S.sn_c0[s + 1] - S.sn_c0[s]);
            const int64_t nt = (nr + 31) / 32;
            mx = std::max<int64_t>(mx, nt * (nt + 1) / 2);
        }
        e->level_tiles[l] = (int32_t)std::min<int64_t>(mx, 512);
    }

    // solve schedule (see solve.cu): forward row-chunk tasks, backward split-K tasks,
    // update-row offsets and the per-front-row gather lists of children's update rows
    {
        const int32_t NS = S.nsuper;
        std::vector<int64_t> uoff(NS + 1, 0), poff(NS, 0);
        std::vector<int32_t> nsplit(NS, 1);
        int64_t parts = 0;
        for (int32_t s = 0; s < NS; ++s) {
            const int32_t ns = S.sn_c0[s + 1] - S.sn_c0[s], nr = S.sn_m[s] - ns;
            uoff[s + 1] = uoff[s] + nr;
            nsplit[s] = std::max(1, (nr + fcw::kSplitRows - 1) / fcw::kSplitRows);
            poff[s] = parts;
            if (nsplit[s] > 1) parts += nsplit[s];
        }
        e->n_urows = uoff[NS];
        e->n_parts = parts;
        std::vector<int2> ft, bt, tft;
        e->tc_fwd_ptr.assign(S.nlevels + 1, 0);
        e->fwd_ptr.assign(S.nlevels + 1, 0);
        e->bwd_ptr.assign(S.nlevels + 1, 0);
        e->level_rows.assign(S.nlevels, fcw::kMaxWidth);
        e->level_gathers.assign(S.nlevels, 0);
        for (int32_t l = 0; l < S.nlevels; ++l) {
            int32_t widest = 0;
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
                const int32_t s = S.level_nodes[q];
                widest = std::max(widest, S.sn_c0[s + 1] - S.sn_c0[s]);
                if (S.child_ptr[s + 1] > S.child_ptr[s]) e->level_gathers[l] = 1;
            }
            // narrow backward tiles on the leaf levels; the forward sweep keeps 64-row
            // tasks everywhere (32-row tasks would recompute X_s for twice as many chunks)
            e->level_rows[l] = widest <= 32 ? 32 : fcw::kMaxWidth;
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
                const int32_t s = S.level_nodes[q];
                const int32_t ns = S.sn_c0[s + 1] - S.sn_c0[s], nr = S.sn_m[s] - ns;
                const int32_t nch = std::max(1, (nr + fcw::kMaxWidth - 1) / fcw::kMaxWidth);
                for (int32_t c = 0; c < nch; ++c) ft.push_back(make_int2(s, c));
                for (int32_t c = 0; c < nsplit[s]; ++c) bt.push_back(make_int2(s, c));
            }
            e->fwd_ptr[l + 1] = (int32_t)ft.size();
            e->bwd_ptr[l + 1] = (int32_t)bt.size();
            // tensor-core forward: per supernode the inverse block with the first 64 update rows,
            // then 128-row update chunks
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
                const int32_t s = S.level_nodes[q];
                const int32_t ns = S.sn_c0[s + 1] - S.sn_c0[s], nr = S.sn_m[s] - ns;
                const int32_t nchunk = 1 + std::max(0, (nr - 64 + 127) / 128);
                for (int32_t c = 0; c < nchunk; ++c) tft.push_back(make_int2(s, c));
            }
            e->tc_fwd_ptr[l + 1] = (int32_t)tft.size();
        }
        const int64_t nfront = S.sn_rowptr[NS];
        std::vector<int32_t> gptr(nfront + 1, 0), gsrc(e->n_urows), gchild(e->n_urows);
        for (int32_t c = 0; c < NS; ++c) {
            const int32_t p = S.sn_parent[c];
            const int32_t nsc = S.sn_c0[c + 1] - S.sn_c0[c];
            for (int64_t q = S.sn_rowptr[c] + nsc; q < S.sn_rowptr[c + 1]; ++q) gptr[S.sn_rowptr[p] + S.relind[q] + 1]++;
        }
        for (int64_t g = 0; g < nfront; ++g) gptr[g + 1] += gptr[g];
        {
            std::vector<int32_t> fill(gptr.begin(), gptr.end() - 1);
            for (int32_t c = 0; c < NS; ++c) {
                const int32_t p = S.sn_parent[c];
                const int32_t nsc = S.sn_c0[c + 1] - S.sn_c0[c];
                for (int64_t q = S.sn_rowptr[c] + nsc; q < S.sn_rowptr[c + 1]; ++q) {
                    const int64_t g = S.sn_rowptr[p] + S.relind[q];
                    gsrc[fill[g]] = (int32_t)(uoff[c] + (q - S.sn_rowptr[c] - nsc));
                    gchild[fill[g]] = c;
                    fill[g]++;
                }
            }
        }
        if (e->n_urows > INT32_MAX || nfront > INT32_MAX) return fail(FCW_E_INVALID, "mesh too large for 32-bit update indices");
        FCW_TRY(e->upload(&e->fwd_tasks, ft));
        FCW_TRY(e->upload(&e->bwd_tasks, bt));
        FCW_TRY(e->upload(&e->tc_fwd_tasks, tft));
        FCW_TRY(e->upload(&e->uoff_d, uoff));
        FCW_TRY(e->upload(&e->poff_d, poff));
        FCW_TRY(e->upload(&e->nsplit_d, nsplit));
        FCW_TRY(e->upload(&e->gm_ptr_d, gptr));
        FCW_TRY(e->upload(&e->gm_src_d, gsrc));
        FCW_TRY(e->upload(&e->gm_child_d, gchild));
    }

    // mesh arrays in elimination order
    const int64_t n = S.n;
    std::vector<double> coords(3 * n), varea(n);
    for (int64_t j = 0; j < n; ++j) {
        const int32_t o = S.perm[j];
        for (int c = 0; c < 3; ++c) coords[3 * j + c] = m.V[3 * (int64_t)o + c];
        varea[j] = m.vertex_area[o];
    }
    std::vector<int32_t> fv(3 * nf), bnd(m.boundary.size());
    for (int64_t i = 0; i < 3 * nf; ++i) fv[i] = S.iperm[m.F[i]];
    for (size_t i = 0; i < m.boundary.size(); ++i) bnd[i] = S.iperm[m.boundary[i]];
    std::vector<float> coef(4 * nf);
    for (int64_t f = 0; f < nf; ++f) {
        const double* g = &m.gb[9 * f];
        const double c11 = g[3] * g[3] + g[4] * g[4] + g[5] * g[5];
        const double c12 = g[3] * g[6] + g[4] * g[7] + g[5] * g[8];
        const double c22 = g[6] * g[6] + g[7] * g[7] + g[8] * g[8];
        coef[4 * f] = (float)c11; coef[4 * f + 1] = (float)c12; coef[4 * f + 2] = (float)c22;
        coef[4 * f + 3] = (float)m.grad_area[f];
    }
    std::vector<int32_t> inc_ptr(n + 1, 0), inc_face(3 * nf);
    std::vector<int8_t> inc_corner(3 * nf);
    for (int64_t i = 0; i < 3 * nf; ++i) inc_ptr[fv[i] + 1]++;
    for (int64_t j = 0; j < n; ++j) inc_ptr[j + 1] += inc_ptr[j];
    {
        std::vector<int32_t> fill(inc_ptr.begin(), inc_ptr.end() - 1);
        for (int64_t f = 0; f < nf; ++f)
            for (int c = 0; c < 3; ++c) {
                const int32_t v = fv[3 * f + c];
                inc_face[fill[v]] = (int32_t)f;
                inc_corner[fill[v]] = (int8_t)c;
                fill[v]++;
            }
    }
    // the same incidences as records holding the face's corners, and the face areas
    // in a fixed point whose full scale is 2^62 >= the total, so that per-bin
    // sums are exact and independent of the order atomics add them in
    std::vector<int4> inc_rec(3 * nf);
    for (int64_t q = 0; q < 3 * nf; ++q) {
        const int32_t f = inc_face[q];
        inc_rec[q] = make_int4(f, fv[3 * f], fv[3 * f + 1], fv[3 * f + 2]);
    }
    double lean_sum = 0.0;
    for (double x : m.lean_area) lean_sum += x;
    const int area_exp = lean_sum > 0.0 ? (int)std::ceil(std::log2(lean_sum)) : 0;
    const double area_scale = std::ldexp(1.0, 62 - area_exp);
    std::vector<long long> farea_fx(nf);
    for (int64_t f = 0; f < nf; ++f) farea_fx[f] = std::llround(m.lean_area[f] * area_scale);
    e->area_unscale = 1.0 / area_scale;
    FCW_TRY(e->upload(&e->inc_rec_d, inc_rec));
    FCW_TRY(e->upload(&e->farea_fx_d, farea_fx));
    std::vector<int4> inc_corners(3 * nf);
    std::vector<float4> inc_coef(3 * nf);
    std::vector<float2> inc_w(3 * nf);
    for (int64_t q = 0; q < 3 * nf; ++q) {
        const int32_t f = inc_face[q];
        const float c11 = coef[4 * f], c12 = coef[4 * f + 1], c22 = coef[4 * f + 2];
        inc_corners[q] = make_int4(fv[3 * f], fv[3 * f + 1], fv[3 * f + 2], inc_corner[q]);
        inc_coef[q] = make_float4(c11, c12, c22, coef[4 * f + 3]);
        // the corner weights in FP32, as the kernel's form defines them
        if (inc_corner[q] == 0) inc_w[q] = make_float2(-(c11 + c12), -(c12 + c22));
        else if (inc_corner[q] == 1) inc_w[q] = make_float2(c11, c12);
        else inc_w[q] = make_float2(c12, c22);
    }
    int4* inc_corners_d;
    float4* inc_coef_d;
    float2* inc_w_d;
    FCW_TRY(e->upload(&inc_corners_d, inc_corners));
    FCW_TRY(e->upload(&inc_coef_d, inc_coef));
    FCW_TRY(e->upload(&inc_w_d, inc_w));
    int32_t *fv_d, *inc_ptr_d, *inc_face_d;
    int8_t* inc_corner_d;
    double *gb_d, *garea_d;
    float* coef_d;
    FCW_TRY(e->upload(&fv_d, fv));
    FCW_TRY(e->upload(&gb_d, m.gb));
    FCW_TRY(e->upload(&garea_d, m.grad_area));
    FCW_TRY(e->upload(&coef_d, coef));
    FCW_TRY(e->upload(&inc_ptr_d, inc_ptr));
    FCW_TRY(e->upload(&inc_face_d, inc_face));
    FCW_TRY(e->upload(&inc_corner_d, inc_corner));
    e->fd.nv = (int32_t)n; e->fd.nf = (int32_t)nf; e->fd.fv = fv_d; e->fd.gb = gb_d; e->fd.garea = garea_d;
    e->fd.coef = coef_d; e->fd.inc_ptr = inc_ptr_d; e->fd.inc_face = inc_face_d; e->fd.inc_corner = inc_corner_d;
    e->fd.inc_corners = inc_corners_d; e->fd.inc_coef = inc_coef_d; e->fd.inc_w = inc_w_d;
    FCW_TRY(e->upload(&e->coords_d, coords));
    FCW_TRY(e->upload(&e->varea_d, varea));
    FCW_TRY(e->upload(&e->boundary_d, bnd));
    FCW_TRY(e->upload(&e->farea_d, m.lean_area));
    e->lean_total = 0.0;
    for (double x : m.lean_area) e->lean_total += x;
    FCW_TRY(e->upload(&e->g11_d, m.g11));
    FCW_TRY(e->upload(&e->g12_d, m.g12));
    FCW_TRY(e->upload(&e->g22_d, m.g22));
    FCW_TRY(e->upload(&e->iperm_d, S.iperm));
    {
        std::vector<uint8_t> gnew(S.n);
        for (int64_t i = 0; i < S.n; ++i) gnew[i] = e->grounded_old[S.perm[i]];
        FCW_TRY(e->upload(&e->grounded_d, gnew));
    }
    if (e->ncomp > 1) {
        e->clevel.n = (int32_t)S.n;
        FCW_TRY(e->upload(&e->clevel.comp, e->comp_h));
        FCW_TRY(e->upload(&e->clevel.mass, e->cmass_h));
        FCW_TRY(e->upload(&e->clevel.area, e->carea_h));
    }
    FCW_TRY(e->upload(&e->perm_d, S.perm));

    // numeric factorisations
    t0 = now_ms();
    double *upd, *aval_d;
    FCW_TRY(e->dalloc(&upd, S.n_upd));
    FCW_TRY(e->dalloc(&aval_d, S.nnz_lower_a));
    FCW_TRY(e->dalloc(&e->val_h, S.nnz_factor));
    FCW_TRY(e->dalloc(&e->inv_h, S.n_inv));
    FCW_TRY(e->dalloc(&e->val_p, S.nnz_factor));
    FCW_TRY(e->dalloc(&e->inv_p, S.n_inv));
    auto run_factor = [&](Op op, double* val, double* inv, const char* what) -> int {
        std::vector<double> av = operator_values(e, op);
        FCW_CUDA(cudaMemcpyAsync(aval_d, av.data(), av.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        FCW_CUDA(cudaMemsetAsync(val, 0, S.nnz_factor * sizeof(double), e->stream));
        FCW_CUDA(cudaMemsetAsync(upd, 0, std::max<int64_t>(S.n_upd, 1) * sizeof(double), e->stream));
        fcw::launch_scatter_a(S.nnz_lower_a, a_dst, aval_d, val, e->stream);
        for (int32_t l = 0; l < S.nlevels; ++l) {
            const int32_t l0 = S.level_ptr[l], cnt = S.level_ptr[l + 1] - l0;
            fcw::launch_factor_front(e->plan, l0, cnt, val, inv, upd, e->err_d, e->stream);
            fcw::launch_factor_update(e->plan, l0, cnt, e->level_tiles[l], val, upd, e->stream);
        }
        fcw::launch_panel_inverse(e->plan, val, inv, e->stream);
        FCW_CUDA(cudaGetLastError());
        return check_kernel_errors(e, what);
    };
    FCW_TRY(run_factor(Op::Heat, e->val_h, e->inv_h, "heat factorisation"));
    FCW_TRY(run_factor(Op::Poisson, e->val_p, e->inv_p, "Poisson factorisation"));
    if (e->prm.build_mixed && e->prm.refine > 0) {
        // L_g in CSR, elimination order: the entries the FP32 factor came from
        std::vector<int64_t> rp(S.n + 1, 0);
        std::vector<int32_t> ci;
        std::vector<double> av;
        ci.reserve(m.Li.size());
        av.reserve(m.Li.size());
        for (int64_t i = 0; i < S.n; ++i) {
            const int32_t old = S.perm[i];
            for (int64_t k = m.Lp[old]; k < m.Lp[old + 1]; ++k) {
                const int32_t j = m.Li[k];
                const bool diag = j == old;
                const double v = (e->grounded_old[old] || e->grounded_old[j]) ? (diag ? 1.0 : 0.0) : m.Lx[k];
                if (v == 0.0 && !diag) continue;
                ci.push_back(S.iperm[j]);
                av.push_back(v);
            }
            rp[i + 1] = (int64_t)ci.size();
        }
        int64_t* rp_d;
        int32_t* ci_d;
        double* av_d;
        FCW_TRY(e->upload(&rp_d, rp));
        FCW_TRY(e->upload(&ci_d, ci));
        FCW_TRY(e->upload(&av_d, av));
        e->lg.n = (int32_t)S.n;
        e->lg.rp = rp_d;
        e->lg.ci = ci_d;
        e->lg.av = av_d;
    }
    if (e->prm.build_mixed) {
        double *val_tmp, *inv_tmp;
        FCW_TRY(e->dalloc(&val_tmp, S.nnz_factor));
        FCW_TRY(e->dalloc(&inv_tmp, S.n_inv));
        FCW_TRY(run_factor(Op::Grounded, val_tmp, inv_tmp, "grounded Poisson factorisation"));
        FCW_TRY(e->dalloc(&e->val_g, S.nnz_factor));
        FCW_TRY(e->dalloc(&e->inv_g, S.n_inv));
        fcw::launch_to_float(S.nnz_factor, val_tmp, e->val_g, e->stream);
        fcw::launch_to_float(S.n_inv, inv_tmp, e->inv_g, e->stream);
        if (e->prm.tc_sweeps) {
            std::vector<int64_t> cptr(S.nsuper + 1, 0);
            for (int32_t s = 0; s < S.nsuper; ++s) {
                const int64_t ns = S.sn_c0[s + 1] - S.sn_c0[s], nr = S.sn_m[s] - ns;
                const int64_t ns8 = (ns + 7) / 8 * 8, nr32 = (nr + 31) / 32 * 32;
                cptr[s + 1] = cptr[s] + ns8 * (ns8 + nr32);
            }
            FCW_TRY(e->upload(&e->core_ptr_d, cptr));
            FCW_TRY(e->dalloc(&e->core_hi, (size_t)cptr[S.nsuper]));
            FCW_TRY(e->dalloc(&e->core_lo, (size_t)cptr[S.nsuper]));
            FCW_TRY(e->dalloc(&e->coreT_hi, (size_t)cptr[S.nsuper]));
            FCW_TRY(e->dalloc(&e->coreT_lo, (size_t)cptr[S.nsuper]));
            fcw::launch_build_cores(e->plan, val_tmp, inv_tmp, e->core_ptr_d, e->core_hi, e->core_lo, e->coreT_hi,
                                    e->coreT_lo, e->stream);
            FCW_CUDA(cudaGetLastError());
        }
        FCW_CUDA(cudaStreamSynchronize(e->stream));
        e->release(val_tmp);
        e->release(inv_tmp);
    }
    FCW_CUDA(cudaStreamSynchronize(e->stream));
    e->release(upd);
    e->release(aval_d);
    e->factor_ms = now_ms() - t0;
    return FCW_OK;
}

int ensure_one(fcw_engine* e, Workspace& w, int32_t K, int32_t stride) {
    if (w.K >= K && w.out_stride >= stride) return FCW_OK;
    const int32_t Kn = std::max(K, w.K);
    const int32_t sn = std::max(stride, w.out_stride);
    void* old[] = {w.Bh, w.Bp64, w.Y, w.dT64, w.src, w.reach, w.band, w.longf, w.out, w.U, w.part,
                   w.counters, w.partials, w.near_list, w.near_count, w.desc, w.csum};
    for (void* p : old)
        if (p) e->release(p);
    w.drop_graph();  // its launches name the old buffers
    cudaStream_t stream = w.stream;
    cudaEvent_t done = w.done;
    w = Workspace{};
    w.stream = stream;
    w.done = done;
    const int64_t n = e->sym.n, nf = e->mesh.nf;
    FCW_TRY(e->dalloc(&w.Bh, (size_t)n * Kn));
    FCW_TRY(e->dalloc(&w.Bp64, (size_t)n * Kn));
    w.Bp32 = reinterpret_cast<float*>(w.Bp64);  // a block uses one precision
    FCW_TRY(e->dalloc(&w.Y, (size_t)n * Kn));
    FCW_TRY(e->dalloc(&w.dT64, (size_t)n * Kn));
    w.dT32 = reinterpret_cast<float*>(w.dT64);
    FCW_TRY(e->dalloc(&w.src, (size_t)Kn));
    FCW_TRY(e->dalloc(&w.reach, (size_t)std::max<int64_t>(e->sym.nsuper, 1) * (Kn / fcw::kReachCols)));
    FCW_TRY(e->dalloc(&w.band, (size_t)nf * Kn));
    FCW_TRY(e->dalloc(&w.longf, (size_t)nf * Kn));
    FCW_TRY(e->dalloc(&w.out, (size_t)sn * Kn));
    const int64_t ntiles = (n + fcw::kStatVTile - 1) / fcw::kStatVTile;
    FCW_TRY(e->dalloc(&w.partials, (size_t)ntiles * Kn * 8));
    FCW_TRY(e->dalloc(&w.near_list, (size_t)n * Kn));
    FCW_TRY(e->dalloc(&w.near_count, (size_t)Kn));
    FCW_TRY(e->dalloc(&w.U, (size_t)std::max<int64_t>(e->n_urows, 1) * Kn));
    FCW_TRY(e->dalloc(&w.part, (size_t)std::max<int64_t>(e->n_parts, 1) * fcw::kMaxWidth * Kn));
    const int64_t nctr = (int64_t)std::max<int32_t>(e->sym.nsuper, 1) * (Kn / fcw::kRhsTile);
    FCW_TRY(e->dalloc(&w.counters, (size_t)nctr));
    FCW_CUDA(cudaMemset(w.counters, 0, nctr * sizeof(int)));
    FCW_TRY(e->dalloc(&w.desc, 1));
    if (e->ncomp > 1) FCW_TRY(e->dalloc(&w.csum, (size_t)(fcw::component_tiles(n) + 1) * Kn));
    w.K = Kn;
    w.out_stride = sn;
    return FCW_OK;
}

// Every workspace of the pool holds at least K columns and `stride` output doubles per column.
// If the device cannot hold another workspace, the pool keeps the ones that fit (at least
// one): fewer blocks are in flight, nothing else changes.
int ensure_workspace(fcw_engine* e, int32_t K, int32_t stride) {
    for (size_t i = 0; i < e->pool.size(); ++i) {
        const int rc = ensure_one(e, e->pool[i], K, stride);
        if (rc == FCW_OK) continue;
        if (i == 0 || rc != FCW_E_NOMEM) return rc;
        e->sync_streams();
        for (size_t j = i; j < e->pool.size(); ++j) {
            Workspace& w = e->pool[j];
            void* bufs[] = {w.Bh, w.Bp64, w.Y, w.dT64, w.src, w.reach, w.band, w.longf, w.out, w.U, w.part,
                            w.counters, w.partials, w.near_list, w.near_count, w.desc, w.csum};
            for (void* p : bufs)
                if (p) e->release(p);
            w.drop_graph();
            for (auto& m : w.marks) cudaEventDestroy(m.second);
            if (w.done) cudaEventDestroy(w.done);
            if (w.stream) cudaStreamDestroy(w.stream);
        }
        e->pool.resize(i);
        e->cur_ws = 0;
        return FCW_OK;
    }
    return FCW_OK;
}

template <typename T>
fcw::SolveArgs<T> solve_args(fcw_engine* e, const T* val, const T* inv, T* B, int32_t K) {
    fcw::SolveArgs<T> a;
    a.p = e->plan;
    a.val = val;
    a.inv = inv;
    a.B = B;
    a.K = K;
    a.U = reinterpret_cast<T*>(e->cw().U);
    a.uoff = e->uoff_d;
    a.gm_ptr = e->gm_ptr_d;
    a.gm_src = e->gm_src_d;
    a.gm_child = e->gm_child_d;
    a.nsplit = e->nsplit_d;
    a.poff = e->poff_d;
    a.part = reinterpret_cast<T*>(e->cw().part);
    a.counters = e->cw().counters;
    a.ktiles = e->cw().K / fcw::kRhsTile;
    a.core_hi = e->core_hi;
    a.core_lo = e->core_lo;
    a.coreT_hi = e->coreT_hi;
    a.coreT_lo = e->coreT_lo;
    a.core_ptr = e->core_ptr_d;
    a.err = e->err_d;
    return a;
}

template <typename T>
void sweep(fcw_engine* e, fcw::SolveArgs<T> a, cudaStream_t st, int stage_fwd, int stage_bwd) {
    const auto& S = e->sym;
    mark(e, st, stage_fwd);
    for (int32_t l = 0; l < S.nlevels; ++l) {
        a.tasks = e->fwd_tasks;
        fcw::launch_fwd_level<T>(a, e->fwd_ptr[l], e->fwd_ptr[l + 1] - e->fwd_ptr[l], e->level_gathers[l] != 0, st);
    }
    a.delta_src = nullptr;
    mark(e, st, stage_bwd);
    for (int32_t l = S.nlevels - 1; l >= 0; --l) {
        a.tasks = e->bwd_tasks;
        fcw::launch_bwd_level<T>(a, e->bwd_ptr[l], e->bwd_ptr[l + 1] - e->bwd_ptr[l], e->level_rows[l], st);
    }
    e->launches += 2 * (int64_t)S.nlevels;
}

// Heat solve for the K sources in ws.src: u (elimination order, n x K) in ws.Bh.
void heat_solve(fcw_engine* e, int32_t K, cudaStream_t st) {
    Workspace& w = e->cw();
    mark(e, st, FCW_STAGE_HEAT_FWD);
    fcw::launch_reach(e->plan, w.src, K, w.reach, st);
    e->launches += 2;
    fcw::SolveArgs<double> a = solve_args<double>(e, e->val_h, e->inv_h, w.Bh, K);
    a.delta_src = w.src;
    a.reach = w.reach;
    a.reach_tiles = K / fcw::kReachCols;
    sweep<double>(e, a, st, FCW_STAGE_HEAT_FWD, FCW_STAGE_HEAT_BWD);
}

// FP32 sweeps on the tensor cores: the same level schedule, the forward with its own task list.
int sweep_tc(fcw_engine* e, fcw::SolveArgs<float> a, cudaStream_t st) {
    const auto& S = e->sym;
    CUtensorMap rmap, bmap;
    if (fcw::make_rows_map(&rmap, a.R, S.n, a.K) || fcw::make_rows_map(&bmap, a.B, S.n, a.K))
        return fail(FCW_E_CUDA, "cuTensorMapEncodeTiled failed for the Poisson right-hand sides");
    mark(e, st, FCW_STAGE_POISSON_FWD);
    a.tasks = e->tc_fwd_tasks;
    for (int32_t l = 0; l < S.nlevels; ++l)
        fcw::launch_fwd_level_tc(a, e->tc_fwd_ptr[l], e->tc_fwd_ptr[l + 1] - e->tc_fwd_ptr[l], rmap, st);
    mark(e, st, FCW_STAGE_POISSON_BWD);
    a.tasks = e->bwd_tasks;
    for (int32_t l = S.nlevels - 1; l >= 0; --l)
        fcw::launch_bwd_level_tc(a, e->bwd_ptr[l], e->bwd_ptr[l + 1] - e->bwd_ptr[l], bmap, st);
    e->launches += 2 * (int64_t)S.nlevels;
    return FCW_OK;
}

// Poisson solve: right-hand sides R, solution into Y (both n x K, elimination order).
template <typename T>
int poisson_solve(fcw_engine* e, const T* val, const T* inv, const T* R, T* Y, int32_t K, cudaStream_t st) {
    fcw::SolveArgs<T> a = solve_args<T>(e, val, inv, Y, K);
    a.R = R;
    if constexpr (sizeof(T) == 4) {
        if (e->core_hi && K % fcw::kTcCols == 0) return sweep_tc(e, a, st);
    }
    sweep<T>(e, a, st, FCW_STAGE_POISSON_FWD, FCW_STAGE_POISSON_BWD);
    return FCW_OK;
}

// Distances for the K sources in ws.src, shifted, source-major in ws.dT64 / ws.dT32.
// With metric arguments, the shift also produces the health/MSD partials and near lists.
int distances_block(fcw_engine* e, int32_t K, int precision, cudaStream_t st, const fcw::MetricArgs* ma = nullptr) {
    Workspace& w = e->cw();
    const int32_t n = (int32_t)e->sym.n;
    heat_solve(e, K, st);
    mark(e, st, FCW_STAGE_DIVERGENCE);
    if (precision == FCW_PREC_MIXED) {
        float* Y = reinterpret_cast<float*>(w.Y);
        fcw::launch_divergence_mixed(e->fd, w.Bh, w.Bp32, K, e->grounded_d, st);
        FCW_TRY(poisson_solve<float>(e, e->val_g, e->inv_g, w.Bp32, Y, K, st));
        // refinement: residual in FP64 and its FP32 solution, in the shift's output buffer
        // (two n x K float halves of dT64) before the shift writes it
        for (int32_t it = 0; it < e->prm.refine && e->lg.rp; ++it) {
            float* r = w.dT32;
            float* d = w.dT32 + (int64_t)n * K;
            fcw::launch_residual(e->lg, K, w.Bp32, Y, r, st);
            FCW_TRY(poisson_solve<float>(e, e->val_g, e->inv_g, r, d, K, st));
            fcw::launch_add((int64_t)n * K, Y, d, e->num_sms, st);
            e->launches += 2;
        }
        if (e->ncomp > 1) {
            fcw::launch_component_level(e->clevel, K, w.src, Y, w.csum, st);
            e->launches += 3;
        }
        mark(e, st, FCW_STAGE_SHIFT);
        if (ma) fcw::launch_shift_stats<float, float>(*ma, K, Y, w.dT32, st);
        else fcw::launch_shift_transpose<float, float>(n, K, Y, w.src, w.dT32, st);
    } else {
        fcw::launch_divergence_fp64(e->fd, w.Bh, w.Bp64, K, st);
        FCW_TRY(poisson_solve<double>(e, e->val_p, e->inv_p, w.Bp64, w.Y, K, st));
        mark(e, st, FCW_STAGE_SHIFT);
        if (ma) fcw::launch_shift_stats<double, double>(*ma, K, w.Y, w.dT64, st);
        else fcw::launch_shift_transpose<double, double>(n, K, w.Y, w.src, w.dT64, st);
    }
    e->launches += 2;
    return FCW_OK;
}

int metric_args(fcw_engine* e, const double* targets, int32_t nt, int32_t nb, double eps, int32_t nsrc,
                fcw::MetricArgs& a) {
    if (nt < 1 || nt > fcw::kMaxTargets) return fail(FCW_E_INVALID, "n_targets must be in [1, 32]");
    if (nb < 0 || nb > fcw::kMaxBetween) return fail(FCW_E_INVALID, "n_between must be in [0, 8]");
    if (!targets) return fail(FCW_E_INVALID, "targets is NULL");
    for (int32_t i = 0; i + 1 < nt; ++i)
        if (!(targets[i] <= targets[i + 1])) return fail(FCW_E_INVALID, "targets must be sorted ascending");
    a = fcw::MetricArgs{};
    a.n = (int32_t)e->sym.n;
    a.nf = (int32_t)e->mesh.nf;
    a.nsrc = nsrc;
    a.stride = fcw_metrics_stride(nt, nb);
    a.n_targets = nt;
    a.n_between = nb;
    a.n_boundary = (int32_t)e->mesh.boundary.size();
    a.coords = e->coords_d;
    a.vertex_area = e->varea_d;
    a.boundary = e->boundary_d;
    a.fv = e->fd.fv;
    a.inc_ptr = e->fd.inc_ptr;
    a.inc_face = e->fd.inc_face;
    a.inc_corner = e->fd.inc_corner;
    a.inc_rec = e->inc_rec_d;
    a.farea_fx = e->farea_fx_d;
    a.area_unscale = e->area_unscale;
    a.total_area = e->lean_total;
    a.farea = e->farea_d;
    a.g11 = e->g11_d;
    a.g12 = e->g12_d;
    a.g22 = e->g22_d;
    a.width = e->mesh.bin_width;
    a.health_h = e->mesh.health_h;
    a.eps = eps;
    a.rtol = 1e-10;
    a.max_iter = 60;
    for (int32_t i = 0; i < nt; ++i) a.targets[i] = targets[i];
    for (int32_t j = 0; j < nb; ++j) a.fracs[j] = (double)(j + 1) / ((double)nb + 1.0);
    a.K = nsrc;
    a.ntiles = (int32_t)((e->sym.n + fcw::kStatVTile - 1) / fcw::kStatVTile);
    a.partials = e->cw().partials;
    a.near_list = e->cw().near_list;
    a.near_count = e->cw().near_count;
    {
        // near radius: a flat disc holding twice the largest reachable target, in whole bins.
        // A source first tries the cut of a flat disc holding the target itself plus four
        // bins (enough for most fields: the radius is two bins below the cut), then the
        // near radius, both from the near list.
        double tmax = 0.0;
        for (int32_t i = 0; i < nt; ++i)
            if (targets[i] > tmax && targets[i] <= e->lean_total) tmax = targets[i];
        const double pi = 3.141592653589793;
        a.near_bins = (int32_t)std::ceil(std::sqrt(2.0 * tmax / pi) / e->mesh.bin_width) + 2;
        a.near_radius = (double)a.near_bins * e->mesh.bin_width;
        a.first_bins = std::min(a.near_bins, (int32_t)std::ceil(std::sqrt(tmax / pi) / e->mesh.bin_width) + 4);
    }
    a.src = e->cw().src;
    a.band = e->cw().band;
    a.longf = e->cw().longf;
    a.out = e->cw().out;
    a.err = e->err_d;
    return FCW_OK;
}

template <typename T>
void metrics_block(fcw_engine* e, fcw::MetricArgs& a, const T* dT, cudaStream_t st) {
    mark(e, st, FCW_STAGE_METRICS);
    fcw::launch_source_metrics<T>(a, dT, st);
    mark(e, st, -1);
    e->launches += 1;
}

int check_engine(fcw_engine* e) {
    if (!e) return fail(FCW_E_INVALID, "engine is NULL");
    cudaError_t ce = cudaSetDevice(e->device);
    if (ce != cudaSuccess) return fail(FCW_E_CUDA, cudaGetErrorString(ce));
    return FCW_OK;
}

int map_sources_host(fcw_engine* e, const int32_t* sources, int64_t n, int32_t K, cudaStream_t st,
                     std::vector<int32_t>& buf) {
    buf.assign(K, -1);
    for (int64_t k = 0; k < n; ++k) {
        const int32_t s = sources[k];
        if (s < 0 || s >= e->sym.n)
            return fail(FCW_E_INVALID, "source_idx out of range: " + std::to_string(s) + " for mesh with " +
                                           std::to_string(e->sym.n) + " vertices");
        buf[k] = e->sym.iperm[s];
    }
    FCW_CUDA(cudaMemcpyAsync(e->cw().src, buf.data(), K * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    return FCW_OK;
}

int32_t round_k(int64_t k) { return (int32_t)(((k + fcw::kRhsTile - 1) / fcw::kRhsTile) * fcw::kRhsTile); }

}  // namespace

namespace {

// Run `launch` (a chain of launches on w.stream) captured as a CUDA graph, once per
// workspace and key, and replayed after that; directly while graphs are off, the stage
// timeline is on, or the stream is already being captured by the caller.
template <class F>
int run_chain(fcw_engine* e, Workspace& w, const std::vector<double>& key, F&& launch) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    FCW_CUDA(cudaStreamIsCapturing(w.stream, &cs));
    if (!e->graphs_on || e->prof_on || cs != cudaStreamCaptureStatusNone) return launch();
    Workspace::Graph* hit = nullptr;
    for (auto& g : w.graphs)
        if (g.key == key) hit = &g;
    if (!hit) {
        constexpr size_t kMaxGraphs = 4;  // e.g. a full block and a call's last, partial one
        if (w.graphs.size() >= kMaxGraphs) {
            cudaGraphExecDestroy(w.graphs.front().exec);
            w.graphs.erase(w.graphs.begin());
        }
        const int64_t l0 = e->launches;
        FCW_CUDA(cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal));
        const int lrc = launch();
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaError_t ce = cudaStreamEndCapture(w.stream, &g);
        if (lrc != FCW_OK) {
            if (g) cudaGraphDestroy(g);
            e->launches = l0;
            return lrc;
        }
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, g, 0);
        if (g) cudaGraphDestroy(g);
        const int64_t captured = e->launches - l0;  // kernels in the chain (counted when it runs)
        e->launches = l0;
        if (ce != cudaSuccess) {  // not capturable here: launch directly from now on
            cudaGetLastError();
            e->graphs_on = false;
            return launch();
        }
        w.graphs.push_back({key, exec, captured});
        hit = &w.graphs.back();
    }
    FCW_CUDA(cudaGraphLaunch(hit->exec, w.stream));
    e->launches += hit->launches;
    return FCW_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void fcw_default_params(fcw_params* p) {
    if (!p) return;
    p->diffusion_length_mm = 0.7;
    p->poisson_shift = 1e-10;
    p->block_k = 1024;
    p->leaf_size = 64;
    p->max_width = 64;
    p->relax = 64;
    p->build_mixed = 1;
    p->device = 0;
    p->pipeline_depth = 4;
    p->tc_sweeps = 0;
    p->robust = 0;
    p->refine = 0;
}

int fcw_metrics_stride(int32_t n_targets, int32_t n_between) {
    if (n_targets < 0 || n_between < 0) return 0;
    const int32_t ne = n_targets > 0 ? (n_targets - 1) * n_between : 0;
    return FCW_M_RADII + 2 * n_targets + 2 * ne;
}

int fcw_last_error(char* buf, size_t len) {
    if (buf && len) {
        std::strncpy(buf, g_err.c_str(), len - 1);
        buf[len - 1] = '\0';
    }
    return (int)g_err.size();
}

int fcw_mesh_arrays(const double* V, int64_t nv, const int32_t* F, int64_t nf, double* vertex_area,
                    double* lean_area, double* g11, double* g12, double* g22, uint8_t* boundary_flag) {
    if (!V || !F) return fail(FCW_E_INVALID, "vertices/faces is NULL");
    fcw::MeshPrep m;
    std::string err;
    if (fcw::prepare_mesh(V, nv, F, nf, m, err)) return fail(FCW_E_INVALID, err);
    if (vertex_area) std::memcpy(vertex_area, m.vertex_area.data(), nv * sizeof(double));
    if (lean_area) std::memcpy(lean_area, m.lean_area.data(), nf * sizeof(double));
    if (g11) std::memcpy(g11, m.g11.data(), nf * sizeof(double));
    if (g12) std::memcpy(g12, m.g12.data(), nf * sizeof(double));
    if (g22) std::memcpy(g22, m.g22.data(), nf * sizeof(double));
    if (boundary_flag) {
        std::memset(boundary_flag, 0, nv);
        for (int32_t b : m.boundary) boundary_flag[b] = 1;
    }
    return FCW_OK;
}

int fcw_analyze(const double* V, int64_t nv, const int32_t* F, int64_t nf, const fcw_params* params,
                fcw_info* info, int32_t* perm_out) {
    if (!V || !F) return fail(FCW_E_INVALID, "vertices/faces is NULL");
    FCW_TRY(validate_params(params));
    fcw::MeshPrep m;
    fcw::Symbolic S;
    std::string err;
    double t0 = now_ms();
    if (fcw::prepare_mesh(V, nv, F, nf, m, err)) return fail(FCW_E_INVALID, err);
    int64_t nflips = 0;
    if (params->robust && fcw::intrinsic_delaunay(m, kMollifyFactor, nflips, err)) return fail(FCW_E_INVALID, err);
    if (fcw::build_symbolic(m, params->leaf_size, params->max_width, params->relax, S, err)) return fail(FCW_E_INVALID, err);
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->n_vertices = nv;
        info->n_faces = nf;
        info->n_boundary = (int64_t)m.boundary.size();
        info->n_supernodes = S.nsuper;
        info->n_levels = S.nlevels;
        info->nnz_factor = S.nnz_factor;
        info->nnz_l = S.nnz_l;
        info->max_ns = S.max_ns;
        info->max_m = S.max_m;
        info->mean_edge_length = m.mean_edge;
        info->t_coef = std::pow(params->diffusion_length_mm / m.mean_edge, 2.0);
        info->t = info->t_coef * m.mean_edge * m.mean_edge;
        info->bin_width = m.bin_width;
        info->health_h = m.health_h;
        info->total_vertex_area = m.total_area;
        info->analyze_ms = now_ms() - t0;
        info->flops_factor = S.flops_factor;
        info->n_flips = nflips;
        std::vector<int32_t> comp;
        info->n_components = mesh_components(m, S.perm, comp);
    }
    if (perm_out) std::memcpy(perm_out, S.perm.data(), nv * sizeof(int32_t));
    return FCW_OK;
}

int fcw_intrinsic_operators(const double* V, int64_t nv, const int32_t* F, int64_t nf, int64_t* nflips, int64_t* nnz,
                            int64_t* Lp, int32_t* Li, double* Lx, double* mass, int32_t* tri, double* len,
                            int32_t* twin) {
    if (!V || !F) return fail(FCW_E_INVALID, "vertices/faces is NULL");
    fcw::MeshPrep m;
    std::string err;
    if (fcw::prepare_mesh(V, nv, F, nf, m, err)) return fail(FCW_E_INVALID, err);
    int64_t nfl = 0;
    if (fcw::intrinsic_delaunay(m, kMollifyFactor, nfl, err)) return fail(FCW_E_INVALID, err);
    if (nflips) *nflips = nfl;
    if (nnz) *nnz = (int64_t)m.Li.size();
    if (Lp) std::memcpy(Lp, m.Lp.data(), (nv + 1) * sizeof(int64_t));
    if (Li) std::memcpy(Li, m.Li.data(), m.Li.size() * sizeof(int32_t));
    if (Lx) std::memcpy(Lx, m.Lx.data(), m.Lx.size() * sizeof(double));
    if (mass) std::memcpy(mass, m.mass.data(), nv * sizeof(double));
    if (nfl > 0) {
        if (tri) std::memcpy(tri, m.itri.data(), m.itri.size() * sizeof(int32_t));
        if (len) std::memcpy(len, m.ilen.data(), m.ilen.size() * sizeof(double));
        if (twin) std::memcpy(twin, m.itwin.data(), m.itwin.size() * sizeof(int32_t));
    }
    return FCW_OK;
}

int fcw_engine_create(const double* V, int64_t nv, const int32_t* F, int64_t nf, const fcw_params* params,
                      fcw_engine** out) {
    if (!out) return fail(FCW_E_INVALID, "out is NULL");
    *out = nullptr;
    if (!V || !F) return fail(FCW_E_INVALID, "vertices/faces is NULL");
    FCW_TRY(validate_params(params));
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(FCW_E_NODEVICE, std::string("no CUDA device available: ") + cudaGetErrorString(ce));
    }
    if (params->device < 0 || params->device >= ndev) return fail(FCW_E_INVALID, "invalid device ordinal");
    fcw_engine* e = new fcw_engine();
    e->prm = *params;
    e->device = params->device;
    int rc = build_engine(e, V, nv, F, nf);
    if (rc == FCW_OK) rc = ensure_workspace(e, params->block_k, fcw_metrics_stride(12, 3));
    if (rc != FCW_OK) {
        std::string msg = g_err;
        delete e;
        g_err = msg;
        return rc;
    }
    *out = e;
    return FCW_OK;
}

int fcw_engine_info(const fcw_engine* e, fcw_info* info) {
    if (!e || !info) return fail(FCW_E_INVALID, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    const auto& S = e->sym;
    const auto& m = e->mesh;
    info->n_vertices = m.nv;
    info->n_faces = m.nf;
    info->n_boundary = (int64_t)m.boundary.size();
    info->n_supernodes = S.nsuper;
    info->n_levels = S.nlevels;
    info->nnz_factor = S.nnz_factor;
    info->nnz_l = S.nnz_l;
    info->max_ns = S.max_ns;
    info->max_m = S.max_m;
    info->mean_edge_length = m.mean_edge;
    info->t_coef = e->t_coef;
    info->t = e->t;
    info->bin_width = m.bin_width;
    info->health_h = m.health_h;
    info->total_vertex_area = m.total_area;
    info->analyze_ms = e->analyze_ms;
    info->factor_ms = e->factor_ms;
    info->flops_factor = S.flops_factor;
    info->device_bytes = e->bytes;
    info->pipeline_depth = (int32_t)e->pool.size();
    info->block_k = e->prm.block_k;
    info->n_flips = e->n_flips;
    info->n_components = e->ncomp;
    return FCW_OK;
}

int fcw_engine_destroy(fcw_engine* e) {
    if (!e) return FCW_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    delete e;
    return FCW_OK;
}

int fcw_compute_distances(fcw_engine* e, const int32_t* sources, int64_t n, int32_t precision, double* out_host) {
    FCW_TRY(check_engine(e));
    if (n < 0 || (n > 0 && (!sources || !out_host))) return fail(FCW_E_INVALID, "NULL argument");
    if (precision == FCW_PREC_MIXED && !e->val_g) return fail(FCW_E_INVALID, "engine was built without the mixed form");
    const int32_t Kmax = e->prm.block_k;
    const int64_t nv = e->sym.n;
    std::vector<int32_t> buf;
    for (int64_t b0 = 0; b0 < n; b0 += Kmax) {
        const int64_t nb = std::min<int64_t>(Kmax, n - b0);
        const int32_t K = round_k(nb);
        FCW_TRY(ensure_workspace(e, K, e->cw().out_stride));
        if (e->hcap_dist < nb * nv) {
            if (e->hdist_d) e->release(e->hdist_d);
            e->hdist_d = nullptr;
            FCW_TRY(e->dalloc(&e->hdist_d, (size_t)(nb * nv)));
            e->hcap_dist = nb * nv;
        }
        Workspace& w = e->cw();
        FCW_TRY(map_sources_host(e, sources + b0, nb, K, w.stream, buf));
        // the chain (solves, divergence, shift, fields back to the caller's order) as one graph
        const std::vector<double> key = {(double)K, (double)precision, -1.0, (double)nb};
        FCW_TRY(run_chain(e, w, key, [&]() -> int {
            FCW_TRY(distances_block(e, K, precision, w.stream));
            const int grid = e->num_sms * 8;
            if (precision == FCW_PREC_MIXED)
                k_fields_out<float><<<grid, 256, 0, w.stream>>>((int32_t)nv, (int32_t)nb, w.dT32, e->iperm_d, e->hdist_d);
            else
                k_fields_out<double><<<grid, 256, 0, w.stream>>>((int32_t)nv, (int32_t)nb, w.dT64, e->iperm_d, e->hdist_d);
            e->launches += 1;
            return FCW_OK;
        }));
        FCW_CUDA(cudaGetLastError());
        FCW_CUDA(cudaMemcpyAsync(out_host + b0 * nv, e->hdist_d, (size_t)(nb * nv) * sizeof(double),
                                 cudaMemcpyDeviceToHost, w.stream));
        FCW_CUDA(cudaStreamSynchronize(w.stream));
        FCW_TRY(check_kernel_errors(e, "distances"));
    }
    return FCW_OK;
}

namespace {

// The drop-in's chain on st: the source's path, heat forward (the path's tasks) and
// backward, divergence, Poisson forward and backward, shift into the caller's order.
// Every sweep is one persistent ticketed launch. The source index is read from nar.src.
int narrow_chain(fcw_engine* e, cudaStream_t st) {
    NarrowState& q = e->nar;
    const int64_t n = e->sym.n;
    const int64_t nu = std::max<int64_t>(e->n_urows, 1);
    double* U_h = q.pend;
    double* U_p = q.pend + nu;
    double* X_h = q.pend + 2 * nu;
    double* X_p = X_h + n;
    FCW_CUDA(cudaMemsetAsync(q.sync, 0, 4 * sizeof(int), st));
    FCW_CUDA(cudaMemsetAsync(q.pend, 0xFF, (size_t)(2 * nu + 2 * n) * sizeof(double), st));  // pending
    FCW_CUDA(cudaMemsetAsync(q.u, 0, (size_t)n * sizeof(double), st));
    fcw::NarrowArgs a;
    a.p = e->plan;
    a.at_ptr = q.at_ptr;
    a.uoff = e->uoff_d;
    a.gm_ptr = e->gm_ptr_d;
    a.gm_src = e->gm_src_d;
    a.gm_child = e->gm_child_d;
    a.iperm = e->iperm_d;
    a.err = e->err_d;
    // heat: the path's forward tasks, then the whole backward
    mark(e, st, FCW_STAGE_HEAT_FWD);
    a.at = q.at_h;
    a.B = q.u;
    a.U = U_h;
    a.tasks = q.ftasks;
    a.ntasks = q.n_ftasks;
    a.order = q.order;
    a.ticket = q.sync;
    fcw::launch_fwd_narrow(a, true, false, q.L, st);
    mark(e, st, FCW_STAGE_HEAT_BWD);
    a.at = q.atb_h;
    a.tasks = q.btasks;
    a.ntasks = q.n_btasks;
    a.X = X_h;
    a.ticket = q.sync + 1;
    fcw::launch_bwd_narrow(a, !e->prof_on, q.L, st);
    mark(e, st, FCW_STAGE_DIVERGENCE);
    fcw::launch_divergence_fp64_one(e->fd, X_h, q.div, st);
    // Poisson (L + shift M)
    mark(e, st, FCW_STAGE_POISSON_FWD);
    a.at = q.at_p;
    a.R = q.div;
    a.B = q.y;
    a.U = U_p;
    a.tasks = q.ftasks;
    a.ntasks = q.n_ftasks;
    a.order = nullptr;
    a.ticket = q.sync + 2;
    fcw::launch_fwd_narrow(a, false, !e->prof_on, q.L, st);
    mark(e, st, FCW_STAGE_POISSON_BWD);
    a.at = q.atb_p;
    a.tasks = q.btasks;
    a.ntasks = q.n_btasks;
    a.X = X_p;
    a.ticket = q.sync + 3;
    fcw::launch_bwd_narrow(a, !e->prof_on, q.L, st);
    mark(e, st, FCW_STAGE_SHIFT);
    fcw::launch_field_out_one((int32_t)n, X_p, q.order, e->iperm_d, q.out, e->num_sms, st);
    mark(e, st, -1);
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}

int narrow_ready(fcw_engine* e) {
    NarrowState& q = e->nar;
    if (q.ready) return FCW_OK;
    const auto& S = e->sym;
    const int32_t NS = S.nsuper;
    const int64_t n = S.n;
    if (fcw::configure_narrow_kernels(S.max_m, e->num_sms, &q.L) != cudaSuccess) {
        cudaGetLastError();
        return fail(FCW_E_INVALID, "front too large for the single-source kernels (max_m " + std::to_string(S.max_m) +
                                       ")");
    }
    std::vector<int64_t> ptr((size_t)NS + 1);
    const int64_t total = fcw::narrow_layout(S.sn_c0.data(), S.sn_m.data(), NS, ptr.data());
    std::vector<int4> ft, bt;
    std::vector<int32_t> fptr, nf, nb;
    fcw::narrow_tasks(S.sn_c0.data(), S.sn_m.data(), NS, S.level_nodes.data(), ft, fptr, nf, bt, nb);
    q.n_ftasks = (int32_t)ft.size();
    q.n_btasks = (int32_t)bt.size();
    FCW_TRY(e->upload(&q.at_ptr, ptr));
    FCW_TRY(e->upload(&q.ftasks, ft));
    FCW_TRY(e->upload(&q.btasks, bt));
    q.fwd_first = fptr;
    q.nfwd_h = nf;
    for (double** arr : {&q.at_h, &q.at_p, &q.atb_h, &q.atb_p}) {
        FCW_TRY(e->dalloc(arr, (size_t)total));
        FCW_CUDA(cudaMemsetAsync(*arr, 0, (size_t)total * sizeof(double), e->stream));
    }
    fcw::launch_build_narrow(e->plan, e->val_h, e->inv_h, q.at_ptr, q.at_h, q.atb_h, e->stream);
    fcw::launch_build_narrow(e->plan, e->val_p, e->inv_p, q.at_ptr, q.at_p, q.atb_p, e->stream);
    FCW_CUDA(cudaGetLastError());
    FCW_TRY(e->dalloc(&q.u, (size_t)n));
    FCW_TRY(e->dalloc(&q.div, (size_t)n));
    FCW_TRY(e->dalloc(&q.y, (size_t)n));
    FCW_TRY(e->dalloc(&q.out, (size_t)n));
    FCW_TRY(e->dalloc(&q.pend, (size_t)(2 * std::max<int64_t>(e->n_urows, 1) + 2 * n)));
    FCW_TRY(e->dalloc(&q.sync, 4));
    const size_t cap = 2 + 2 * (size_t)q.n_ftasks;
    FCW_TRY(e->dalloc(&q.order, cap));
    FCW_CUDA(cudaHostAlloc(&q.horder, cap * sizeof(int32_t), cudaHostAllocDefault));
    FCW_CUDA(cudaStreamSynchronize(e->stream));
    q.launches = 6;
    if (e->graphs_on) {
        FCW_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        const int lrc = narrow_chain(e, e->stream);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (lrc != FCW_OK) {
            if (g) cudaGraphDestroy(g);
            return lrc;
        }
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&q.exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (ce != cudaSuccess) {  // not capturable here: the chain launches directly
            cudaGetLastError();
            q.exec = nullptr;
        }
    }
    q.ready = true;
    return FCW_OK;
}

// The drop-in chain for one source (in range) on e->stream: its path's task list to the
// device, then the chain (the captured graph, or direct launches).
int narrow_run(fcw_engine* e, int32_t source) {
    FCW_TRY(narrow_ready(e));
    NarrowState& q = e->nar;
    cudaStream_t st = e->stream;
    // the source's path to the root, bottom-up, with each supernode's forward tasks
    const auto& S = e->sym;
    int32_t* o = q.horder;
    int32_t len = 0, prev = -1;
    o[0] = S.iperm[source];
    for (int32_t s = S.col_sn[o[0]]; s >= 0; prev = s, s = S.sn_parent[s])
        for (int32_t t = q.fwd_first[s]; t < q.fwd_first[s] + q.nfwd_h[s]; ++t) {
            o[2 + 2 * len] = t;
            o[3 + 2 * len] = prev;
            ++len;
        }
    o[1] = len;
    FCW_CUDA(cudaMemcpyAsync(q.order, o, (size_t)(2 + 2 * len) * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    if (q.exec && e->graphs_on && !e->prof_on) FCW_CUDA(cudaGraphLaunch(q.exec, st));
    else FCW_TRY(narrow_chain(e, st));
    e->launches += q.launches;
    return FCW_OK;
}

// fcw_compute_metrics for one source in FP64: the drop-in chain, then the statistics and
// the per-source kernel at one column (records identical in meaning to the batched path's).
int narrow_metrics(fcw_engine* e, int32_t source, const double* targets, int32_t nt, int32_t nb, double eps,
                   double* out_host) {
    e->sync_streams();  // the workspace's metric scratch may still be in use by a device-API call
    const int32_t stride = fcw_metrics_stride(nt, nb);
    FCW_TRY(ensure_workspace(e, fcw::kRhsTile, stride));
    fcw::MetricArgs a;
    FCW_TRY(metric_args(e, targets, nt, nb, eps, 1, a));
    FCW_TRY(narrow_run(e, source));
    NarrowState& q = e->nar;
    cudaStream_t st = e->stream;
    const int64_t n = e->sym.n, nu = std::max<int64_t>(e->n_urows, 1);
    const double* X_p = q.pend + 2 * nu + n;  // the Poisson solution (elimination order)
    a.src = q.order;                           // its first entry: the source's elimination index
    fcw::launch_shift_stats_one(a, X_p, e->cw().dT64, st);
    fcw::launch_source_metrics<double>(a, e->cw().dT64, st);
    e->launches += 2;
    FCW_CUDA(cudaGetLastError());
    FCW_CUDA(cudaMemcpyAsync(out_host, a.out, (size_t)stride * sizeof(double), cudaMemcpyDeviceToHost, st));
    FCW_CUDA(cudaStreamSynchronize(st));
    return check_kernel_errors(e, "metrics");
}

}  // namespace

int fcw_compute_distance(fcw_engine* e, int32_t source, double* out_host) {
    FCW_TRY(check_engine(e));
    if (!out_host) return fail(FCW_E_INVALID, "NULL argument");
    if (source < 0 || source >= e->sym.n)
        return fail(FCW_E_INVALID, "source_idx out of range: " + std::to_string(source) + " for mesh with " +
                                       std::to_string(e->sym.n) + " vertices");
    FCW_TRY(narrow_run(e, source));
    NarrowState& q = e->nar;
    cudaStream_t st = e->stream;
    FCW_CUDA(cudaMemcpyAsync(out_host, q.out, (size_t)e->sym.n * sizeof(double), cudaMemcpyDeviceToHost, st));
    FCW_CUDA(cudaStreamSynchronize(st));
    return check_kernel_errors(e, "distance");
}

namespace {

// One block's launch chain on workspace w, its inputs in w.desc: source mapping,
// distances, metrics. With graphs on (and the stage timeline off) the chain is
// captured once per workspace and set of arguments, and replayed for later blocks.
int block_chain(fcw_engine* e, Workspace& w, int32_t K, int32_t precision, fcw::MetricArgs& a,
                const double* targets, int32_t nt, int32_t nb, double eps) {
    auto launch = [&]() -> int {
        k_map_block_sources<<<(K + 127) / 128, 128, 0, w.stream>>>(w.desc, e->iperm_d, (int32_t)e->sym.n, K, w.src,
                                                                   e->err_d);
        e->launches += 1;
        const int rc = distances_block(e, K, precision, w.stream, &a);
        if (rc != FCW_OK) return rc;
        if (precision == FCW_PREC_MIXED) metrics_block<float>(e, a, w.dT32, w.stream);
        else metrics_block<double>(e, a, w.dT64, w.stream);
        return FCW_OK;
    };
    std::vector<double> key = {(double)K, (double)precision, (double)nt, (double)nb, eps};
    key.insert(key.end(), targets, targets + nt);
    return run_chain(e, w, key, launch);
}

}  // namespace

int fcw_compute_metrics_device(fcw_engine* e, const int32_t* sources_dev, int64_t n, int32_t precision,
                               const double* targets, int32_t nt, int32_t nb, double eps, double* out_dev,
                               void* stream) {
    FCW_TRY(check_engine(e));
    if (n < 0 || (n > 0 && (!sources_dev || !out_dev))) return fail(FCW_E_INVALID, "NULL argument");
    if (precision == FCW_PREC_MIXED && !e->val_g) return fail(FCW_E_INVALID, "engine was built without the mixed form");
    if (n == 0) return FCW_OK;
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    const int32_t stride = fcw_metrics_stride(nt, nb);
    const int32_t Kmax = e->prm.block_k;
    FCW_TRY(ensure_workspace(e, std::min<int64_t>(round_k(n), Kmax), stride));
    // Blocks of K sources round-robin over the workspace pool, each workspace on its own
    // stream, so independent blocks overlap. The pool streams start after the caller's
    // stream reaches this call, and the caller's stream waits for all of them at the end.
    const size_t depth = e->pool.size();
    FCW_CUDA(cudaEventRecord(e->ev_in, user));
    size_t used = 0;
    int rc = FCW_OK;
    for (int64_t b0 = 0, blk = 0; b0 < n && rc == FCW_OK; b0 += Kmax, ++blk) {
        const int64_t nbk = std::min<int64_t>(Kmax, n - b0);
        const int32_t K = round_k(nbk);
        e->cur_ws = (size_t)blk % depth;
        Workspace& w = e->cw();
        if (blk < (int64_t)depth) {
            FCW_CUDA(cudaStreamWaitEvent(w.stream, e->ev_in, 0));
            used = (size_t)blk + 1;
        }
        fcw::MetricArgs a;
        rc = metric_args(e, targets, nt, nb, eps, K, a);
        if (rc != FCW_OK) break;
        a.desc = w.desc;
        k_set_block<<<1, 1, 0, w.stream>>>(w.desc, sources_dev + b0, nbk, out_dev + b0 * stride);
        e->launches += 1;
        rc = block_chain(e, w, K, precision, a, targets, nt, nb, eps);
    }
    for (size_t i = 0; i < used; ++i) {
        FCW_CUDA(cudaEventRecord(e->pool[i].done, e->pool[i].stream));
        FCW_CUDA(cudaStreamWaitEvent(user, e->pool[i].done, 0));
    }
    e->cur_ws = 0;
    if (rc != FCW_OK) return rc;
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}

int fcw_compute_metrics(fcw_engine* e, const int32_t* sources, int64_t n, int32_t precision, const double* targets,
                        int32_t nt, int32_t nb, double eps, double* out_host) {
    FCW_TRY(check_engine(e));
    if (n < 0 || (n > 0 && (!sources || !out_host))) return fail(FCW_E_INVALID, "NULL argument");
    if (n == 0) return FCW_OK;
    for (int64_t k = 0; k < n; ++k)
        if (sources[k] < 0 || sources[k] >= e->sym.n)
            return fail(FCW_E_INVALID, "source_idx out of range: " + std::to_string(sources[k]) + " for mesh with " +
                                           std::to_string(e->sym.n) + " vertices");
    if (n == 1 && precision == FCW_PREC_FP64) return narrow_metrics(e, sources[0], targets, nt, nb, eps, out_host);
    const int32_t stride = fcw_metrics_stride(nt, nb);
    if (e->hcap_src < n) {
        if (e->hsrc_d) e->release(e->hsrc_d);
        e->hsrc_d = nullptr;
        FCW_TRY(e->dalloc(&e->hsrc_d, (size_t)n));
        e->hcap_src = n;
    }
    if (e->hcap_out < n * stride) {
        if (e->hout_d) e->release(e->hout_d);
        e->hout_d = nullptr;
        FCW_TRY(e->dalloc(&e->hout_d, (size_t)n * stride));
        e->hcap_out = n * stride;
    }
    FCW_CUDA(cudaMemcpyAsync(e->hsrc_d, sources, n * sizeof(int32_t), cudaMemcpyHostToDevice, e->stream));
    FCW_TRY(fcw_compute_metrics_device(e, e->hsrc_d, n, precision, targets, nt, nb, eps, e->hout_d, e->stream));
    FCW_CUDA(cudaMemcpyAsync(out_host, e->hout_d, n * stride * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    return check_kernel_errors(e, "metrics");
}

int fcw_samples_capacity(int32_t n_targets, int32_t n_between) {
    if (n_targets < 0 || n_between < 0) return 0;
    return n_targets + (n_targets > 0 ? (n_targets - 1) * n_between : 0);
}

namespace {

int sample_args(const double* records, int64_t n, int32_t nt, int32_t nb, const double* targets, double cap,
                float* radii, float* areas, int32_t* count, fcw::SampleArgs& a) {
    if (nt < 1 || nt > fcw::kMaxTargets) return fail(FCW_E_INVALID, "n_targets must be in [1, 32]");
    if (nb < 0 || nb > fcw::kMaxBetween) return fail(FCW_E_INVALID, "n_between must be in [0, 8]");
    if (!targets) return fail(FCW_E_INVALID, "targets is NULL");
    if (!std::isnan(cap) && !(cap >= 0.0 && cap < 0.5))
        return fail(FCW_E_INVALID, "boundary_cap must be in [0, 0.5), or NaN for no cap");
    if (n < 0 || (n > 0 && (!records || !radii || !areas || !count))) return fail(FCW_E_INVALID, "NULL argument");
    a = fcw::SampleArgs{};
    a.n = n;
    a.n_targets = nt;
    a.n_between = nb;
    a.stride = fcw_metrics_stride(nt, nb);
    a.capacity = fcw_samples_capacity(nt, nb);
    for (int32_t i = 0; i < nt; ++i) a.targets[i] = targets[i];
    a.cap = cap;
    a.records = records;
    a.radii_out = radii;
    a.areas_out = areas;
    a.count_out = count;
    return FCW_OK;
}

}  // namespace

int fcw_assemble_samples_device(const double* records_dev, int64_t n, int32_t n_targets, int32_t n_between,
                                const double* targets, double boundary_cap, float* radii_out, float* areas_out,
                                int32_t* count_out, void* stream) {
    fcw::SampleArgs a;
    FCW_TRY(sample_args(records_dev, n, n_targets, n_between, targets, boundary_cap, radii_out, areas_out, count_out,
                        a));
    if (n == 0) return FCW_OK;
    fcw::launch_assemble_samples(a, static_cast<cudaStream_t>(stream));
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}

int fcw_assemble_samples(fcw_engine* e, const double* records, int64_t n, int32_t n_targets, int32_t n_between,
                         const double* targets, double boundary_cap, float* radii, float* areas, int32_t* count) {
    FCW_TRY(check_engine(e));
    fcw::SampleArgs a;
    FCW_TRY(sample_args(records, n, n_targets, n_between, targets, boundary_cap, radii, areas, count, a));
    if (n == 0) return FCW_OK;
    const int64_t stride = a.stride, cap = a.capacity;
    if (e->hcap_out < n * stride) {
        if (e->hout_d) e->release(e->hout_d);
        e->hout_d = nullptr;
        FCW_TRY(e->dalloc(&e->hout_d, (size_t)(n * stride)));
        e->hcap_out = n * stride;
    }
    if (e->hcap_smp < n * cap) {
        if (e->hsr_d) e->release(e->hsr_d);
        if (e->hsa_d) e->release(e->hsa_d);
        e->hsr_d = e->hsa_d = nullptr;
        FCW_TRY(e->dalloc(&e->hsr_d, (size_t)(n * cap)));
        FCW_TRY(e->dalloc(&e->hsa_d, (size_t)(n * cap)));
        e->hcap_smp = n * cap;
    }
    if (e->hcap_cnt < n) {
        if (e->hcnt_d) e->release(e->hcnt_d);
        e->hcnt_d = nullptr;
        FCW_TRY(e->dalloc(&e->hcnt_d, (size_t)n));
        e->hcap_cnt = n;
    }
    FCW_CUDA(cudaMemcpyAsync(e->hout_d, records, n * stride * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    a.records = e->hout_d;
    a.radii_out = e->hsr_d;
    a.areas_out = e->hsa_d;
    a.count_out = e->hcnt_d;
    fcw::launch_assemble_samples(a, e->stream);
    FCW_CUDA(cudaGetLastError());
    FCW_CUDA(cudaMemcpyAsync(radii, e->hsr_d, n * cap * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    FCW_CUDA(cudaMemcpyAsync(areas, e->hsa_d, n * cap * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    FCW_CUDA(cudaMemcpyAsync(count, e->hcnt_d, n * sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream));
    FCW_CUDA(cudaStreamSynchronize(e->stream));
    return FCW_OK;
}

int fcw_engine_graphs(fcw_engine* e, int enable) {
    FCW_TRY(check_engine(e));
    e->graphs_on = enable != 0;
    return FCW_OK;
}

int fcw_engine_profile(fcw_engine* e, int enable) {
    FCW_TRY(check_engine(e));
    FCW_TRY(collect_marks(e));
    e->prof_on = enable != 0;
    for (double& x : e->stage_ms) x = 0.0;
    e->launches = 0;
    return FCW_OK;
}

int fcw_engine_stage_times(fcw_engine* e, double* ms_out, int32_t n, int64_t* launches) {
    FCW_TRY(check_engine(e));
    FCW_TRY(collect_marks(e));
    for (int32_t i = 0; i < n && i < FCW_N_STAGES; ++i) ms_out[i] = e->stage_ms[i];
    if (launches) *launches = e->launches;
    return FCW_OK;
}

int fcw_synchronize(fcw_engine* e, void* stream) {
    FCW_TRY(check_engine(e));
    FCW_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    return check_kernel_errors(e, "device call");
}

int fcw_heat_solve_device(fcw_engine* e, const int32_t* sources_dev, int32_t k, double* u_dev, void* stream) {
    FCW_TRY(check_engine(e));
    if (k <= 0 || !sources_dev || !u_dev) return fail(FCW_E_INVALID, "invalid arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int32_t K = round_k(k);
    FCW_TRY(ensure_workspace(e, K, e->cw().out_stride));
    k_map_sources<<<(K + 127) / 128, 128, 0, st>>>(k, sources_dev, e->iperm_d, (int32_t)e->sym.n, K, e->cw().src,
                                                   e->err_d);
    heat_solve(e, K, st);
    // u_dev[old][c] = Bh[iperm[old]][c]
    fcw::launch_permute_rows((int32_t)e->sym.n, k, e->cw().Bh, K, e->iperm_d, u_dev, k, nullptr, st);
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}

int fcw_divergence_device(fcw_engine* e, const double* u_dev, int32_t k, double* div_dev, void* stream) {
    FCW_TRY(check_engine(e));
    if (k <= 0 || !u_dev || !div_dev) return fail(FCW_E_INVALID, "invalid arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int32_t K = round_k(k);
    FCW_TRY(ensure_workspace(e, K, e->cw().out_stride));
    FCW_CUDA(cudaMemsetAsync(e->cw().Bh, 0, (size_t)e->sym.n * K * sizeof(double), st));
    fcw::launch_permute_rows((int32_t)e->sym.n, k, u_dev, k, nullptr, e->cw().Bh, K, e->iperm_d, st);
    fcw::launch_divergence_fp64(e->fd, e->cw().Bh, e->cw().Bp64, K, st);
    fcw::launch_permute_rows((int32_t)e->sym.n, k, e->cw().Bp64, K, e->iperm_d, div_dev, k, nullptr, st);
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}

int fcw_poisson_solve_device(fcw_engine* e, const double* div_dev, const int32_t* sources_dev, int32_t k,
                             double* phi_dev, void* stream) {
    FCW_TRY(check_engine(e));
    if (k <= 0 || !div_dev || !sources_dev || !phi_dev) return fail(FCW_E_INVALID, "invalid arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int32_t K = round_k(k);
    FCW_TRY(ensure_workspace(e, K, e->cw().out_stride));
    k_map_sources<<<(K + 127) / 128, 128, 0, st>>>(k, sources_dev, e->iperm_d, (int32_t)e->sym.n, K, e->cw().src,
                                                   e->err_d);
    FCW_CUDA(cudaMemsetAsync(e->cw().Bp64, 0, (size_t)e->sym.n * K * sizeof(double), st));
    fcw::launch_permute_rows((int32_t)e->sym.n, k, div_dev, k, nullptr, e->cw().Bp64, K, e->iperm_d, st);
    FCW_TRY(poisson_solve<double>(e, e->val_p, e->inv_p, e->cw().Bp64, e->cw().Y, K, st));
    fcw::launch_shift_transpose<double, double>((int32_t)e->sym.n, K, e->cw().Y, e->cw().src, e->cw().dT64, st);
    // phi_dev[old][c] = dT[c][iperm[old]]: transpose back through the permute kernel, column by column
    for (int32_t c = 0; c < k; ++c)
        fcw::launch_permute_rows((int32_t)e->sym.n, 1, e->cw().dT64 + (int64_t)c * e->sym.n, 1, e->iperm_d,
                                 phi_dev + c, k, nullptr, st);
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}

int fcw_field_metrics_device(fcw_engine* e, const double* d_dev, const int32_t* sources_dev, int32_t k,
                             const double* targets, int32_t nt, int32_t nb, double eps, double* out_dev,
                             void* stream) {
    FCW_TRY(check_engine(e));
    if (k <= 0 || !d_dev || !sources_dev || !out_dev) return fail(FCW_E_INVALID, "invalid arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int32_t K = round_k(k);
    const int32_t stride = fcw_metrics_stride(nt, nb);
    FCW_TRY(ensure_workspace(e, K, stride));
    fcw::MetricArgs a;
    FCW_TRY(metric_args(e, targets, nt, nb, eps, K, a));
    a.out = out_dev;
    k_map_sources<<<(K + 127) / 128, 128, 0, st>>>(k, sources_dev, e->iperm_d, (int32_t)e->sym.n, K, e->cw().src,
                                                   e->err_d);
    k_fields_in<<<e->num_sms * 8, 256, 0, st>>>((int32_t)e->sym.n, k, K, d_dev, e->iperm_d, e->cw().Y);
    mark(e, st, FCW_STAGE_SHIFT);
    fcw::launch_shift_stats<double, double>(a, K, e->cw().Y, e->cw().dT64, st);
    e->launches += 3;
    metrics_block<double>(e, a, e->cw().dT64, st);
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free field metrics
//
// For callers that may not allocate device memory once they are running: a host
// that reserves the whole device up front for its own pool, or a measurement or
// serving loop that must keep its device footprint fixed. This entry point runs
// the same kernels as fcw_field_metrics_device, but every buffer it needs beyond
// the caller's inputs and outputs (and the engine's own arrays, allocated when
// the engine was created) comes from one fixed array compiled into the library.
// ---------------------------------------------------------------------------
namespace {

// Per-call scratch for fcw_field_metrics_static. Every device that loads this
// library holds these bytes until the process exits.
constexpr size_t kStaticScratchBytes = 64u << 20;
constexpr int32_t kStaticMaxFields = 32;
static __device__ __align__(256) unsigned char g_field_scratch[kStaticScratchBytes];

// The array's device address, looked up once per device. In host code the name
// g_field_scratch only stands in for the symbol; it is not a device pointer.
constexpr int kMaxDevices = 64;
void* g_field_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_field_scratch_mutex;

int static_scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return fail(FCW_E_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_field_scratch_mutex);
    if (!g_field_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_field_scratch);  // the engine's device is current
        if (rc != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return fail(FCW_E_CUDA, std::string("cudaGetSymbolAddress(static field scratch) failed: ") +
                                        cudaGetErrorString(rc));
        }
        g_field_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_field_scratch_addr[device]);
    return FCW_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" int fcw_field_metrics_static(fcw_engine* e, const double* d_dev, const int32_t* sources_dev, int32_t k,
                                        const double* targets, int32_t nt, int32_t nb, double eps, double* out_dev,
                                        void* stream) {
    FCW_TRY(check_engine(e));
    if (k <= 0 || !d_dev || !sources_dev || !out_dev) return fail(FCW_E_INVALID, "invalid arguments");
    if (k > kStaticMaxFields)
        return fail(FCW_E_INVALID, "fcw_field_metrics_static takes at most " + std::to_string(kStaticMaxFields) +
                                       " fields per call, got " + std::to_string(k));
    const int32_t K = 32;  // one 32-column tile of the shift kernel; columns >= k are padding
    const int64_t n = e->sym.n, nf = e->mesh.nf;
    const int64_t ntiles = (n + fcw::kStatVTile - 1) / fcw::kStatVTile;
    const size_t need = align256((size_t)n * K * sizeof(double))          // vertex-major fields
                        + align256((size_t)n * K * sizeof(double))        // shifted, one field per row
                        + align256((size_t)ntiles * K * 8 * sizeof(double))  // health/MSD partials
                        + align256((size_t)n * K * sizeof(int32_t))       // near-vertex lists
                        + align256((size_t)K * sizeof(int32_t))           // near-vertex counts
                        + align256((size_t)nf * K * sizeof(int4))         // near faces by bin
                        + align256((size_t)nf * K * sizeof(int32_t))      // long faces
                        + align256((size_t)K * sizeof(int32_t));          // sources (elimination order)
    if (need > kStaticScratchBytes)
        return fail(FCW_E_INVALID, "mesh too large for fcw_field_metrics_static: needs " + std::to_string(need) +
                                       " bytes of scratch, the static array holds " +
                                       std::to_string(kStaticScratchBytes));
    unsigned char* base = nullptr;
    FCW_TRY(static_scratch_address(e->device, &base));
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += align256(bytes);
        return p;
    };
    double* Y = reinterpret_cast<double*>(take((size_t)n * K * sizeof(double)));
    double* dT = reinterpret_cast<double*>(take((size_t)n * K * sizeof(double)));
    double* partials = reinterpret_cast<double*>(take((size_t)ntiles * K * 8 * sizeof(double)));
    int32_t* near_list = reinterpret_cast<int32_t*>(take((size_t)n * K * sizeof(int32_t)));
    int32_t* near_count = reinterpret_cast<int32_t*>(take((size_t)K * sizeof(int32_t)));
    int4* band = reinterpret_cast<int4*>(take((size_t)nf * K * sizeof(int4)));
    int32_t* longf = reinterpret_cast<int32_t*>(take((size_t)nf * K * sizeof(int32_t)));
    int32_t* src = reinterpret_cast<int32_t*>(take((size_t)K * sizeof(int32_t)));

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fcw::MetricArgs a;
    FCW_TRY(metric_args(e, targets, nt, nb, eps, K, a));
    a.src = src;
    a.band = band;
    a.longf = longf;
    a.partials = partials;
    a.near_list = near_list;
    a.near_count = near_count;  // cleared by launch_shift_stats before the shift kernel
    a.out = out_dev;
    k_map_sources<<<1, 128, 0, st>>>(k, sources_dev, e->iperm_d, (int32_t)n, K, src, e->err_d);
    k_fields_in<<<e->num_sms * 8, 256, 0, st>>>((int32_t)n, k, K, d_dev, e->iperm_d, Y);
    mark(e, st, FCW_STAGE_SHIFT);
    fcw::launch_shift_stats<double, double>(a, K, Y, dT, st);
    e->launches += 3;
    mark(e, st, FCW_STAGE_METRICS);
    fcw::launch_source_metrics<double>(a, dT, st);
    mark(e, st, -1);
    e->launches += 1;
    FCW_CUDA(cudaGetLastError());
    return FCW_OK;
}
