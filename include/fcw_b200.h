/*
 * fcw_b200.h -- C ABI of the B200 heat-method distance engine.
 *
 * The engine replaces FastCorticalWiring's per-source hot path: one
 * heat-method distance field per cortical source vertex, followed by the
 * per-source metrics computed from it. All entry points return an int status
 * (FCW_OK on success); no exception or C++ type crosses the boundary.
 * fcw_last_error() returns the message of the last failure on the calling
 * thread. Vertex indices are 0-based indices into the cortical submesh the
 * engine was created with (the arrays core_analysis.py passes to its
 * distance engine).
 *
 * Threading: an engine handle is used by one host thread at a time. Calls
 * that take a stream enqueue work on it; the others synchronise before
 * returning.
 */
#ifndef FCW_B200_H
#define FCW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    FCW_OK = 0,
    FCW_E_INVALID = 1,    /* bad argument (message in fcw_last_error) */
    FCW_E_CUDA = 2,       /* CUDA runtime error */
    FCW_E_NOMEM = 3,      /* device allocation failed or HBM budget exceeded */
    FCW_E_NUMERIC = 4,    /* factorisation or kernel reported a numerical failure */
    FCW_E_TIMEOUT = 5,    /* a bounded wait expired */
    FCW_E_NODEVICE = 6    /* no CUDA device visible */
};

enum {
    FCW_PREC_FP64 = 0,    /* FP64 solves with the reference operators (the drop-in) */
    FCW_PREC_MIXED = 1    /* FP64 heat solve, FP32 grounded Poisson solve */
};

typedef struct fcw_params {
    double diffusion_length_mm; /* sqrt(t) in mm; >= 0.5 (distance_engines.py:82-89) */
    double poisson_shift;       /* Poisson regulariser: L + shift*M (fastcw_lean.py:481, 500) */
    int32_t block_k;            /* sources per right-hand-side block, a multiple of 64 */
    int32_t leaf_size;          /* nested-dissection leaf size */
    int32_t max_width;          /* widest supernode (columns), <= 64 */
    int32_t relax;              /* etree subtrees of at most this many columns become one supernode */
    int32_t build_mixed;        /* also factor the grounded FP32 Poisson operator */
    int32_t device;             /* CUDA device ordinal */
    int32_t pipeline_depth;     /* blocks in flight on separate streams in the device metrics path (1-8) */
    int32_t tc_sweeps;          /* mixed Poisson sweeps on the tensor cores (1) or FMA register tiles (0, default) */
    int32_t robust;             /* 1: operators of the intrinsic Delaunay triangulation (use_robust,
                                   distance_engines.py:119-125); 0 (default): the extrinsic cotan
                                   operators of fastcw_lean.py:394-413 */
    int32_t refine;             /* mixed form: iterative-refinement steps of the FP32 Poisson solve
                                   (0-4, default 0): each computes the residual of the grounded
                                   system in FP64 and adds the FP32 solution of it */
} fcw_params;

typedef struct fcw_info {
    int64_t n_vertices, n_faces, n_boundary;
    int64_t n_supernodes, n_levels, nnz_factor, nnz_l;
    int32_t max_ns, max_m;
    double mean_edge_length;    /* distance_engines.py:17-21 */
    double t_coef;              /* (diffusion_length / mean_edge)^2 (distance_engines.py:121-122) */
    double t;                   /* t_coef * mean_edge^2 (fastcw_lean.py:489) */
    double bin_width;           /* lean_geometry.py:99-114 */
    double health_h;            /* median face max edge (core_analysis.py:705) */
    double total_vertex_area;   /* sum of barycentric vertex areas */
    double analyze_ms, factor_ms, flops_factor;
    int64_t device_bytes;       /* device memory held by the engine */
    int32_t pipeline_depth;     /* blocks in flight the device holds workspaces for (<= params) */
    int32_t block_k;            /* sources per block */
    int64_t n_flips;            /* intrinsic edge flips (robust operators; 0 otherwise) */
    int64_t n_components;       /* connected components of the submesh (core_analysis.py:1349-1381) */
} fcw_info;

/* Per-source metric record: FCW_M_* offsets, then radii[nt], perimeters[nt],
 * extra_r[(nt-1)*nb], extra_a[(nt-1)*nb]; stride = fcw_metrics_stride(nt, nb). */
enum {
    FCW_M_MSD_U = 0,     /* core_analysis.py:1573-1578 */
    FCW_M_MSD_W = 1,     /* core_analysis.py:1579-1581 */
    FCW_M_DIST_B = 2,    /* core_analysis.py:1567-1572 */
    FCW_M_NEG = 3,       /* lean_geometry.py:343-357 negative fraction */
    FCW_M_VIOL = 4,      /* chord-violation fraction */
    FCW_M_BAD = 5,       /* 1.0 if the field fails the health screen */
    FCW_M_NEVAL = 6,     /* exact band evaluations used (lean_geometry.py:302-340) */
    FCW_M_RADII = 7
};

/* Pipeline stages timed by fcw_engine_profile / fcw_engine_stage_times. */
enum {
    FCW_STAGE_HEAT_FWD = 0,      /* reach + forward heat sweep (delta right-hand sides) */
    FCW_STAGE_HEAT_BWD = 1,      /* backward heat sweep */
    FCW_STAGE_DIVERGENCE = 2,    /* fused gradient -> normalise -> divergence */
    FCW_STAGE_POISSON_FWD = 3,
    FCW_STAGE_POISSON_BWD = 4,
    FCW_STAGE_SHIFT = 5,         /* phi -= phi[source], transpose to one field per source */
    FCW_STAGE_METRICS = 6,       /* health, MSD, distance to boundary, radius inversion, perimeter, samples */
    FCW_N_STAGES = 7
};

/* Fill *p with the defaults (0.7 mm, 1e-10, K=1024, leaf 64, width 64, relax 64, mixed on, 4 blocks in flight,
 * Poisson sweeps on FMA register tiles, extrinsic operators, no refinement). */
void fcw_default_params(fcw_params* p);

int fcw_metrics_stride(int32_t n_targets, int32_t n_between);

/* Message of the last failure on this thread; returns its length. */
int fcw_last_error(char* buf, size_t len);

/* Host-only symbolic analysis: mesh preparation, nested dissection, supernodes.
 * perm_out (nullable, n_vertices entries) receives the elimination order. */
int fcw_analyze(const double* vertices, int64_t n_vertices, const int32_t* faces, int64_t n_faces,
                const fcw_params* params, fcw_info* info, int32_t* perm_out);

/* Host-side per-mesh quantities in the caller's order (any pointer may be NULL):
 * vertex areas (nv), lean face area/g11/g12/g22 (nf each), boundary vertex
 * flags (nv, 0/1). Replaces core_analysis.py:651-707 and lean_geometry.py:44-63. */
int fcw_mesh_arrays(const double* vertices, int64_t n_vertices, const int32_t* faces, int64_t n_faces,
                    double* vertex_area, double* lean_area, double* g11, double* g12, double* g22,
                    uint8_t* boundary_flag);

/* The robust operators on the host (no device): the intrinsic Delaunay
 * triangulation by edge flips and its cotan Laplacian and lumped mass, as the
 * engine builds them when params->robust is set. First call with Lp == NULL to
 * get *nflips and *nnz; then Lp (n_vertices + 1), Li and Lx (nnz) receive L as
 * full symmetric CSC, mass (n_vertices) the lumped mass, and, when nflips > 0, the
 * flipped tufted cover (2 n_faces faces: the mesh's faces, then their back sides):
 * tri (3 corner vertices per cover face), len and twin (one per halfedge h =
 * 3 face + corner, from corner to the next; twin -1 on non-manifold edges). Any
 * output pointer may be NULL. */
int fcw_intrinsic_operators(const double* vertices, int64_t n_vertices, const int32_t* faces, int64_t n_faces,
                            int64_t* nflips, int64_t* nnz, int64_t* Lp, int32_t* Li, double* Lx, double* mass,
                            int32_t* tri, double* len, int32_t* twin);

/* Build the engine: operators, symbolic analysis, device factorisation of
 * M + tL and L + shift*M (and the grounded FP32 Poisson operator when
 * params->build_mixed). Replaces PotpourriDistanceEngine.__init__
 * (distance_engines.py:75-125) and ConsistentBatchHeatEngine.__init__
 * (fastcw_lean.py:481-502). The mesh may have several connected components
 * (fcw_info.n_components): every field still spans all vertices, and the
 * vertices off the source's component get the M-weighted mean distance over
 * that component, in both precisions, as the FP64 operator gives them. */
typedef struct fcw_engine fcw_engine;
int fcw_engine_create(const double* vertices, int64_t n_vertices, const int32_t* faces, int64_t n_faces,
                      const fcw_params* params, fcw_engine** out);
int fcw_engine_info(const fcw_engine* e, fcw_info* info);
int fcw_engine_destroy(fcw_engine* e);

/* One source, FP64 heat method, result in host memory (n_vertices doubles),
 * shifted so that d[source] = 0. Replaces BaseDistanceEngine.compute_distance
 * (distance_engines.py:67-69, 131-133). Runs its own chain (one-column sweeps);
 * the first call on an engine builds that chain's panel layouts (four arrays of
 * one factor's size) and captures it as a CUDA graph, so it should come before
 * any capture of the engine's stream. Copies run at full speed into page-locked
 * out_host. A source out of range is FCW_E_INVALID. */
int fcw_compute_distance(fcw_engine* e, int32_t source, double* out_host);

/* Distances for n sources into host memory, row j = distances from sources[j]
 * (n x n_vertices, C order), in the requested precision. Replaces
 * ConsistentBatchHeatEngine.compute_distance_batch (fastcw_lean.py:504-531). */
int fcw_compute_distances(fcw_engine* e, const int32_t* sources, int64_t n, int32_t precision, double* out_host);

/* All per-source metrics for n sources (host arrays in and out): health screen,
 * MSD, distance to boundary, radius/perimeter at each sorted target area and
 * n_between log-spaced samples between consecutive radii (core_analysis.py:1513-1611).
 * Vertex areas, boundary vertices and the health length are the engine's own,
 * computed from the same submesh exactly as core_analysis computes them. */
int fcw_compute_metrics(fcw_engine* e, const int32_t* sources, int64_t n, int32_t precision,
                        const double* targets, int32_t n_targets, int32_t n_between, double eps,
                        double* out_host);

/* Same, with sources and the output record array in device memory, enqueued on
 * stream (a cudaStream_t; NULL = legacy default stream). */
int fcw_compute_metrics_device(fcw_engine* e, const int32_t* sources_dev, int64_t n, int32_t precision,
                               const double* targets_host, int32_t n_targets, int32_t n_between,
                               double eps, double* out_dev, void* stream);

/* Cleaned (radius, area) samples of metric records (the fcw_compute_metrics
 * layout, n records of fcw_metrics_stride(nt, nb) doubles). Per healthy source:
 * the finite solved radii paired with their target areas, then the finite
 * supplementary samples, less those whose disc loses more than boundary_cap of
 * its area to a straight boundary at the record's distance to boundary rounded
 * to float32 (NaN: no cap; else in [0, 0.5)); stably sorted by radius, radii
 * within max(1e-12, 1e-9 * span) of their predecessor dropped, stored as float32
 * in rows of fcw_samples_capacity(nt, nb) with count_out[k] used. Flagged fields
 * get count 0. Replaces core_analysis.py:1599-1611 with boundary_area_loss_fraction
 * (:759-777) and _clean_vertex_samples (:1424-1439); the CSR over vertices
 * (:1619-1632) is the caller's concatenation of the rows. */
int fcw_samples_capacity(int32_t n_targets, int32_t n_between);
int fcw_assemble_samples_device(const double* records_dev, int64_t n, int32_t n_targets, int32_t n_between,
                                const double* targets, double boundary_cap, float* radii_out, float* areas_out,
                                int32_t* count_out, void* stream);
/* The same on host buffers, staged through the engine's device buffers. */
int fcw_assemble_samples(fcw_engine* e, const double* records, int64_t n, int32_t n_targets, int32_t n_between,
                         const double* targets, double boundary_cap, float* radii, float* areas, int32_t* count);

/* CUDA graphs in fcw_compute_metrics(_device): enable (1, the default) / disable (0).
 * Each workspace captures its block's launch chain once per set of arguments (K,
 * precision, targets, n_between, eps) and replays it for later blocks; the block's
 * sources and output pointer reach the chain through a device descriptor. While the
 * stage timeline is on, blocks launch directly. */
int fcw_engine_graphs(fcw_engine* e, int enable);

/* Stage timeline: enable (1) / disable (0) CUDA-event marks between pipeline
 * stages on the working stream and reset the accumulated times and launch count. */
int fcw_engine_profile(fcw_engine* e, int enable);
/* Accumulated milliseconds per stage (FCW_STAGE_*, n entries) and the number of
 * kernels launched since the last reset (nullable). Synchronises on the marks. */
int fcw_engine_stage_times(fcw_engine* e, double* ms_out, int32_t n, int64_t* launches);

/* Wait for the work enqueued on stream and report any error the kernels raised
 * (invalid source index, numerical failure). */
int fcw_synchronize(fcw_engine* e, void* stream);

/* Stage entry points (device pointers, caller vertex order, fields n_vertices x k
 * row-major unless noted), for checking each kernel on given inputs. */
/* (M + tL) u = delta_sources, FP64 (fastcw_lean.py:517-519). */
int fcw_heat_solve_device(fcw_engine* e, const int32_t* sources_dev, int32_t k, double* u_dev, void* stream);
/* div = sum_f A_f X_f . grad B_v, X = -grad u/|grad u| (fastcw_lean.py:416-442). */
int fcw_divergence_device(fcw_engine* e, const double* u_dev, int32_t k, double* div_dev, void* stream);
/* (L + shift*M) phi = div, then phi -= phi[source] per column (fastcw_lean.py:524-526). */
int fcw_poisson_solve_device(fcw_engine* e, const double* div_dev, const int32_t* sources_dev, int32_t k,
                             double* phi_dev, void* stream);
/* Metrics of given fields d (k x n_vertices, row j = field of sources[j]). */
int fcw_field_metrics_device(fcw_engine* e, const double* d_dev, const int32_t* sources_dev, int32_t k,
                             const double* targets_host, int32_t n_targets, int32_t n_between, double eps,
                             double* out_dev, void* stream);

/* One tensor-core product tile of the mixed Poisson sweeps, for checking their
 * arithmetic (no reference counterpart): C = A B (trans = 0, A m x k row-major)
 * or C = P^T B (trans = 1, P k x m row-major), B k x n row-major, C m x n, all
 * FP32 device arrays; m <= 128, k <= 64, n in {64, 128}. Each operand is split into
 * two TF32 terms and terms = 3 accumulates hi*hi + hi*lo + lo*hi (terms = 1: hi*hi)
 * with tcgen05.mma in tensor memory, through the sweeps' shared-memory layouts
 * (both operands K-major; the transposed P is transposed as it is written, as the
 * backward sweep's panels are).
 * terms = 0 only writes lane l, column c of the accumulator as l * 1024 + c and
 * reads it back (raw_dev); terms = 2 adds the hi*hi product to that pattern.
 * raw_dev (nullable) receives the 128 x n accumulator lanes; status_dev (one int,
 * zero on entry) gets a nonzero bit if the completion wait expired. */
int fcw_tc_product_check(const float* a_dev, const float* b_dev, float* c_dev, int32_t m, int32_t k, int32_t n,
                         int32_t terms, int32_t trans, float* raw_dev, int32_t* status_dev, void* stream);

/* Allocation-free field metrics, for callers that may not allocate device
 * memory while they run: a host that reserves the device for its own memory
 * pool, or a loop that must keep its device footprint fixed. Same arguments and
 * results as fcw_field_metrics_device; this entry point has no counterpart in
 * the reference. Its scratch is one 64 MiB array compiled into the library
 * (held by every device that loads it until the process exits); it takes at most
 * 32 fields per call and rejects meshes whose scratch would not fit with
 * FCW_E_INVALID (roughly 34k vertices with 32 fields). It calls no allocator.
 * The first call on each device looks up the array's device address; make that
 * call before any stream capture. Every call reuses the same array, so calls
 * that overlap on the GPU (other streams, other threads) race: serialise them.
 * Like the other entry points that take a stream, it returns once the work is
 * enqueued; an invalid source index found on the device is reported by the
 * next fcw_synchronize on that stream (FCW_E_INVALID). */
int fcw_field_metrics_static(fcw_engine* e, const double* d_dev, const int32_t* sources_dev, int32_t k,
                             const double* targets_host, int32_t n_targets, int32_t n_between, double eps,
                             double* out_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FCW_B200_H */
