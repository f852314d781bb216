// Internal declarations shared by the host runtime and the CUDA kernels.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fcw {

// ---------------------------------------------------------------------------
// Per-mesh host arrays, in the caller's (cortical submesh) vertex order.
// Every quantity restates a reference computation; see prep.cpp.
// ---------------------------------------------------------------------------
struct MeshPrep {
    int64_t nv = 0, nf = 0;
    std::vector<double> V;             // nv*3
    std::vector<int32_t> F;            // nf*3
    double mean_edge = 0.0;            // distance_engines.py:17-21
    double bin_width = 0.0;            // lean_geometry.py:99-114
    double health_h = 0.0;             // core_analysis.py:705 (median face max edge)
    double total_area = 0.0;           // sum of barycentric vertex areas (core_analysis.py:1512)
    std::vector<double> grad_area;     // fastcw_lean.py:375-391 face area
    std::vector<double> gb;            // nf*9: gb0, gb1, gb2 (3-vectors)
    std::vector<double> lean_area, g11, g12, g22;  // lean_geometry.py:44-63
    std::vector<double> vertex_area;   // core_analysis.py:959-978 (face order)
    std::vector<double> mass;          // fastcw_lean.py:410-412 (corner order)
    std::vector<int32_t> boundary;     // core_analysis.py:651-665
    // stiffness L = G^T diag(A) G, full symmetric CSC (fastcw_lean.py:394-409)
    std::vector<int64_t> Lp;
    std::vector<int32_t> Li;
    std::vector<double> Lx;
    // after intrinsic_delaunay flipped some edge: the intrinsic triangulation (corner
    // vertices per face, length and twin per halfedge, -1 on fixed edges)
    std::vector<int32_t> itri, itwin;
    std::vector<double> ilen;
};

int prepare_mesh(const double* V, int64_t nv, const int32_t* F, int64_t nf, MeshPrep& out, std::string& err);

// Replace L and the lumped mass by those of the intrinsic Delaunay triangulation
// (intrinsic.cpp); mollify_factor scales the mean edge length into the triangle
// inequality margin. nflips = 0 leaves the operators untouched.
int intrinsic_delaunay(MeshPrep& m, double mollify_factor, int64_t& nflips, std::string& err);

// ---------------------------------------------------------------------------
// Symbolic sparse Cholesky analysis (host). All indices are in the
// elimination ("new") order unless stated otherwise.
// ---------------------------------------------------------------------------
struct Symbolic {
    int64_t n = 0;
    std::vector<int32_t> perm;    // perm[new] = old
    std::vector<int32_t> iperm;   // iperm[old] = new
    int32_t nsuper = 0;
    std::vector<int32_t> sn_c0;   // first column; size nsuper+1 (sn_c0[nsuper] = n)
    std::vector<int32_t> sn_m;    // rows in the front = ns + nr
    std::vector<int64_t> sn_rowptr;  // offsets into rows; size nsuper+1
    std::vector<int32_t> rows;    // first ns entries are the supernode's own columns
    std::vector<int64_t> sn_valptr;  // panel offset (m x ns, row-major)
    std::vector<int64_t> sn_invptr;  // inverse diagonal block offset (ns x ns, row-major, lower)
    std::vector<int64_t> sn_updptr;  // update matrix offset (nr x nr, row-major)
    std::vector<int32_t> sn_parent;
    std::vector<int32_t> sn_level;   // height: 0 for leaves
    std::vector<int32_t> col_sn;     // supernode owning each column
    int32_t nlevels = 0;
    std::vector<int32_t> level_ptr;  // size nlevels+1
    std::vector<int32_t> level_nodes;
    std::vector<int32_t> child_ptr;  // size nsuper+1
    std::vector<int32_t> child_list;
    std::vector<int32_t> relind;     // aligned with rows: for pos >= ns, position of rows[pos] in the parent's row list
    // row-oriented off-diagonal segments for the forward pull
    std::vector<int64_t> seg_ptr;    // size n+1
    std::vector<int32_t> seg_sn;
    std::vector<int32_t> seg_pos;
    // assembly of A's lower triangle into the panels
    std::vector<int64_t> a_dst;      // destination offsets in the value array
    std::vector<int64_t> a_src;      // index of the entry in MeshPrep::Li/Lx
    std::vector<int32_t> a_col;      // its column in the caller's order (diagonal if Li[a_src] == a_col)
    int64_t nnz_factor = 0, n_inv = 0, n_upd = 0, nnz_lower_a = 0;
    int32_t max_ns = 0, max_m = 0;
    int64_t nnz_l = 0;               // nonzeros of L counting the dense panels
    double flops_factor = 0.0;
};

int build_symbolic(const MeshPrep& mesh, int leaf_size, int max_width, int relax, Symbolic& S, std::string& err);

}  // namespace fcw
