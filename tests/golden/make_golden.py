#!/usr/bin/env python3
"""Generate the golden fixtures from the reference's own code.

Run with --reference PATH naming a FastCorticalWiring checkout whose modules
import (numba, scipy). The tests never run this:
its outputs are committed next to it as small .npz files.

Reference code run here, unmodified:
  * fastcw_lean.ConsistentBatchHeatEngine (factor="scipy")  -- heat-method distances
  * fastcw_lean.fused_normalized_divergence                 -- divergence of X
  * lean_geometry.per_source_geometry / area_at / perimeter_at / solve_radius / field_health
  * core_analysis.FastCorticalWiringAnalysis.compute_all_wiring_costs, with an
    engine registered into distance_engines.ENGINE_REGISTRY that wraps the
    heat engine (the same hook lean_testkit.install_stubs uses)
  * lean_testkit icosphere/bumpy meshes + euclid stub fields (geometry KATs)

Fixtures:
  golden_heat_L4.npz      seeded folded L4 mesh, distances/heat/divergence for 8 sources,
                          per-source FP64 geometry, health, MSD/boundary, and the
                          float32 arrays the analysis loop writes (incl. sample CSR)
  golden_metrics_L5.npz   same analysis outputs on a seeded folded L5 mesh (16 sources)
  golden_geometry_kat.npz lean geometry on euclid-stub and non-Lipschitz fields (L4 bumpy),
                          area/perimeter at fixed radii, per_source_geometry, NaN rules
  golden_components_L4.npz the analysis on a submesh of two connected components (a seeded
                          folded L4 mesh with a half-size folded L3 mesh inside it): fields and
                          outputs for 10 sources in both components
  golden_samples_L5.npz   sample assembly with a boundary cap on the L5 mesh: 24 sources near
                          the boundary run through compute_all_wiring_costs(boundary_cap_fraction=0.05),
                          their FP64 geometry records and float32 distance to boundary, the sample
                          CSR; boundary_area_loss_fraction on an (r, d) grid; _clean_vertex_samples
                          on crafted pair lists; the keys and dtypes save_analysis_npz writes
"""

import argparse
import contextlib
import io
import os
import sys
import warnings
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _ref_modules(path):
    sys.path.insert(0, path)
    import lean_testkit as tk  # noqa: E402

    tk.install_stubs()
    import core_analysis as ca  # noqa: E402
    import distance_engines as de  # noqa: E402
    import fastcw_lean as fl  # noqa: E402
    import lean_geometry as lg  # noqa: E402

    class ConsistentHeatReference(de.BaseDistanceEngine):
        """The reference's own batched heat engine, one source per call."""

        def __init__(self, vertices, faces, **kw):
            super().__init__(vertices, faces, **kw)
            L = float(self.engine_kwargs.get("diffusion_length_mm", 0.7))
            h = lg.mean_edge_length(self.vertices, self.faces)
            self._eng = fl.ConsistentBatchHeatEngine(self.vertices, self.faces, t_coef=(L / h) ** 2,
                                                     factor="scipy")

        @property
        def name(self):
            return "consistent_heat_reference"

        def compute_distance(self, s):
            return self._eng.compute_distance(int(s))

    de.ENGINE_REGISTRY["consistent_heat_reference"] = ConsistentHeatReference
    return ca, de, fl, lg, tk


SCALES = [0.002, 0.00267988, 0.00359088, 0.00481157, 0.00644721, 0.00863888,
          0.01157558, 0.01551059, 0.02078326, 0.02784833, 0.03731509, 0.05]


def _analysis_fixture(ca, lg, fl, mesh, n_sources, with_stages):
    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()):
        an = ca.FastCorticalWiringAnalysis(mesh.vertices, mesh.faces, mesh.cortex_mask,
                                           engine_type="consistent_heat_reference")
    order = np.asarray(an._bfs_order)
    pick = order[np.linspace(0, order.size - 1, n_sources).astype(int)]
    subset = an.sub_to_orig[pick]
    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()), \
            warnings.catch_warnings():
        warnings.simplefilter("ignore")
        an.compute_all_wiring_costs(scale=SCALES, vertex_subset=subset, n_samples_between_scales=3)
    out = dict(
        V=mesh.vertices, F=mesh.faces, mask=mesh.cortex_mask, level=mesh.level, seed=mesh.seed,
        jitter=mesh.jitter, scales=np.asarray(SCALES), sources_sub=pick.astype(np.int64),
        sources_orig=subset.astype(np.int64), bfs_order=order.astype(np.int64),
        boundary=an.boundary_indices.astype(np.int64), vertex_area=an.vertex_areas_sub,
        health_h=an._health_h, bin_width=an._lean_width,
        t=an.distance_engine._eng.t,
    )
    for k, v in an.get_metric_arrays().items():
        out["f32_" + k] = v[subset]
    out["field_flag"] = an.field_flag[subset]
    indptr, rs, as_ = [0], [], []
    for o in subset:
        r, a = an.get_vertex_samples(int(o))
        rs.append(r)
        as_.append(a)
        indptr.append(indptr[-1] + r.size)
    out["sample_indptr"] = np.asarray(indptr, np.int64)
    out["sample_r"] = np.concatenate(rs).astype(np.float32)
    out["sample_a"] = np.concatenate(as_).astype(np.float32)
    # FP64 per-stage values from the reference engine and lean geometry
    eng = an.distance_engine._eng
    phi = eng.compute_distance_batch(pick)
    out["phi"] = phi
    T = np.array(SCALES) * float(an.vertex_areas_sub.sum())
    out["targets"] = T
    fr = np.array([0.25, 0.5, 0.75])
    nF = an.faces.shape[0]
    bufs = (np.empty(nF), np.empty(nF, np.int32), np.empty(nF, np.int32))
    R, P, ER, EA, NE, H = [], [], [], [], [], []
    for j, s in enumerate(pick):
        r, p, er, ea = np.empty(12), np.empty(12), np.empty(33), np.empty(33)
        ne = lg.per_source_geometry(phi[j], an.faces, an._lean_area, an._lean_g11, an._lean_g12,
                                    an._lean_g22, an._lean_width, T, fr, 1e-10, 60, *bufs, r, p, er, ea)
        R.append(r)
        P.append(p)
        ER.append(er)
        EA.append(ea)
        NE.append(ne)
        H.append(lg.field_health(phi[j], an.vertices, int(s), an._health_h))
    out.update(radii=np.array(R), perim=np.array(P), extra_r=np.array(ER), extra_a=np.array(EA),
               n_eval=np.array(NE), health=np.array([[h[0], h[1], float(h[2])] for h in H]))
    if with_stages:
        src2 = pick[:3]
        rhs = np.zeros((eng.n_vertices, src2.size))
        rhs[src2, np.arange(src2.size)] = 1.0
        u = np.ascontiguousarray(eng._heat.solve(rhs))
        div = np.empty_like(u)
        fl.fused_normalized_divergence(u, eng.F, eng.area, eng.gb0, eng.gb1, eng.gb2, div)
        out.update(stage_sources=src2.astype(np.int64), stage_u=u, stage_div=div)
    return out


def _params_fixture(ca, mesh, n_sources, diffusion_length_mm, n_between):
    """The analysis with non-default settings: diffusion length, the default scales, n_between."""
    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()):
        an = ca.FastCorticalWiringAnalysis(mesh.vertices, mesh.faces, mesh.cortex_mask,
                                           engine_type="consistent_heat_reference",
                                           engine_kwargs={"diffusion_length_mm": diffusion_length_mm})
    order = np.asarray(an._bfs_order)
    pick = order[np.linspace(0, order.size - 1, n_sources).astype(int)]
    subset = an.sub_to_orig[pick]
    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()), \
            warnings.catch_warnings():
        warnings.simplefilter("ignore")
        an.compute_all_wiring_costs(scale=None, vertex_subset=subset, n_samples_between_scales=n_between)
    out = dict(V=mesh.vertices, F=mesh.faces, mask=mesh.cortex_mask, level=mesh.level, seed=mesh.seed,
               jitter=mesh.jitter, diffusion_length_mm=float(diffusion_length_mm), n_between=int(n_between),
               scales=np.asarray(ca.FastCorticalWiringAnalysis.DEFAULT_SCALES, dtype=np.float64),
               sources_orig=subset.astype(np.int64), t=an.distance_engine._eng.t)
    for k, v in an.get_metric_arrays().items():
        out["f32_" + k] = v[subset]
    out["field_flag"] = an.field_flag[subset]
    indptr, rs, as_ = [0], [], []
    for o in subset:
        r, a = an.get_vertex_samples(int(o))
        rs.append(r)
        as_.append(a)
        indptr.append(indptr[-1] + r.size)
    out["sample_indptr"] = np.asarray(indptr, np.int64)
    out["sample_r"] = np.concatenate(rs).astype(np.float32)
    out["sample_a"] = np.concatenate(as_).astype(np.float32)
    return out


def _samples_fixture(ca, lg, mesh, n_sources, cap):
    import io_utils as iu  # noqa: E402  (the reference's writer)
    import tempfile

    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()):
        an = ca.FastCorticalWiringAnalysis(mesh.vertices, mesh.faces, mesh.cortex_mask,
                                           engine_type="consistent_heat_reference")
    # sources spread over 0..40 mm from the boundary (in space), where the cap removes
    # some supplementary samples and keeps others
    Vs = an.vertices
    bnd = an.boundary_indices
    dist = np.min(np.linalg.norm(Vs[:, None, :] - Vs[bnd][None, :, :], axis=2), axis=1)
    cand = np.argsort(dist, kind="stable")
    want = np.linspace(0.0, 40.0, n_sources)
    pick = np.unique(cand[np.searchsorted(dist[cand], want)])
    subset = an.sub_to_orig[pick]
    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()), \
            warnings.catch_warnings():
        warnings.simplefilter("ignore")
        an.compute_all_wiring_costs(scale=SCALES, vertex_subset=subset, n_samples_between_scales=3,
                                    boundary_cap_fraction=cap)
    out = dict(level=mesh.level, seed=mesh.seed, jitter=mesh.jitter, scales=np.asarray(SCALES),
               cap=np.float64(cap), sources_sub=pick.astype(np.int64), sources_orig=subset.astype(np.int64))
    out["field_flag"] = an.field_flag[subset]
    out["f32_dist_to_boundary"] = an.dist_to_boundary[subset]
    indptr, rs, as_ = [0], [], []
    for o in subset:
        r, a = an.get_vertex_samples(int(o))
        rs.append(r)
        as_.append(a)
        indptr.append(indptr[-1] + r.size)
    out["sample_indptr"] = np.asarray(indptr, np.int64)
    out["sample_r"] = np.concatenate(rs).astype(np.float32)
    out["sample_a"] = np.concatenate(as_).astype(np.float32)
    eng = an.distance_engine._eng
    phi = eng.compute_distance_batch(pick)
    T = np.array(SCALES) * float(an.vertex_areas_sub.sum())
    fr = np.array([0.25, 0.5, 0.75])
    nF = an.faces.shape[0]
    bufs = (np.empty(nF), np.empty(nF, np.int32), np.empty(nF, np.int32))
    R, ER, EA = [], [], []
    for j in range(pick.size):
        r, p, er, ea = np.empty(12), np.empty(12), np.empty(33), np.empty(33)
        lg.per_source_geometry(phi[j], an.faces, an._lean_area, an._lean_g11, an._lean_g12, an._lean_g22,
                               an._lean_width, T, fr, 1e-10, 60, *bufs, r, p, er, ea)
        R.append(r)
        ER.append(er)
        EA.append(ea)
    out.update(targets=T, radii=np.array(R), extra_r=np.array(ER), extra_a=np.array(EA))
    # boundary_area_loss_fraction on a grid, including the non-finite and degenerate cases
    rr = np.array([0.0, -1.0, np.nan, np.inf, 1e-3, 1.0, 5.0, 10.0, 14.5, 15.2, 31.0])
    dd = np.array([0.0, 1e-9, 0.5, 5.0, 9.99, 10.0, 10.01, 20.0, np.inf, np.nan, -1.0])
    out["loss_r"], out["loss_d"] = np.meshgrid(rr, dd, indexing="ij")
    out["loss"] = np.vectorize(ca.FastCorticalWiringAnalysis.boundary_area_loss_fraction)(out["loss_r"],
                                                                                          out["loss_d"])
    # _clean_vertex_samples on crafted lists: ties, near-duplicates, a single pair, unsorted input
    rng = np.random.default_rng(3)
    cases = [[(1.0, 2.0)], [(3.0, 1.0), (1.0, 2.0), (2.0, 3.0)],
             [(1.0, 1.0), (1.0 + 1e-13, 2.0), (1.0, 3.0), (2.0, 4.0)],
             [(5.0, 1.0), (5.0 + 3e-9, 2.0), (5.0 + 2e-8, 3.0), (10.0, 4.0)]]
    cases.append([(float(x), float(y)) for x, y in rng.random((40, 2)) * 10])
    cin, cout = [], []
    for c in cases:
        cin.append(np.asarray(c, np.float64))
        cout.append(np.asarray(ca.FastCorticalWiringAnalysis._clean_vertex_samples(c), np.float64))
    out["clean_in_indptr"] = np.cumsum([0] + [len(c) for c in cin]).astype(np.int64)
    out["clean_in"] = np.concatenate(cin)
    out["clean_out_indptr"] = np.cumsum([0] + [len(c) for c in cout]).astype(np.int64)
    out["clean_out"] = np.concatenate(cout)
    # what the reference's NPZ writer stores: key, dtype, shape
    with tempfile.TemporaryDirectory() as tmp:
        path = iu.save_analysis_npz(tmp, "a.npz", an, n_samples_between_scales=3)
        z = np.load(path)
        out["npz_keys"] = np.asarray(sorted(z.files))
        out["npz_dtypes"] = np.asarray([str(z[k].dtype) for k in sorted(z.files)])
        out["npz_ndims"] = np.asarray([z[k].ndim for k in sorted(z.files)], np.int64)
        out["npz_schema"] = np.asarray(int(z["fastcw_output_schema_version"]))
    return out


def _geometry_kat(ca, lg, tk):
    V, F = tk.icosphere(4)
    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()):
        an = ca.FastCorticalWiringAnalysis(tk.bumpy(V), F, np.ones(len(V), bool), engine_type="euclid_stub")
    Vs, Fs = an.vertices, an.faces
    nF = len(Fs)
    area, g11, g12, g22 = lg.precompute_face_metric(Vs, Fs)
    w = lg.default_bin_width(Vs, Fs)
    bufs = (np.empty(nF), np.empty(nF, np.int32), np.empty(nF, np.int32))
    rng = np.random.default_rng(1)
    field_sources = [int(s) for s in rng.choice(len(Vs), 3, replace=False)] + [7]
    fields = [an._compute_geodesic_distances_from_subvertex(s) for s in field_sources[:3]]
    d = an._compute_geodesic_distances_from_subvertex(7).copy()
    bad = rng.choice(len(d), len(d) // 50, replace=False)
    d[bad] += rng.uniform(0, 15, bad.size)
    fields.append(d)
    fields = np.array(fields)
    radii = np.array([rng.uniform(0.5, np.nanmax(f) * 0.8, 12) for f in fields])
    A, DA, P, NL = [], [], [], []
    for f, rr in zip(fields, radii):
        nb, ptr, pre, nl = lg.build_distance_buckets(f, Fs, area, w, *bufs)
        a_row, da_row, p_row = [], [], []
        for r in rr:
            a, da = lg.area_at(r, f, Fs, area, w, nb, ptr, pre, bufs[1], bufs[0], bufs[2], nl)
            a_row.append(a)
            da_row.append(da)
            p_row.append(lg.perimeter_at(r, f, Fs, area, g11, g12, g22, w, nb, ptr, bufs[1], bufs[0], bufs[2], nl))
        A.append(a_row)
        DA.append(da_row)
        P.append(p_row)
        NL.append(nl)
    T = np.array(SCALES) * float(an.vertex_areas_sub.sum())
    fr = np.array([0.25, 0.5, 0.75])
    G = []
    for f in (fields[0], fields[3]):
        ro, po, er, ea = np.empty(12), np.empty(12), np.empty(33), np.empty(33)
        n = lg.per_source_geometry(f, Fs, area, g11, g12, g22, w, T, fr, 1e-12, 60, *bufs, ro, po, er, ea)
        G.append((ro, po, er, ea, n))
    f = fields[3]
    nb, ptr, pre, nl = lg.build_distance_buckets(f, Fs, area, w, *bufs)
    a_nan, _ = lg.area_at(np.nan, f, Fs, area, w, nb, ptr, pre, bufs[1], bufs[0], bufs[2], nl)
    r_nan, _ = lg.solve_radius(np.nan, f, Fs, area, w, nb, ptr, pre, bufs[1], bufs[0], bufs[2], nl, 1e-12, 60)
    r_big, _ = lg.solve_radius(pre[nb] * 2, f, Fs, area, w, nb, ptr, pre, bufs[1], bufs[0], bufs[2], nl, 1e-12, 60)
    r_zero, _ = lg.solve_radius(0.0, f, Fs, area, w, nb, ptr, pre, bufs[1], bufs[0], bufs[2], nl, 1e-12, 60)
    return dict(
        V=Vs, F=Fs, fields=fields, field_sources=np.array(field_sources), radii_eval=radii, area_eval=np.array(A), darea_eval=np.array(DA),
        perim_eval=np.array(P), n_long=np.array(NL), bin_width=w, targets=T, fracs=fr,
        geo_radii=np.array([g[0] for g in G]), geo_perim=np.array([g[1] for g in G]),
        geo_extra_r=np.array([g[2] for g in G]), geo_extra_a=np.array([g[3] for g in G]),
        geo_n_eval=np.array([g[4] for g in G]), total_area=pre[nb],
        nan_area=a_nan, nan_radius=r_nan, big_radius=r_big, zero_radius=r_zero,
    )


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="folder holding the reference's Python modules")
    ap.add_argument("--only", default=None, help="write only this fixture (file name)")
    args = ap.parse_args()
    sys.path.insert(0, REPO)
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    ca, de, fl, lg, tk = _ref_modules(args.reference)
    l4 = folded_icosphere(4, seed=11, jitter=0.2)
    l5 = folded_icosphere(5, seed=5)
    l4b = folded_icosphere(4, seed=21, jitter=0.3)

    def metrics_l5():
        fx = _analysis_fixture(ca, lg, fl, l5, 16, False)
        fx.pop("phi")  # large; the L5 fixture pins outputs, not fields
        return fx

    a, b = folded_icosphere(4, seed=3, jitter=0.2), folded_icosphere(3, seed=5, jitter=0.1)
    two = SimpleNamespace(vertices=np.vstack([a.vertices, 0.5 * b.vertices]),
                          faces=np.vstack([a.faces, b.faces + len(a.vertices)]),
                          cortex_mask=np.concatenate([a.cortex_mask, b.cortex_mask]), level=4, seed=3, jitter=0.2)

    fixtures = {
        "golden_heat_L4.npz": lambda: _analysis_fixture(ca, lg, fl, l4, 8, True),
        "golden_metrics_L5.npz": metrics_l5,
        "golden_geometry_kat.npz": lambda: _geometry_kat(ca, lg, tk),
        "golden_samples_L5.npz": lambda: _samples_fixture(ca, lg, l5, 24, 0.05),
        "golden_params_L4.npz": lambda: _params_fixture(ca, l4b, 12, 1.0, 1),
        "golden_components_L4.npz": lambda: _analysis_fixture(ca, lg, fl, two, 10, False),
    }
    for name, make in fixtures.items():
        if args.only and name != args.only:
            continue
        np.savez_compressed(os.path.join(HERE, name), **make())
        print(name, os.path.getsize(os.path.join(HERE, name)))


if __name__ == "__main__":
    main()
