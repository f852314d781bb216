"""Time the reference's own per-source loop against the oracle port, on this machine.

Test infrastructure: the bench's CPU arms run the oracle port (the reference is Python, so
there is nothing to build, and its modules do not travel to the GPU machine). This script
calibrates that port against the reference itself where the reference's modules import:
it runs the reference's FastCorticalWiringAnalysis.compute_all_wiring_costs
(core_analysis.py:1441-1672) with the reference's ConsistentBatchHeatEngine
(fastcw_lean.py:475-531, SciPy factorisation, one source per compute_distance call, the
lean geometry compiled by numba), and the port's per-source pipeline (oracle.HeatOracle and
oracle.source_metrics, what bench.py's cpu_baseline and --impl reference time) on the same
BFS-spaced sources of the same mesh, single-threaded, factorisations excluded.

    python -m oracle.time_reference --reference PATH [--level 5] [--sources 48]

PATH is a folder holding the reference's Python modules. Prints one JSON line.
"""

from __future__ import annotations

import argparse
import contextlib
import io
import json
import os
import sys
import time
import warnings

os.environ.setdefault("OMP_NUM_THREADS", "1")
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
os.environ.setdefault("NUMBA_NUM_THREADS", "1")

import numpy as np  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

SCALES = [0.002, 0.00267988, 0.00359088, 0.00481157, 0.00644721, 0.00863888,
          0.01157558, 0.01551059, 0.02078326, 0.02784833, 0.03731509, 0.05]


def _reference_loop(path, mesh, picks_sub):
    sys.path.insert(0, path)
    import lean_testkit as tk

    tk.install_stubs()
    import core_analysis as ca
    import distance_engines as de
    import fastcw_lean as fl
    import lean_geometry as lg

    class ConsistentHeatReference(de.BaseDistanceEngine):
        """The reference's batched heat engine, one source per call."""

        def __init__(self, vertices, faces, **kw):
            super().__init__(vertices, faces, **kw)
            h = lg.mean_edge_length(self.vertices, self.faces)
            self._eng = fl.ConsistentBatchHeatEngine(self.vertices, self.faces, t_coef=(0.7 / h) ** 2,
                                                     factor="scipy")

        @property
        def name(self):
            return "consistent_heat_reference"

        def compute_distance(self, s):
            return self._eng.compute_distance(int(s))

    de.ENGINE_REGISTRY["consistent_heat_reference"] = ConsistentHeatReference
    quiet = (contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()))
    with quiet[0], quiet[1], warnings.catch_warnings():
        warnings.simplefilter("ignore")
        an = ca.FastCorticalWiringAnalysis(mesh.vertices, mesh.faces, mesh.cortex_mask,
                                           engine_type="consistent_heat_reference")
        subset = an.sub_to_orig[np.asarray(picks_sub)]
        # warm the numba kernels and the factor's first solve on one source
        an.compute_all_wiring_costs(scale=SCALES, vertex_subset=subset[:1], n_samples_between_scales=3)
        t0 = time.perf_counter()
        an.compute_all_wiring_costs(scale=SCALES, vertex_subset=subset, n_samples_between_scales=3)
        sec = time.perf_counter() - t0
    return sec


def _port_loop(mesh, picks_sub):
    import oracle
    from fastcorticalwiring_b200 import mesh as M

    pm = M.prepare(mesh.vertices, mesh.faces, mesh.cortex_mask)
    targets = pm.targets(M.RUNNER_SCALES)
    ho = oracle.HeatOracle(pm.V, pm.F)

    def one(s):
        d = ho.distances([int(s)])[0]
        return oracle.source_metrics(d, int(s), pm, targets)

    one(picks_sub[0])
    t0 = time.perf_counter()
    for s in picks_sub:
        one(s)
    return time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="folder holding the reference's Python modules")
    ap.add_argument("--level", type=int, default=5)
    ap.add_argument("--sources", type=int, default=48)
    args = ap.parse_args()
    from fastcorticalwiring_b200 import mesh as M
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    mesh = folded_icosphere(args.level, seed=0, jitter=0.0)
    pm = M.prepare(mesh.vertices, mesh.faces, mesh.cortex_mask)
    picks = [int(x) for x in pm.bfs[np.linspace(0, pm.n_vertices - 1, args.sources).astype(int)]]
    ref_sec = _reference_loop(args.reference, mesh, picks)
    port_sec = _port_loop(mesh, picks)
    n = len(picks)
    print(json.dumps({"mesh": f"L{args.level} folded icosphere, {pm.n_vertices} cortical vertices",
                      "sources": n, "threads": 1,
                      "reference_loop_sources_per_s": n / ref_sec, "port_sources_per_s": n / port_sec,
                      "port_over_reference": ref_sec / port_sec}))


if __name__ == "__main__":
    main()
