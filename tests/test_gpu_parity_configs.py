"""CUDA engine vs the oracle at the benchmark's mesh sizes (needs a B200).

The workloads are the seeded folded icospheres the benchmark measures:
  * L6, jitter 0.2 (36,866 cortical vertices, 41 etree levels);
  * L7, the headline mesh (147,458 cortical vertices, 33 etree levels);
  * L8, jitter 0.2 (589,826 cortical vertices, 59 etree levels).
At these sizes the engine runs code paths the small meshes never reach: deep etree
level schedules, split-K backward tasks over long structures, the chain of root
separators, retries of the metrics kernel's first cut, and several blocks in flight.

Sources are BFS-spaced over the whole mesh and the engine runs them in 1024-source
blocks; the sources checked against the oracle are spread over every block and over
the blocks' column tiles. The oracle (oracle.HeatOracle + oracle.source_metrics) runs
the reference's method in FP64 on the CPU for the checked sources only.

Bars:
  * FP64 engine: radius, perimeter and samples within 1e-9 relative (the radius solve
    stops at rtol 1e-10), MSD and distance to boundary within 1e-9, distances within
    1e-10 x max|d|; health fractions and flags identical.
  * mixed engine: radius, perimeter and sample areas within 1e-4 relative, MSD within
    1e-5, distance to boundary within 1e-4, distances within 1e-4 x max|d|; health
    flags identical except where the oracle's count sits within two vertices of the
    screen's threshold (one vertex's FP32 rounding can move it across).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import engine, mesh as M  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402

CONFIGS = {
    "L6j": dict(level=6, jitter=0.2, n_run=4096, n_check=64),
    "L7": dict(level=7, jitter=0.0, n_run=4096, n_check=64),
    "L8j": dict(level=8, jitter=0.2, n_run=2048, n_check=16),
}
BARS = {
    "fp64": dict(geom=1e-9, msd=1e-9, dist_b=1e-9, phi=1e-10),
    "mixed": dict(geom=1e-4, msd=1e-5, dist_b=1e-4, phi=1e-4),
}
HEALTH_TOL = 1e-3  # lean_geometry.py:343-357


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def _check_positions(n_run, n_check):
    """Positions in the run spread over every 1024-source block and varied column offsets."""
    step = n_run // n_check
    return np.array([j * step + (j * 37) % step for j in range(n_check)], dtype=np.int64)


@pytest.fixture(scope="module", params=list(CONFIGS))
def config(request):
    import oracle

    name = request.param
    c = CONFIGS[name]
    m = folded_icosphere(c["level"], seed=0, jitter=c["jitter"])
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    run = pm.bfs[np.linspace(0, pm.n_vertices - 1, c["n_run"]).astype(int)].astype(np.int32)
    pos = _check_positions(c["n_run"], c["n_check"])
    chk = run[pos]
    targets = pm.targets(M.RUNNER_SCALES)
    ho = oracle.HeatOracle(pm.V, pm.F)
    phi = ho.distances(chk)
    ref = [oracle.source_metrics(phi[j], int(s), pm, targets) for j, s in enumerate(chk)]
    eng = engine.HeatEngine(pm.V, pm.F, block_k=1024, pipeline_depth=2)
    z = dict(name=name, pm=pm, run=run, pos=pos, chk=chk, targets=targets, phi=phi, ref=ref, eng=eng)
    yield z
    eng.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_metrics_match_oracle_at_benchmark_sizes(config, precision):
    z = config
    pm, eng, ref = z["pm"], z["eng"], z["ref"]
    bar = BARS[precision]
    rec = eng.compute_metrics(z["run"], z["targets"], n_between=3, precision=precision)
    r = engine.split_records(rec[z["pos"]], len(M.RUNNER_SCALES), 3)
    n = pm.n_vertices
    errs = dict(radius=0.0, perimeter=0.0, extra_a=0.0, msd=0.0, dist_b=0.0)
    borderline = 0
    for j, o in enumerate(ref):
        near = min(abs(o["neg"] - HEALTH_TOL), abs(o["viol"] - HEALTH_TOL)) <= 2.0 / n
        if precision == "fp64":
            assert r["neg"][j] == o["neg"] and r["viol"][j] == o["viol"], (j, r["neg"][j], o["neg"])
            assert bool(r["bad"][j]) == o["bad"], j
        elif bool(r["bad"][j]) != o["bad"]:
            assert near, (j, r["neg"][j], r["viol"][j], o["neg"], o["viol"])
            borderline += 1
        if r["bad"][j] or o["bad"]:
            assert np.all(np.isnan(r["radii"][j])) if r["bad"][j] else True
            continue
        errs["radius"] = max(errs["radius"], float(np.max(_rel(r["radii"][j], o["radii"]))))
        errs["perimeter"] = max(errs["perimeter"], float(np.max(_rel(r["perim"][j], o["perim"]))))
        errs["extra_a"] = max(errs["extra_a"], float(np.max(_rel(r["extra_a"][j], o["extra_a"]))))
        errs["msd"] = max(errs["msd"], float(_rel(r["msd_u"][j], o["msd_u"])), float(_rel(r["msd_w"][j], o["msd_w"])))
        errs["dist_b"] = max(errs["dist_b"], float(_rel(r["dist_b"][j], o["dist_b"])))
    print(f"\nPARITY {z['name']} {precision} sources={len(ref)} flagged={int(r['bad'].sum())} "
          f"borderline={borderline} " + " ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    assert borderline <= 1
    assert errs["radius"] <= bar["geom"] and errs["perimeter"] <= bar["geom"] and errs["extra_a"] <= bar["geom"]
    assert errs["msd"] <= bar["msd"]
    assert errs["dist_b"] <= bar["dist_b"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_distances_match_oracle_at_benchmark_sizes(config, precision):
    """Four of the checked sources' whole fields, in blocks of the run's size."""
    z = config
    pick = np.linspace(0, len(z["chk"]) - 1, 4).astype(int)
    d = z["eng"].compute_distances(z["chk"][pick], precision=precision)
    ref = z["phi"][pick]
    err = np.max(np.abs(d - ref), axis=1) / np.max(np.abs(ref), axis=1)
    print(f"\nPARITY {z['name']} {precision} phi_max_abs_over_max={np.max(err):.2e}")
    assert np.max(err) <= BARS[precision]["phi"], err
    for j, s in enumerate(z["chk"][pick]):
        assert d[j, s] == 0.0
