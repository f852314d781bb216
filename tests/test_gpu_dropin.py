"""The single-source drop-in, fcw_compute_distance (needs a B200).

It runs its own chain: the heat forward solve along the source's path to the root
(one CTA), then persistent sweeps that take supernodes in dependency order from a
ticket counter (heat backward, Poisson forward and backward), a one-column
divergence and the shift. Its fields must match the batched FP64 path (another
schedule of the same factors: to 1e-12 of the field's maximum) and the oracle (1e-9),
for sources whose paths to the root differ in length (a leaf column, a middle one,
the root separator), and repeated calls must give the same bits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import _lib, engine, mesh as M  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402


@pytest.fixture(scope="module")
def l6():
    m = folded_icosphere(6, seed=3, jitter=0.2)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    eng = engine.HeatEngine(pm.V, pm.F)
    perm = _lib.analyze(pm.V, pm.F)[1]  # perm[elimination index] = vertex
    n = pm.n_vertices
    picks = [int(perm[0]), int(perm[n // 3]), int(perm[n // 2]), int(perm[n - 1])]
    picks += [int(x) for x in pm.bfs[np.linspace(0, n - 1, 12).astype(int)]]
    yield pm, eng, picks
    eng.close()


def _maxrel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_dropin_matches_batched_fp64(l6):
    pm, eng, picks = l6
    batched = eng.compute_distances(np.asarray(picks, np.int32), precision="fp64")
    for j, s in enumerate(picks):
        d = eng.compute_distance(s)
        assert d.shape == (pm.n_vertices,) and d.dtype == np.float64
        assert d[s] == 0.0
        assert _maxrel(d, batched[j]) <= 1e-12, (s, _maxrel(d, batched[j]))


def test_dropin_matches_oracle(l6):
    import oracle

    pm, eng, picks = l6
    sel = picks[:4]
    ref = oracle.HeatOracle(pm.V, pm.F).distances(np.asarray(sel))
    for j, s in enumerate(sel):
        assert _maxrel(eng.compute_distance(s), ref[j]) <= 1e-9


def test_dropin_is_deterministic_and_graph_free_path_agrees(l6):
    pm, eng, picks = l6
    s = picks[5]
    a = eng.compute_distance(s)
    b = eng.compute_distance(picks[6])
    c = eng.compute_distance(s)
    assert np.array_equal(a, c)
    assert not np.array_equal(a, b)
    eng.graphs(False)
    try:
        d = eng.compute_distance(s)
    finally:
        eng.graphs(True)
    assert np.array_equal(a, d)


def test_dropin_rejects_bad_source_and_recovers(l6):
    pm, eng, picks = l6
    for bad in (-1, pm.n_vertices):
        with pytest.raises((ValueError, RuntimeError)):
            eng.compute_distance(bad)
    d = eng.compute_distance(picks[0])
    assert d[picks[0]] == 0.0 and np.all(np.isfinite(d))


def test_single_source_metrics_match_batched(l6):
    """compute_metrics on one source in FP64 runs the drop-in chain and one-column statistics;
    its records must equal the batched path's for the same sources (two schedules of the same
    FP64 solve: to 1e-10 relative; flags and counts exactly)."""
    pm, eng, picks = l6
    targets = pm.targets(M.RUNNER_SCALES)
    sel = np.asarray(picks[:6], np.int32)
    batched = engine.split_records(eng.compute_metrics(sel, targets, precision="fp64"), targets.size, 3)
    for j, s in enumerate(sel):
        one = engine.split_records(eng.compute_metrics(np.array([s], np.int32), targets, precision="fp64"),
                                   targets.size, 3)
        assert bool(one["bad"][0]) == bool(batched["bad"][j])
        if batched["bad"][j]:
            continue
        for key in ("radii", "perim", "msd_u", "msd_w", "dist_b", "extra_r", "extra_a"):
            a, b = np.asarray(one[key][0], float), np.asarray(batched[key][j], float)
            ok = np.isfinite(b)
            assert np.array_equal(np.isfinite(a), ok), key
            assert np.all(np.abs(a[ok] - b[ok]) <= 1e-10 * np.abs(b[ok])), key


@pytest.mark.parametrize("level,jitter,robust", [(5, 0.2, True), (8, 0.2, False)])
def test_dropin_matches_batched_on_other_meshes(level, jitter, robust):
    """The drop-in chain on the robust (intrinsic Delaunay) operators and on the L8 mesh (59
    etree levels, the deepest measured), against the batched FP64 path of the same engine."""
    m = folded_icosphere(level, seed=1, jitter=jitter)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    eng = engine.HeatEngine(pm.V, pm.F, robust=int(robust), block_k=64)
    try:
        picks = [int(x) for x in pm.bfs[np.linspace(0, pm.n_vertices - 1, 3).astype(int)]]
        batched = eng.compute_distances(np.asarray(picks, np.int32), precision="fp64")
        for j, s in enumerate(picks):
            d = eng.compute_distance(s)
            assert d[s] == 0.0
            assert _maxrel(d, batched[j]) <= 1e-12, (level, s, _maxrel(d, batched[j]))
    finally:
        eng.close()
