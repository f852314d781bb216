"""ShardedWiringAnalysis on two gloo ranks (CPU): each rank computes the records of its slice
of the BFS sources, the records are gathered in rank order, and both ranks end with arrays
identical to a one-process run on the same records.

The engine is replaced by a stand-in whose records and samples are functions of the source
index (the sharding and the gather are under test here, not the solver, which the GPU tests
cover); it also reports which sources each rank computed."""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np

from fastcorticalwiring_b200 import _lib
from fastcorticalwiring_b200.meshgen import folded_icosphere

SCALES = (0.001, 0.004, 0.016)


class _StandInEngine:
    def __init__(self):
        self.seen = []

    def compute_metrics(self, sources, targets, n_between=3, eps=1e-6, precision="mixed"):
        src = np.asarray(sources, dtype=np.float64)
        self.seen.extend(np.asarray(sources).tolist())
        nt = len(targets)
        rec = np.zeros((src.size, _lib.metrics_stride(nt, n_between)))
        rec[:, 0], rec[:, 1], rec[:, 2] = src * 0.5, src * 0.25, src + 1.0
        rec[:, 5] = (np.asarray(sources) % 17 == 0).astype(float)  # some flagged fields
        for i in range(nt):
            rec[:, 7 + i] = src + i
            rec[:, 7 + nt + i] = 2.0 * src + i
        return rec

    def assemble_samples(self, records, targets, n_between=3, boundary_cap=None):
        n = records.shape[0]
        cap = _lib.samples_capacity(len(targets), n_between)
        counts = (records[:, 2].astype(np.int64) % 5).astype(np.int32)
        radii = np.tile(np.arange(cap, dtype=np.float32), (n, 1)) + records[:, 2:3].astype(np.float32)
        return radii, 2.0 * radii, counts


class _StandInDistanceEngine:
    def __init__(self, vertices, faces, **kw):
        self.engine = _StandInEngine()


def _mesh():
    m = folded_icosphere(3, seed=2, jitter=0.1)
    return m.vertices, m.faces, m.cortex_mask


def _arrays(a):
    out = {"msd_u": a.msd_unweighted, "msd_w": a.msd_weighted, "dist_b": a.dist_to_boundary,
           "flag": a.field_flag, "indptr": a.sample_indptr, "radii": a.sample_radii_flat, "areas": a.sample_areas_flat}
    for s in SCALES:
        out[f"r{s}"] = a.radius_function[s]
        out[f"p{s}"] = a.perimeter_function[s]
    return out


def _run(subset=None):
    import warnings

    from fastcorticalwiring_b200 import analysis, sharded

    analysis.B200DistanceEngine = _StandInDistanceEngine
    a = sharded.ShardedWiringAnalysis(*_mesh())
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)  # the stand-in flags some fields
        a.compute_all_wiring_costs(scale=list(SCALES), n_samples_between_scales=2, vertex_subset=subset)
    return _arrays(a), a.distance_engine.engine.seen


def _subset():
    """Every third original vertex (the reference's vertex_subset, core_analysis.py:1519-1533)."""
    m = _mesh()
    return list(range(0, m[0].shape[0], 3))


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        arrays, seen = _run()
        sub_arrays, sub_seen = _run(_subset())
        q.put((rank, arrays, seen, sub_arrays, sub_seen))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_match_one_process():
    from fastcorticalwiring_b200 import mesh as M, sharded

    one, seen_one = _run()
    sub_one, _ = _run(_subset())
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=180) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every source computed once, each rank its contiguous slice of the BFS order
    order = M.prepare(*_mesh()).bfs
    assert np.array_equal(np.concatenate([np.asarray(g[2]) for g in got]), order)
    assert np.array_equal(np.asarray(seen_one), order)
    for r, g in enumerate(got):
        assert np.array_equal(np.asarray(g[2]), sharded.shard(order, world, r))
    for g in got:
        for k, v in one.items():
            assert np.array_equal(g[1][k], v, equal_nan=True), k
        for k, v in sub_one.items():  # a vertex subset shards the same way
            assert np.array_equal(g[3][k], v, equal_nan=True), k
    assert sum(len(g[4]) for g in got) < order.size  # only the subset's sources were computed


def test_shard_slices():
    from fastcorticalwiring_b200 import sharded

    order = np.arange(10)
    parts = [sharded.shard(order, 3, r) for r in range(3)]
    assert [p.tolist() for p in parts] == [[0, 1, 2, 3], [4, 5, 6], [7, 8, 9]]
    assert np.array_equal(sharded.gather_rows(np.ones((2, 3))), np.ones((2, 3)))  # no process group
    import pytest

    with pytest.raises(ValueError):
        sharded.shard(order, 2, 2)


def test_run_returns_the_reference_tuple_and_prints_its_report(capsys):
    """compute_all_wiring_costs returns ((msd_unweighted, msd_weighted), radius_function,
    perimeter_function) and prints the end-of-run report, as core_analysis.py:1634-1672 does;
    verbose prints one line per block of sources."""
    import warnings

    from fastcorticalwiring_b200 import analysis

    analysis.B200DistanceEngine = _StandInDistanceEngine
    a = analysis.WiringAnalysis(*_mesh(), block_sources=64)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        (msd_u, msd_w), radius, perim = a.compute_all_wiring_costs(scale=list(SCALES), n_samples_between_scales=2,
                                                                    verbose=True)
    assert msd_u is a.msd_unweighted and msd_w is a.msd_weighted
    assert radius is a.radius_function and perim is a.perimeter_function
    out = capsys.readouterr().out.splitlines()
    assert any(line.startswith("[64/") for line in out)
    assert any(line.startswith(f"WARNING: {a.n_flagged_fields} of ") for line in out)
    assert sum(line.startswith("  vertex ") for line in out) == min(10, a.n_flagged_fields)
    assert "MSD (unweighted, Ecker 2013 definition):" in out
    v = msd_u[np.isfinite(msd_u)]
    assert f"  min={v.min():.2f}, max={v.max():.2f}, mean={v.mean():.2f}" in out
    for s in SCALES:
        assert any(line.startswith(f"Radius stats @ {s * 100:.2f}%: min=") for line in out)
        assert any(line.startswith(f"Perimeter stats @ {s * 100:.2f}%: min=") for line in out)


def test_construction_reports_the_components(capsys):
    """The constructor prints the submesh's connected components (core_analysis.py:1349-1381)."""
    from fastcorticalwiring_b200 import analysis

    analysis.B200DistanceEngine = _StandInDistanceEngine
    a = folded_icosphere(3, seed=2, jitter=0.1)
    b = folded_icosphere(2, seed=4, jitter=0.0)
    V = np.vstack([a.vertices, 0.5 * b.vertices])
    F = np.vstack([a.faces, b.faces + len(a.vertices)])
    an = analysis.WiringAnalysis(V, F, np.concatenate([a.cortex_mask, b.cortex_mask]))
    out = capsys.readouterr().out.splitlines()
    assert "Connected components in cortical submesh: 2" in out
    sizes = an.component_sizes
    assert sizes.size == 2 and sizes.sum() == an.mesh.n_vertices
    assert f"Component sizes: {sizes[0]}, {sizes[1]}" in out
