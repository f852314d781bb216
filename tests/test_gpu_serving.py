"""The serving loop (needs a B200): each job's results are the same alone and in a mix.

Four hemisphere jobs of different sizes (three order-4 meshes and one order-5
mesh, each with its own folding seed) run one at a time, then together through
a server whose HBM budget is below the four jobs' sum, so later jobs wait for
memory and then overlap with the running ones. Every job's records must
agree with its solo run to 1e-9 relative (the same kernels on the same inputs;
only the order of atomically appended faces inside a distance bin differs).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import serving  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402


def _jobs():
    out = []
    for i, (level, seed) in enumerate([(4, 1), (5, 9), (4, 2), (4, 3)]):
        m = folded_icosphere(level, seed=seed, jitter=0.2)
        out.append(serving.Job(f"job{i}", m.vertices, m.faces, m.cortex_mask, precision="mixed"))
    return out


def _same(a, b):
    assert a.shape == b.shape
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    d = np.abs(a[~na] - b[~nb])
    assert np.all(d <= 1e-9 * np.maximum(np.abs(b[~nb]), 1e-12))


def test_results_alone_and_in_the_mix():
    jobs = _jobs()
    alone = {}
    for j in jobs:
        srv = serving.Server(hbm_budget_bytes=100e9, engine_params=dict(block_k=256))
        try:
            alone[j.job_id] = srv.run([(0.0, j)])[j.job_id]
        finally:
            srv.close()
    # a budget below the four jobs' sum: some of them queue for memory
    est = [serving.estimate_device_bytes(int(j.cortex_mask.sum()), 2 * int(j.cortex_mask.sum()), 256, 2,
                                         int(j.cortex_mask.sum()), 97) for j in jobs]
    budget = sum(est) - min(est) // 2
    srv = serving.Server(hbm_budget_bytes=budget, engine_params=dict(block_k=256))
    try:
        mix = srv.run([(0.002 * i, j) for i, j in enumerate(jobs)])
    finally:
        srv.close()
    assert sorted(mix) == sorted(alone)
    for k in alone:
        assert np.array_equal(mix[k].sources, alone[k].sources)
        _same(mix[k].records, alone[k].records)
        assert mix[k].latency_s > 0
    # admission kept the resident jobs' estimates within the budget, and not all four ran at once
    res = list(mix.values())
    for r in res:
        resident = [q for q in res if q.t_admit <= r.t_admit < q.t_done]
        assert sum(q.estimate_bytes for q in resident) <= budget
        assert len(resident) < 4
    s = serving.latency_summary(mix)
    assert s["jobs"] == 4 and s["p50_s"] <= s["p99_s"]
