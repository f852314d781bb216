"""Faults injected on the host (needs a B200): corrupt distance fields reach the device metrics
kernels through fcw_field_metrics_device, and the health screen must flag them and NaN their
geometry while healthy neighbours in the same block are unaffected.

Mirrors the reference's acceptance check (verify_lean_integration.py:191-211), which
monkeypatches the solver to truncate one field (min(d, 0.2 max d), "like the non-robust
failures") and expects it flagged, NaN'd and its neighbours untouched; plus a field with a
NaN and one whose values are perturbed at 2% of the vertices (the non-Lipschitz field of
test_fastcw_lean.py:46-49). Nothing here faults the GPU: the bad values are data.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import _lib, engine, mesh as M  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402


def _field_metrics(eng, fields, sources, targets, n_between=3):
    import torch

    d = torch.tensor(np.ascontiguousarray(fields), dtype=torch.float64, device="cuda")
    src = torch.tensor(np.asarray(sources, np.int32), device="cuda")
    t = np.ascontiguousarray(targets, dtype=np.float64)
    stride = _lib.metrics_stride(t.size, n_between)
    out = torch.full((src.numel(), stride), float("nan"), dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().fcw_field_metrics_device(eng.handle, d.data_ptr(), src.data_ptr(), src.numel(),
                                                    _lib.ptr(t), t.size, n_between, 1e-6, out.data_ptr(), None))
    eng.synchronize(0)
    return engine.split_records(out.cpu().numpy(), t.size, n_between)


def test_corrupted_fields_are_flagged_and_neighbours_unaffected():
    import oracle

    m = folded_icosphere(4, seed=7, jitter=0.0)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    src = pm.bfs[np.linspace(0, pm.n_vertices - 1, 6).astype(int)]
    phi = oracle.HeatOracle(pm.V, pm.F).distances(src)
    targets = pm.targets(M.RUNNER_SCALES)
    eng = engine.HeatEngine(pm.V, pm.F, block_k=64)
    try:
        clean = _field_metrics(eng, phi, src, targets)
        assert not clean["bad"].any()
        bad = phi.copy()
        bad[1] = np.minimum(bad[1], 0.2 * np.nanmax(bad[1]))     # truncated (verify_lean_integration.py:199)
        bad[3, pm.n_vertices // 2] = np.nan                       # a non-finite value
        rng = np.random.default_rng(0)
        idx = rng.choice(pm.n_vertices, size=max(1, pm.n_vertices // 50), replace=False)
        bad[4, idx] *= 0.5                                         # non-Lipschitz at 2% of the vertices
        r = _field_metrics(eng, bad, src, targets)
    finally:
        eng.close()
    for j in (1, 3, 4):
        ref = oracle.field_health(bad[j], pm.V, src[j], pm.health_h)
        assert ref[2] and bool(r["bad"][j]), j
        # a flagged record has no geometry; the analysis layer also blanks its MSD and boundary
        # distance (core_analysis.py:1559-1564), the record keeps them for diagnosis
        assert np.all(np.isnan(r["radii"][j])) and np.all(np.isnan(r["perim"][j]))
        assert np.all(np.isnan(r["extra_r"][j])) and np.all(np.isnan(r["extra_a"][j]))
    for j in (0, 2, 5):  # healthy neighbours in the same call: the records of the clean run (to the
        assert not r["bad"][j]  # order of the band sums, which atomics set)
        assert np.max(np.abs(r["radii"][j] - clean["radii"][j]) / clean["radii"][j]) <= 1e-12
        assert abs(r["msd_w"][j] - clean["msd_w"][j]) <= 1e-12 * clean["msd_w"][j]
