"""fcw_field_metrics_static: the allocation-free field-metrics entry point (needs a B200).

Some callers cannot allocate device memory while they run (a host that owns the
whole device through its own pool, or a fixed-footprint measurement loop). The
static entry point computes the same records as fcw_field_metrics_device from
the same fields, with its scratch in an array compiled into the library. This
file is collected last so a failure here leaves every other test already run.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import _lib, engine, mesh as M  # noqa: E402
from tests.conftest import GOLDEN  # noqa: E402


def _call(fn, eng, fields, sources, targets, n_between=3):
    import torch
    d = torch.tensor(np.ascontiguousarray(fields), dtype=torch.float64, device="cuda")
    src = torch.tensor(sources, dtype=torch.int32, device="cuda")
    t = np.ascontiguousarray(targets, dtype=np.float64)
    stride = _lib.metrics_stride(t.size, n_between)
    out = torch.full((src.numel(), stride), float("nan"), dtype=torch.float64, device="cuda")
    _lib.check(fn(eng.handle, d.data_ptr(), src.data_ptr(), src.numel(), _lib.ptr(t), t.size, n_between, 1e-6,
                  out.data_ptr(), None))
    eng.synchronize(0)
    return out.cpu().numpy()


def test_static_entry_matches_allocating_entry_on_consecutive_calls():
    z = dict(np.load(os.path.join(GOLDEN, "golden_heat_L4.npz")))
    pm = M.prepare(z["V"], z["F"], z["mask"])
    eng = engine.HeatEngine(pm.V, pm.F)
    lib = _lib.load()
    try:
        ref = _call(lib.fcw_field_metrics_device, eng, z["phi"], z["sources_sub"], z["targets"])
        for _ in range(2):  # the shared scratch keeps the previous call's contents
            got = _call(lib.fcw_field_metrics_static, eng, z["phi"], z["sources_sub"], z["targets"])
            both_nan = np.isnan(got) & np.isnan(ref)
            rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
            assert np.all(both_nan | (rel <= 1e-12)), np.nanmax(np.where(both_nan, 0.0, rel))
        # a different, smaller batch afterwards still agrees (no stale state leaks in)
        part = _call(lib.fcw_field_metrics_static, eng, z["phi"][:3], z["sources_sub"][:3], z["targets"])
        rel = np.abs(part - ref[:3]) / np.maximum(np.abs(ref[:3]), 1e-300)
        assert np.all(np.isnan(part) & np.isnan(ref[:3]) | (rel <= 1e-12))
        # more fields than the static scratch takes is refused, not truncated
        with pytest.raises(_lib.FCWError) as ei:
            _call(lib.fcw_field_metrics_static, eng, np.repeat(z["phi"][:1], 33, axis=0),
                  np.repeat(z["sources_sub"][:1], 33), z["targets"])
        assert ei.value.code == _lib.FCW_E_INVALID and "at most 32 fields" in str(ei.value)
    finally:
        eng.close()


def test_static_entry_first_on_a_fresh_engine_matches_the_reference_and_allocates_nothing():
    """Called first on a fresh engine (no allocating metrics call before it), the static entry
    point reproduces the reference's own geometry on the reference's fields; a repeated call
    leaves both the device's free memory and the engine's device-byte count unchanged; and a
    source index outside the mesh is reported by the next fcw_synchronize, as for the other
    stream entry points."""
    import torch

    z = dict(np.load(os.path.join(GOLDEN, "golden_heat_L4.npz")))
    pm = M.prepare(z["V"], z["F"], z["mask"])
    eng = engine.HeatEngine(pm.V, pm.F)
    lib = _lib.load()
    try:
        t = np.ascontiguousarray(z["targets"], dtype=np.float64)
        stride = _lib.metrics_stride(t.size, 3)
        d = torch.tensor(np.ascontiguousarray(z["phi"]), dtype=torch.float64, device="cuda")
        src = torch.tensor(z["sources_sub"], dtype=torch.int32, device="cuda")
        out = torch.full((src.numel(), stride), float("nan"), dtype=torch.float64, device="cuda")

        def run(sources=src):
            _lib.check(lib.fcw_field_metrics_static(eng.handle, d.data_ptr(), sources.data_ptr(), sources.numel(),
                                                    _lib.ptr(t), t.size, 3, 1e-6, out.data_ptr(), None))
            eng.synchronize(0)
            return out.cpu().numpy()

        bytes0 = eng.info()["device_bytes"]
        r = engine.split_records(run(), t.size, 3)
        assert not r["bad"].any()
        for key in ("radii", "perim", "extra_r", "extra_a"):
            rel = np.abs(r[key] - z[key]) / np.maximum(np.abs(z[key]), 1e-300)
            assert np.max(rel) <= 1e-12, (key, np.max(rel))
        assert np.array_equal(np.float32(r["dist_b"]), z["f32_dist_to_boundary"])
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        run()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
        assert eng.info()["device_bytes"] == bytes0
        bad = torch.tensor([0, pm.n_vertices + 5], dtype=torch.int32, device="cuda")
        with pytest.raises(_lib.FCWError) as ei:
            run(bad)
        assert ei.value.code == _lib.FCW_E_INVALID and "source index" in str(ei.value)
        # the error word is cleared once reported: the next call succeeds (same records to the
        # band-sum order, which atomics set)
        r2 = engine.split_records(run(), t.size, 3)
        assert np.max(np.abs(r2["radii"] - r["radii"]) / r["radii"]) <= 1e-12
    finally:
        eng.close()
