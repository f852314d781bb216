"""C-ABI surface and host-side logic, no GPU needed."""
import ctypes
import os
import re

import numpy as np
import pytest

from fastcorticalwiring_b200 import _lib, engine, mesh as M
from tests.conftest import GOLDEN, ROOT


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "fcw_b200.h")).read()
    return set(re.findall(r"^\s*(?:int|void)\s+(fcw_\w+)\s*\(", text, flags=re.M))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared_symbols()
    assert declared == set(_lib.EXPORTED)
    for name in declared:
        assert getattr(lib, name) is not None


def test_params_struct_matches_defaults():
    p = _lib.default_params()
    assert p.diffusion_length_mm == 0.7 and p.poisson_shift == 1e-10
    assert p.block_k % 64 == 0 and 1 <= p.relax <= p.max_width <= 64
    assert _lib.metrics_stride(12, 3) == 7 + 24 + 66


def _l4():
    z = np.load(os.path.join(GOLDEN, "golden_heat_L4.npz"))
    return z, M.prepare(z["V"], z["F"], z["mask"])


def test_native_mesh_arrays_match_reference_bit_exact():
    z, pm = _l4()
    arr = _lib.mesh_arrays(pm.V, pm.F)
    assert np.array_equal(arr["vertex_area"], z["vertex_area"])
    assert np.array_equal(arr["boundary"], z["boundary"])
    assert np.array_equal(arr["lean_area"], pm.lean_area)
    for g in ("g11", "g12", "g22"):
        assert np.array_equal(arr[g], getattr(pm, g))


def test_analysis_info_matches_reference_quantities():
    z, pm = _l4()
    info, perm = _lib.analyze(pm.V, pm.F)
    assert info["bin_width"] == float(z["bin_width"])
    assert info["health_h"] == float(z["health_h"])
    assert abs(info["t"] - float(z["t"])) <= 1e-15
    assert sorted(perm.tolist()) == list(range(pm.n_vertices))
    assert info["max_ns"] <= 64


def test_quantile_matches_numpy_on_random_meshes():
    rng = np.random.default_rng(4)
    for level in (2, 3):
        from fastcorticalwiring_b200.meshgen import folded_icosphere
        m = folded_icosphere(level, seed=int(rng.integers(100)), jitter=0.2)
        pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
        info, _ = _lib.analyze(pm.V, pm.F)
        assert info["bin_width"] == pm.bin_width
        assert info["health_h"] == pm.health_h


@pytest.mark.parametrize("level", [3, 4, 5])
def test_symbolic_structure_contains_true_fill(level):
    """Every nonzero of the exact Cholesky factor lies inside the supernodal structure."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import splu
    import oracle
    from fastcorticalwiring_b200.meshgen import folded_icosphere
    m = folded_icosphere(level, seed=level, jitter=0.2)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    info, perm = _lib.analyze(pm.V, pm.F)
    L, mass, *_ = oracle.operators(pm.V, pm.F)
    A = (sp.diags(mass) + 0.49 * L).tocsc()[perm][:, perm].tocsc()
    lu = splu(A, permc_spec="NATURAL", diag_pivot_thresh=0.0, options=dict(SymmetricMode=True))
    assert np.array_equal(lu.perm_c, np.arange(A.shape[0]))      # no reordering happened
    assert lu.L.nnz <= info["nnz_l"]


def test_engine_kwarg_rules_follow_potpourri_engine():
    z, pm = _l4()
    for bad in ({"t_coef": 1.0}, {"diffusion_length_mm": 0.4},
                {"diffusion_length_mm": float("nan")}, {"not_a_setting": 1}):
        with pytest.raises(ValueError):
            engine.B200DistanceEngine(pm.V, pm.F, **bad)


def test_unknown_engine_name_is_rejected():
    with pytest.raises(ValueError, match="Unknown engine_type 'batch_heat'"):
        engine.create_distance_engine("batch_heat", np.zeros((3, 3)), np.array([[0, 1, 2]]))
    assert not hasattr(engine.BaseDistanceEngine, "compute_distance_batch")


def test_no_cpu_fallback_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    z, pm = _l4()
    with pytest.raises(_lib.FCWError) as ei:
        engine.HeatEngine(pm.V, pm.F)
    assert ei.value.code == _lib.FCW_E_NODEVICE


def test_invalid_mesh_is_rejected_at_the_boundary():
    V = np.zeros((3, 3))
    with pytest.raises(_lib.FCWError) as ei:
        _lib.analyze(V, np.array([[0, 1, 5]], dtype=np.int32))
    assert ei.value.code == _lib.FCW_E_INVALID and "out of range" in str(ei.value)


def test_record_layout_matches_the_header():
    """fcw_metrics_stride and the FCW_M_* offsets: 7 scalars, radii, perimeters, then the samples."""
    for nt, nb in ((1, 0), (12, 3), (32, 8)):
        ne = (nt - 1) * nb
        stride = _lib.metrics_stride(nt, nb)
        assert stride == 7 + 2 * nt + 2 * ne
        rec = np.arange(2 * stride, dtype=np.float64).reshape(2, stride)
        r = engine.split_records(rec, nt, nb)
        assert r["msd_u"][1] == stride + _lib.M_MSD_U and r["dist_b"][0] == _lib.M_DIST_B
        assert r["radii"].shape == (2, nt) and r["radii"][0, 0] == _lib.M_RADII
        assert r["perim"][0, 0] == _lib.M_RADII + nt
        assert r["extra_r"].shape == (2, ne) and r["extra_a"].shape == (2, ne)
        if ne:
            assert r["extra_a"][0, -1] == stride - 1
    assert _lib.samples_capacity(32, 8) == 32 + 31 * 8


def test_registered_engine_subclasses_the_host_contract():
    """register(registry, base) installs a class that is also a subclass of the host's own engine ABC
    (distance_engines.BaseDistanceEngine in the reference), so isinstance checks there hold."""
    from abc import ABC, abstractmethod

    class HostBase(ABC):  # the shape of distance_engines.py:54-69
        def __init__(self, vertices, faces, **engine_kwargs):
            self.engine_kwargs = dict(engine_kwargs)

        @property
        @abstractmethod
        def name(self):
            raise NotImplementedError

        @abstractmethod
        def compute_distance(self, source_idx):
            raise NotImplementedError

    reg = {}
    engine.register(reg, base=HostBase)
    cls = reg["b200"]
    assert issubclass(cls, HostBase) and issubclass(cls, engine.B200DistanceEngine)
    assert engine.engine_class() is engine.B200DistanceEngine
    z, pm = _l4()
    with pytest.raises(_lib.FCWError):  # no device here: construction reaches the engine and fails loudly
        cls(pm.V, pm.F)


def test_refine_steps_are_validated():
    """fcw_params.refine (iterative-refinement steps of the mixed Poisson solve) is checked on
    the host: 0-4 are accepted, other values are FCW_E_INVALID."""
    from fastcorticalwiring_b200 import _lib
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    m = folded_icosphere(2, seed=0, jitter=0.0)
    _lib.analyze(m.vertices, m.faces, refine=2)
    for bad in (-1, 5):
        with pytest.raises(_lib.FCWError):
            _lib.analyze(m.vertices, m.faces, refine=bad)


def test_component_count_matches_scipy():
    """fcw_info.n_components counts the submesh's connected components as the reference's
    diagnostic does (core_analysis.py:1349-1381); the engine grounds one vertex of each."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components

    from fastcorticalwiring_b200.meshgen import folded_icosphere

    a = folded_icosphere(3, seed=1, jitter=0.1)
    b = folded_icosphere(2, seed=2, jitter=0.1)
    c = folded_icosphere(2, seed=3, jitter=0.0)
    parts = [a, b, c]
    for k in (1, 2, 3):
        V = np.vstack([p.vertices * (1.0 - 0.2 * i) for i, p in enumerate(parts[:k])])
        offs = np.cumsum([0] + [len(p.vertices) for p in parts[:k]])
        F = np.vstack([p.faces + offs[i] for i, p in enumerate(parts[:k])])
        pm = M.prepare(V, F, np.concatenate([p.cortex_mask for p in parts[:k]]))
        n = pm.n_vertices
        G = sp.coo_matrix((np.ones(pm.F.size), (pm.F.ravel(), pm.F[:, [1, 2, 0]].ravel())), shape=(n, n))
        info, _ = _lib.analyze(pm.V, pm.F)
        assert info["n_components"] == connected_components(G, directed=False)[0] == k
        # the intrinsic edge flips stay inside a component
        assert _lib.analyze(pm.V, pm.F, robust=1)[0]["n_components"] == k


def test_elimination_order_is_deterministic():
    """The nested dissection runs the halves of its top splits on separate threads; the order
    (and so the factor's structure) must not depend on their timing."""
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    m = folded_icosphere(6, seed=3, jitter=0.2)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    info0, perm0 = _lib.analyze(pm.V, pm.F)
    assert sorted(perm0.tolist()) == list(range(pm.n_vertices))
    for _ in range(4):
        info, perm = _lib.analyze(pm.V, pm.F)
        assert np.array_equal(perm, perm0)
        assert info["nnz_factor"] == info0["nnz_factor"] and info["n_supernodes"] == info0["n_supernodes"]
