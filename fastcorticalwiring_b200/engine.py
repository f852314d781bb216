"""The `b200` distance engine: Python face of libfcw_b200.so.

Two layers:

* `HeatEngine` -- a thin owner of one `fcw_engine*` (one cortical submesh on one
  GPU): single-source FP64 distances (the drop-in), batched distances, and the
  batched per-source metrics in FP64 or mixed precision.
* `B200DistanceEngine` -- the plug-in for FastCorticalWiring's engine registry,
  following the contract of `distance_engines.BaseDistanceEngine`
  (distance_engines.py:54-69) and the keyword rules of
  `PotpourriDistanceEngine` (distance_engines.py:75-125).

There is no CPU path: without the library or a GPU, construction raises.
"""

from __future__ import annotations

import ctypes
import warnings
from abc import ABC, abstractmethod

import numpy as np

from . import _lib

DEFAULT_DIFFUSION_LENGTH_MM = 0.7          # distance_engines.py:12
MIN_DIFFUSION_LENGTH_MM = 0.5              # distance_engines.py:13
RECOMMENDED_MIN_DIFFUSION_LENGTH_MM = 0.7  # distance_engines.py:14

ENGINE_DEFAULTS = dict(block_k=1024, leaf_size=64, max_width=64, relax=64, build_mixed=1, device=0, pipeline_depth=4,
                       tc_sweeps=0, robust=0, refine=0)


_PINNED = None


def _field_array(n: int) -> np.ndarray:
    """A new float64 array for one field, in page-locked host memory when CUDA is up, so the
    device copies into it at full speed (about 3x a copy into pageable memory, which the
    driver stages through a bounce buffer). The memory comes from torch's caching host
    allocator, which takes the block back when the array is freed and hands it out again,
    so a loop of single-source calls allocates nothing after its first calls."""
    global _PINNED
    if _PINNED is None:
        try:
            import torch

            _PINNED = bool(torch.cuda.is_available())
        except Exception:
            _PINNED = False
    if _PINNED:
        import torch

        return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    return np.empty(n, dtype=np.float64)


class HeatEngine:
    """One cortical submesh factored on one GPU."""

    def __init__(self, vertices, faces, diffusion_length_mm=DEFAULT_DIFFUSION_LENGTH_MM, poisson_shift=1e-10,
                 **params):
        lib = _lib.load()
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32)
        cfg = dict(ENGINE_DEFAULTS)
        cfg.update(params)
        p = _lib.default_params(diffusion_length_mm=float(diffusion_length_mm), poisson_shift=float(poisson_shift),
                                **cfg)
        self._params = p
        h = ctypes.c_void_p()
        _lib.check(lib.fcw_engine_create(_lib.ptr(self.vertices), self.vertices.shape[0], _lib.ptr(self.faces),
                                         self.faces.shape[0], ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.n_vertices = int(self.vertices.shape[0])
        self.block_k = int(p.block_k)

    # -- lifecycle -------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _lib.load().fcw_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("engine is closed")
        return self._h

    def info(self) -> dict:
        inf = _lib.FCWInfo()
        _lib.check(_lib.load().fcw_engine_info(self.handle, ctypes.byref(inf)))
        return inf.as_dict()

    # -- distances -------------------------------------------------------
    def compute_distance(self, source_idx: int) -> np.ndarray:
        out = _field_array(self.n_vertices)
        _lib.check(_lib.load().fcw_compute_distance(self.handle, int(source_idx), _lib.ptr(out)))
        return out

    def compute_distances(self, sources, precision="fp64") -> np.ndarray:
        src = np.ascontiguousarray(sources, dtype=np.int32).reshape(-1)
        out = np.empty((src.size, self.n_vertices), dtype=np.float64)
        _lib.check(_lib.load().fcw_compute_distances(self.handle, _lib.ptr(src), src.size, _precision(precision),
                                                     _lib.ptr(out)))
        return out

    # -- metrics ---------------------------------------------------------
    def compute_metrics(self, sources, targets, n_between=3, eps=1e-6, precision="mixed") -> np.ndarray:
        """Raw per-source records (n, stride), see include/fcw_b200.h FCW_M_*."""
        src = np.ascontiguousarray(sources, dtype=np.int32).reshape(-1)
        t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
        stride = _lib.metrics_stride(t.size, n_between)
        out = np.empty((src.size, stride), dtype=np.float64)
        _lib.check(_lib.load().fcw_compute_metrics(self.handle, _lib.ptr(src), src.size, _precision(precision),
                                                   _lib.ptr(t), t.size, int(n_between), float(eps), _lib.ptr(out)))
        return out

    def compute_metrics_device(self, sources_dev, targets, n_between, eps, precision, out_dev, stream) -> None:
        """Device-resident form: sources_dev/out_dev are torch CUDA tensors (int32 / float64).

        out_dev holds one record of metrics_stride(len(targets), n_between) doubles per source."""
        t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
        import torch

        stride = _lib.metrics_stride(t.size, n_between)
        if sources_dev.dtype != torch.int32 or not sources_dev.is_contiguous():
            raise ValueError("sources_dev must be a contiguous int32 tensor")
        if out_dev.dtype != torch.float64 or not out_dev.is_contiguous():
            raise ValueError("out_dev must be a contiguous float64 tensor")
        if out_dev.numel() < sources_dev.numel() * stride:
            raise ValueError(f"out_dev holds {out_dev.numel()} doubles; {sources_dev.numel()} records of "
                             f"{stride} need {sources_dev.numel() * stride}")
        _lib.check(_lib.load().fcw_compute_metrics_device(
            self.handle, ctypes.c_void_p(sources_dev.data_ptr()), int(sources_dev.numel()), _precision(precision),
            _lib.ptr(t), t.size, int(n_between), float(eps), ctypes.c_void_p(out_dev.data_ptr()),
            ctypes.c_void_p(stream)))

    def assemble_samples(self, records, targets, n_between=3, boundary_cap=None):
        """Cleaned (radius, area) samples of metric records (core_analysis.py:1599-1611).

        Returns (radii, areas, counts): float32 rows of fcw_samples_capacity entries, of
        which counts[k] are used. boundary_cap: None, or the cap in [0, 0.5).
        """
        rec = np.ascontiguousarray(records, dtype=np.float64)
        t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
        n = rec.shape[0]
        cap = _lib.samples_capacity(t.size, n_between)
        radii = np.empty((n, cap), dtype=np.float32)
        areas = np.empty((n, cap), dtype=np.float32)
        counts = np.empty(n, dtype=np.int32)
        c = float("nan") if boundary_cap is None else float(boundary_cap)
        _lib.check(_lib.load().fcw_assemble_samples(self.handle, _lib.ptr(rec), n, t.size, int(n_between), _lib.ptr(t),
                                                    c, _lib.ptr(radii), _lib.ptr(areas), _lib.ptr(counts)))
        return radii, areas, counts

    def graphs(self, enable=True) -> None:
        """Replay each workspace's captured launch chain (the default) or launch blocks directly."""
        _lib.check(_lib.load().fcw_engine_graphs(self.handle, int(bool(enable))))

    def profile(self, enable=True) -> None:
        """Turn the per-stage CUDA-event timeline on/off (and reset it)."""
        _lib.check(_lib.load().fcw_engine_profile(self.handle, int(bool(enable))))

    def stage_times(self):
        """(dict stage -> ms accumulated since the last reset, kernels launched)."""
        ms = np.zeros(len(_lib.STAGES))
        n = ctypes.c_int64(0)
        _lib.check(_lib.load().fcw_engine_stage_times(self.handle, _lib.ptr(ms), ms.size, ctypes.byref(n)))
        return dict(zip(_lib.STAGES, ms.tolist())), int(n.value)

    def synchronize(self, stream=0) -> None:
        _lib.check(_lib.load().fcw_synchronize(self.handle, ctypes.c_void_p(stream)))


def _precision(p) -> int:
    if p in ("fp64", _lib.FCW_PREC_FP64):
        return _lib.FCW_PREC_FP64
    if p in ("mixed", _lib.FCW_PREC_MIXED):
        return _lib.FCW_PREC_MIXED
    raise ValueError(f"precision must be 'fp64' or 'mixed', got {p!r}")


def assemble_samples_device(records, targets, n_between=3, boundary_cap=None, device=0):
    """fcw_assemble_samples_device on host records, without an engine: the records go to
    `device`, the (radii, areas, counts) rows come back (as HeatEngine.assemble_samples)."""
    import torch

    rec = np.ascontiguousarray(records, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
    n = rec.shape[0]
    cap = _lib.samples_capacity(t.size, n_between)
    if n == 0:
        return (np.empty((0, cap), np.float32), np.empty((0, cap), np.float32), np.empty(0, np.int32))
    dev = f"cuda:{int(device)}"
    with torch.cuda.device(dev):
        rec_d = torch.from_numpy(rec).to(dev)
        radii = torch.empty((n, cap), dtype=torch.float32, device=dev)
        areas = torch.empty((n, cap), dtype=torch.float32, device=dev)
        counts = torch.empty(n, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream()
        c = float("nan") if boundary_cap is None else float(boundary_cap)
        _lib.check(_lib.load().fcw_assemble_samples_device(
            ctypes.c_void_p(rec_d.data_ptr()), n, t.size, int(n_between), _lib.ptr(t), c,
            ctypes.c_void_p(radii.data_ptr()), ctypes.c_void_p(areas.data_ptr()), ctypes.c_void_p(counts.data_ptr()),
            ctypes.c_void_p(stream.cuda_stream)))
        stream.synchronize()
        return radii.cpu().numpy(), areas.cpu().numpy(), counts.cpu().numpy()


def split_records(rec: np.ndarray, n_targets: int, n_between: int) -> dict:
    """Named views of raw records (n, stride)."""
    ne = max(0, n_targets - 1) * n_between
    r0 = _lib.M_RADII
    return dict(
        msd_u=rec[:, _lib.M_MSD_U], msd_w=rec[:, _lib.M_MSD_W], dist_b=rec[:, _lib.M_DIST_B],
        neg=rec[:, _lib.M_NEG], viol=rec[:, _lib.M_VIOL], bad=rec[:, _lib.M_BAD] != 0.0,
        n_eval=rec[:, _lib.M_NEVAL].astype(np.int64),
        radii=rec[:, r0:r0 + n_targets], perim=rec[:, r0 + n_targets:r0 + 2 * n_targets],
        extra_r=rec[:, r0 + 2 * n_targets:r0 + 2 * n_targets + ne],
        extra_a=rec[:, r0 + 2 * n_targets + ne:r0 + 2 * n_targets + 2 * ne],
    )


# ---------------------------------------------------------------------------
# Plug-in for FastCorticalWiring's distance-engine registry
# ---------------------------------------------------------------------------
class BaseDistanceEngine(ABC):
    """The engine contract of distance_engines.py:54-69."""

    def __init__(self, vertices, faces, **engine_kwargs):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32)
        self.engine_kwargs = dict(engine_kwargs or {})

    @property
    @abstractmethod
    def name(self) -> str:
        raise NotImplementedError

    @abstractmethod
    def compute_distance(self, source_idx: int) -> np.ndarray:
        raise NotImplementedError


class B200DistanceEngine(BaseDistanceEngine):
    """Heat-method distances on a B200, one source per call (FP64).

    Keyword rules follow PotpourriDistanceEngine (distance_engines.py:75-125):
    `diffusion_length_mm` (default 0.7) must be finite and >= 0.5 (ValueError),
    values below 0.7 warn (RuntimeWarning); `t_coef` is rejected.
    `allow_eigen_fallback` is accepted and ignored (there is no SuiteSparse
    backend to check). Other keys are engine tunables (block_k, leaf_size,
    max_width, relax, build_mixed, device, pipeline_depth, tc_sweeps).

    `use_robust` picks the operators. False (the default): the consistent
    extrinsic cotan Laplacian L = G^T diag(A) G and barycentric lumped mass of
    fastcw_lean.py:394-413, the method the engine is checked against. True: the
    cotan Laplacian and lumped mass of the intrinsic Delaunay triangulation, as
    the production potpourri3d engine uses (distance_engines.py:119-125); the
    normalised gradient and its divergence stay on the mesh's faces.
    """

    def __init__(self, vertices, faces, **engine_kwargs):
        super().__init__(vertices, faces, **engine_kwargs)
        kw = dict(self.engine_kwargs)
        kw.pop("allow_eigen_fallback", None)
        robust = bool(kw.pop("use_robust", False))
        if "t_coef" in kw:
            raise ValueError("Set diffusion_length_mm instead of t_coef.")
        L = float(kw.pop("diffusion_length_mm", DEFAULT_DIFFUSION_LENGTH_MM))
        if not np.isfinite(L) or L < MIN_DIFFUSION_LENGTH_MM:
            raise ValueError(f"diffusion_length_mm must be finite and at least {MIN_DIFFUSION_LENGTH_MM} mm.")
        if L < RECOMMENDED_MIN_DIFFUSION_LENGTH_MM:
            warnings.warn(f"diffusion_length_mm={L} is below the validated {RECOMMENDED_MIN_DIFFUSION_LENGTH_MM} mm.",
                          RuntimeWarning)
        unknown = set(kw) - set(ENGINE_DEFAULTS) - {"poisson_shift"} - {"robust"}
        if unknown:
            raise ValueError(f"Unsupported engine kwargs for b200 engine: {', '.join(sorted(unknown))}")
        kw["robust"] = int(robust)
        self._engine = HeatEngine(self.vertices, self.faces, diffusion_length_mm=L, **kw)
        info = self._engine.info()
        self.use_robust = robust
        self.n_flips = int(info["n_flips"])
        self.n_components = int(info["n_components"])  # connected components of the submesh
        self.diffusion_length_mm = L
        self.mean_edge_length = float(info["mean_edge_length"])
        self.t_coef = float(info["t_coef"])
        self.precision = "fp64"
        self.block_k = self._engine.block_k

    @property
    def name(self) -> str:
        return "b200"

    @property
    def engine(self) -> HeatEngine:
        return self._engine

    def compute_distance(self, source_idx: int) -> np.ndarray:
        src = int(source_idx)
        n = self.vertices.shape[0]
        if src < 0 or src >= n:
            raise ValueError(f"source_idx out of range: {src} for mesh with {n} vertices")
        return np.ascontiguousarray(self._engine.compute_distance(src))

    def compute_all_metrics(self, sources, targets, n_between=3, eps=1e-6, precision="mixed") -> dict:
        """Batched per-source metrics (the arrays core_analysis.compute_all_wiring_costs fills)."""
        t = np.asarray(targets, dtype=np.float64)
        rec = self._engine.compute_metrics(sources, t, n_between=n_between, eps=eps, precision=precision)
        return split_records(rec, t.size, n_between)


ENGINE_REGISTRY = {"b200": B200DistanceEngine}


def create_distance_engine(engine_type, vertices, faces, engine_kwargs=None):
    """Registry lookup with the reference's behaviour (distance_engines.py:265-273)."""
    key = str(engine_type).strip().lower()
    if key not in ENGINE_REGISTRY:
        valid = ", ".join(sorted(ENGINE_REGISTRY.keys()))
        raise ValueError(f"Unknown engine_type '{engine_type}'. Valid options: {valid}")
    return ENGINE_REGISTRY[key](vertices, faces, **dict(engine_kwargs or {}))


def engine_class(base=None):
    """B200DistanceEngine, or a subclass of it that is also a subclass of `base` (the host
    application's own engine ABC, e.g. distance_engines.BaseDistanceEngine), so isinstance
    checks against the host's contract hold."""
    if base is None or issubclass(B200DistanceEngine, base):
        return B200DistanceEngine
    return type("B200DistanceEngine", (B200DistanceEngine, base),
                {"__module__": __name__, "__doc__": B200DistanceEngine.__doc__})


def register(registry: dict, base=None) -> None:
    """Add the b200 engine to another registry (e.g. distance_engines.ENGINE_REGISTRY), as a
    subclass of `base` when given (e.g. distance_engines.BaseDistanceEngine)."""
    registry["b200"] = engine_class(base)
