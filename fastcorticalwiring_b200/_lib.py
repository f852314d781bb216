"""ctypes binding of libfcw_b200.so (declarations in include/fcw_b200.h).

The library is built in-tree by fastcorticalwiring_b200.build. Loading never
falls back to anything: a missing or unloadable library raises ImportError,
and a missing GPU surfaces as FCWError(FCW_E_NODEVICE) from engine creation.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libfcw_b200.so")

FCW_OK, FCW_E_INVALID, FCW_E_CUDA, FCW_E_NOMEM, FCW_E_NUMERIC, FCW_E_TIMEOUT, FCW_E_NODEVICE = range(7)
FCW_PREC_FP64, FCW_PREC_MIXED = 0, 1
M_MSD_U, M_MSD_W, M_DIST_B, M_NEG, M_VIOL, M_BAD, M_NEVAL, M_RADII = range(8)

# Every symbol include/fcw_b200.h declares.
EXPORTED = (
    "fcw_default_params", "fcw_metrics_stride", "fcw_last_error", "fcw_analyze", "fcw_mesh_arrays",
    "fcw_engine_create", "fcw_engine_info", "fcw_engine_destroy", "fcw_compute_distance",
    "fcw_compute_distances", "fcw_compute_metrics", "fcw_compute_metrics_device", "fcw_synchronize",
    "fcw_heat_solve_device", "fcw_divergence_device", "fcw_poisson_solve_device", "fcw_field_metrics_device",
    "fcw_engine_profile", "fcw_engine_graphs", "fcw_engine_stage_times", "fcw_field_metrics_static",
    "fcw_samples_capacity", "fcw_assemble_samples_device", "fcw_assemble_samples", "fcw_tc_product_check",
    "fcw_intrinsic_operators",
)
STAGES = ("heat_fwd", "heat_bwd", "divergence", "poisson_fwd", "poisson_bwd", "shift", "metrics")


class FCWParams(ctypes.Structure):
    _fields_ = [
        ("diffusion_length_mm", ctypes.c_double),
        ("poisson_shift", ctypes.c_double),
        ("block_k", ctypes.c_int32),
        ("leaf_size", ctypes.c_int32),
        ("max_width", ctypes.c_int32),
        ("relax", ctypes.c_int32),
        ("build_mixed", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("pipeline_depth", ctypes.c_int32),
        ("tc_sweeps", ctypes.c_int32),
        ("robust", ctypes.c_int32),
        ("refine", ctypes.c_int32),
    ]


class FCWInfo(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int64), ("n_faces", ctypes.c_int64), ("n_boundary", ctypes.c_int64),
        ("n_supernodes", ctypes.c_int64), ("n_levels", ctypes.c_int64), ("nnz_factor", ctypes.c_int64),
        ("nnz_l", ctypes.c_int64),
        ("max_ns", ctypes.c_int32), ("max_m", ctypes.c_int32),
        ("mean_edge_length", ctypes.c_double), ("t_coef", ctypes.c_double), ("t", ctypes.c_double),
        ("bin_width", ctypes.c_double), ("health_h", ctypes.c_double), ("total_vertex_area", ctypes.c_double),
        ("analyze_ms", ctypes.c_double), ("factor_ms", ctypes.c_double), ("flops_factor", ctypes.c_double),
        ("device_bytes", ctypes.c_int64),
        ("pipeline_depth", ctypes.c_int32), ("block_k", ctypes.c_int32),
        ("n_flips", ctypes.c_int64), ("n_components", ctypes.c_int64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class FCWError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"[fcw error {code}] {message}")
        self.code = code


_lib = None


def load():
    """Load the library (once). Raises ImportError if it is missing or broken."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fastcorticalwiring_b200.build`")
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as exc:
        raise ImportError(f"cannot load {LIB_PATH}: {exc}") from exc
    P, I32, I64, D, V = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, None
    sig = {
        "fcw_default_params": (V, [P]),
        "fcw_metrics_stride": (ctypes.c_int, [I32, I32]),
        "fcw_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
        "fcw_analyze": (ctypes.c_int, [P, I64, P, I64, P, P, P]),
        "fcw_mesh_arrays": (ctypes.c_int, [P, I64, P, I64, P, P, P, P, P, P]),
        "fcw_engine_create": (ctypes.c_int, [P, I64, P, I64, P, ctypes.POINTER(P)]),
        "fcw_engine_info": (ctypes.c_int, [P, P]),
        "fcw_engine_destroy": (ctypes.c_int, [P]),
        "fcw_compute_distance": (ctypes.c_int, [P, I32, P]),
        "fcw_compute_distances": (ctypes.c_int, [P, P, I64, I32, P]),
        "fcw_compute_metrics": (ctypes.c_int, [P, P, I64, I32, P, I32, I32, D, P]),
        "fcw_compute_metrics_device": (ctypes.c_int, [P, P, I64, I32, P, I32, I32, D, P, P]),
        "fcw_synchronize": (ctypes.c_int, [P, P]),
        "fcw_engine_profile": (ctypes.c_int, [P, ctypes.c_int]),
        "fcw_engine_graphs": (ctypes.c_int, [P, ctypes.c_int]),
        "fcw_engine_stage_times": (ctypes.c_int, [P, P, I32, P]),
        "fcw_heat_solve_device": (ctypes.c_int, [P, P, I32, P, P]),
        "fcw_divergence_device": (ctypes.c_int, [P, P, I32, P, P]),
        "fcw_poisson_solve_device": (ctypes.c_int, [P, P, P, I32, P, P]),
        "fcw_field_metrics_device": (ctypes.c_int, [P, P, P, I32, P, I32, I32, D, P, P]),
        "fcw_field_metrics_static": (ctypes.c_int, [P, P, P, I32, P, I32, I32, D, P, P]),
        "fcw_samples_capacity": (ctypes.c_int, [I32, I32]),
        "fcw_assemble_samples_device": (ctypes.c_int, [P, I64, I32, I32, P, D, P, P, P, P]),
        "fcw_assemble_samples": (ctypes.c_int, [P, P, I64, I32, I32, P, D, P, P, P]),
        "fcw_tc_product_check": (ctypes.c_int, [P, P, P, I32, I32, I32, I32, I32, P, P, P]),
        "fcw_intrinsic_operators": (ctypes.c_int, [P, I64, P, I64, P, P, P, P, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(2048)
    load().fcw_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != FCW_OK:
        raise FCWError(rc, last_error())


def ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def default_params(**overrides) -> FCWParams:
    p = FCWParams()
    load().fcw_default_params(ctypes.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown engine parameter {k!r}")
        setattr(p, k, v)
    return p


def metrics_stride(n_targets: int, n_between: int) -> int:
    return int(load().fcw_metrics_stride(int(n_targets), int(n_between)))


def samples_capacity(n_targets: int, n_between: int) -> int:
    return int(load().fcw_samples_capacity(int(n_targets), int(n_between)))


def analyze(V, F, **params):
    """Host-only symbolic analysis: (info dict, elimination order)."""
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int32)
    p = default_params(**params)
    info = FCWInfo()
    perm = np.empty(V.shape[0], dtype=np.int32)
    check(load().fcw_analyze(ptr(V), V.shape[0], ptr(F), F.shape[0], ctypes.byref(p), ctypes.byref(info), ptr(perm)))
    return info.as_dict(), perm


def mesh_arrays(V, F):
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int32)
    nv, nf = V.shape[0], F.shape[0]
    va, la, g11, g12, g22 = np.empty(nv), np.empty(nf), np.empty(nf), np.empty(nf), np.empty(nf)
    bf = np.empty(nv, dtype=np.uint8)
    check(load().fcw_mesh_arrays(ptr(V), nv, ptr(F), nf, ptr(va), ptr(la), ptr(g11), ptr(g12), ptr(g22), ptr(bf)))
    return dict(vertex_area=va, lean_area=la, g11=g11, g12=g12, g22=g22, boundary=np.flatnonzero(bf).astype(np.int32))


def intrinsic_operators(V, F):
    """The robust operators on the host: dict with nflips, L (scipy CSC), mass, and the
    flipped tufted cover (tri, len, twin over 2 n_faces faces; None when nothing flipped)."""
    import scipy.sparse as sp

    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int32)
    nv, nf = V.shape[0], F.shape[0]
    nfl, nnz = ctypes.c_int64(0), ctypes.c_int64(0)
    lib = load()
    check(lib.fcw_intrinsic_operators(ptr(V), nv, ptr(F), nf, ctypes.byref(nfl), ctypes.byref(nnz),
                                      None, None, None, None, None, None, None))
    Lp = np.empty(nv + 1, np.int64)
    Li = np.empty(nnz.value, np.int32)
    Lx = np.empty(nnz.value, np.float64)
    mass = np.empty(nv, np.float64)
    tri = np.empty(6 * nf, np.int32)
    ln = np.empty(6 * nf, np.float64)
    tw = np.empty(6 * nf, np.int32)
    check(lib.fcw_intrinsic_operators(ptr(V), nv, ptr(F), nf, ctypes.byref(nfl), ctypes.byref(nnz), ptr(Lp),
                                      ptr(Li), ptr(Lx), ptr(mass), ptr(tri), ptr(ln), ptr(tw)))
    flipped = nfl.value > 0
    return dict(nflips=int(nfl.value), L=sp.csc_matrix((Lx, Li, Lp), shape=(nv, nv)), mass=mass,
                tri=tri.reshape(2 * nf, 3) if flipped else None, len=ln.reshape(2 * nf, 3) if flipped else None,
                twin=tw.reshape(2 * nf, 3) if flipped else None)
