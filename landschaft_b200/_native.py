"""ctypes binding of ``liblsb_omni.so`` (the C ABI of ``include/lsb_omniscape.h``).

The product path has no fallback: when the library is missing, or when no CUDA
device is present, every compute call raises.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "liblsb_omni.so"

LSB_OK, LSB_ERR_ARGUMENT, LSB_ERR_NOT_CONVERGED, LSB_ERR_CONDITION, LSB_ERR_WORKSPACE, LSB_ERR_CUDA = range(6)
PREC_FP64, PREC_FP32_REFINE = 0, 1
PC_AUTO, PC_JACOBI, PC_MG = 0, 1, 2
EDGE_AVERAGE, EDGE_SERIES = 0, 1

# Every symbol the header declares (the CPU test checks the library exports them).
EXPORTS = ("lsb_params_default", "lsb_omniscape_workspace_size", "lsb_omniscape", "lsb_omniscape_correction",
           "lsb_omniscape_grad", "lsb_omniscape_grad_workspace_size", "lsb_last_launch_count",
           "lsb_time_window_kernels", "lsb_version", "lsb_omniscape_noalloc", "lsb_tune_set", "lsb_tune_get",
           "lsb_tune_clear", "lsb_raster_params_default", "lsb_rasters_workspace_size", "lsb_rasters",
           "lsb_graph_params_default", "lsb_graph_pairs_workspace_size", "lsb_graph_pairs",
           "lsb_graph_solve_workspace_size", "lsb_graph_solve")


class Condition(C.Structure):
    _fields_ = [("present", C.c_void_p), ("future", C.c_void_p), ("equal", C.c_int32), ("pad_", C.c_int32),
                ("lower", C.c_double), ("upper", C.c_double)]


class Params(C.Structure):
    _fields_ = [("radius", C.c_int32), ("buffer", C.c_int32), ("block_size", C.c_int32),
                ("four_neighbors", C.c_int32), ("resistance_is_conductance", C.c_int32),
                ("correct_artifacts", C.c_int32), ("flow_potential", C.c_int32), ("edge_weights", C.c_int32),
                ("condition1", Condition), ("condition2", Condition), ("memory_limit", C.c_double),
                ("precision", C.c_int32), ("preconditioner", C.c_int32), ("tol", C.c_double),
                ("max_iter", C.c_int32), ("threads_per_window", C.c_int32), ("use_graph", C.c_int32),
                ("mask_nodata", C.c_int32), ("accumulate", C.c_int32), ("target_begin", C.c_int64),
                ("target_end", C.c_int64)]


class Stats(C.Structure):
    _fields_ = [("n_targets", C.c_int64), ("n_solved", C.c_int64), ("n_failed", C.c_int64),
                ("iters_total", C.c_int64), ("iters_max", C.c_int32), ("refine_max", C.c_int32),
                ("batches", C.c_int32), ("threads_per_window", C.c_int32), ("preconditioner", C.c_int32),
                ("pad_", C.c_int32), ("worst_residual", C.c_double), ("window_ms", C.c_double),
                ("unknown_iters", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


class RasterParams(C.Structure):
    _fields_ = [("four_neighbors", C.c_int32), ("precision", C.c_int32), ("tol", C.c_double),
                ("max_iter", C.c_int32), ("smem_limit_kb", C.c_int32), ("memory_limit", C.c_double)]


class GraphParams(C.Structure):
    _fields_ = [("tol", C.c_double), ("accept", C.c_double), ("max_iter", C.c_int32), ("max_ctas", C.c_int32)]


class GraphStats(C.Structure):
    _fields_ = [("jobs", C.c_int64), ("failures", C.c_int64), ("iters_max", C.c_int32), ("ctas", C.c_int32),
                ("iters_mean", C.c_double), ("worst_residual", C.c_double)]


class NativeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_lib = None
_lock = threading.Lock()


def load():
    """The native library (raises when it is missing: there is no CPU fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH.name} is not built: run landschaft_b200._build.build() "
                               "(or __graft_entry__.build())")
        lib = C.CDLL(str(LIB_PATH))
        vp, i64, sz = C.c_void_p, C.c_int64, C.c_size_t
        lib.lsb_params_default.argtypes = [C.POINTER(Params)]
        lib.lsb_params_default.restype = None
        lib.lsb_omniscape_workspace_size.argtypes = [i64, i64, C.POINTER(Params), C.POINTER(sz)]
        lib.lsb_omniscape_workspace_size.restype = C.c_int
        lib.lsb_omniscape.argtypes = [vp, vp, i64, i64, C.POINTER(Params), vp, vp, vp, vp, sz, C.POINTER(Stats),
                                      C.c_char_p, sz, vp]
        lib.lsb_omniscape.restype = C.c_int
        lib.lsb_omniscape_correction.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, i64, i64, vp,
                                                 vp, sz, C.c_char_p, sz, vp]
        lib.lsb_omniscape_correction.restype = C.c_int
        lib.lsb_omniscape_grad.argtypes = [vp, vp, vp, i64, i64, C.POINTER(Params), vp, vp, vp, vp, sz,
                                           C.POINTER(Stats), C.c_char_p, sz, vp]
        lib.lsb_omniscape_grad.restype = C.c_int
        lib.lsb_omniscape_grad_workspace_size.argtypes = [i64, i64, C.POINTER(Params), C.POINTER(sz)]
        lib.lsb_omniscape_grad_workspace_size.restype = C.c_int
        lib.lsb_last_launch_count.argtypes = []
        lib.lsb_last_launch_count.restype = i64
        lib.lsb_time_window_kernels.argtypes = [C.c_int32]
        lib.lsb_time_window_kernels.restype = None
        lib.lsb_omniscape_noalloc.argtypes = [vp, vp, i64, i64, C.POINTER(Params), vp, vp, vp, C.POINTER(Stats),
                                              C.c_char_p, sz, vp]
        lib.lsb_omniscape_noalloc.restype = C.c_int
        lib.lsb_version.argtypes = []
        lib.lsb_version.restype = C.c_char_p
        i32 = C.c_int32
        lib.lsb_tune_set.argtypes = [i32] * 6
        lib.lsb_tune_set.restype = C.c_int
        lib.lsb_tune_get.argtypes = [i32] * 4 + [C.POINTER(i32), C.POINTER(i32)]
        lib.lsb_tune_get.restype = C.c_int
        lib.lsb_tune_clear.argtypes = []
        lib.lsb_tune_clear.restype = None
        lib.lsb_raster_params_default.argtypes = [C.POINTER(RasterParams)]
        lib.lsb_raster_params_default.restype = None
        lib.lsb_rasters_workspace_size.argtypes = [i64, vp, vp, C.POINTER(RasterParams), C.POINTER(sz)]
        lib.lsb_rasters_workspace_size.restype = C.c_int
        lib.lsb_rasters.argtypes = [i64, vp, vp, vp, vp, vp, C.POINTER(RasterParams), vp, vp, vp, sz,
                                    C.POINTER(Stats), C.c_char_p, sz, vp]
        lib.lsb_rasters.restype = C.c_int
        lib.lsb_graph_params_default.argtypes = [C.POINTER(GraphParams)]
        lib.lsb_graph_params_default.restype = None
        lib.lsb_graph_pairs_workspace_size.argtypes = [i64, i64, C.POINTER(GraphParams), C.POINTER(sz)]
        lib.lsb_graph_pairs_workspace_size.restype = C.c_int
        lib.lsb_graph_pairs.argtypes = [i64, vp, vp, vp, vp, i32, i64, vp, vp, C.POINTER(GraphParams), vp, vp, vp,
                                        sz, C.POINTER(GraphStats), C.c_char_p, sz, vp]
        lib.lsb_graph_pairs.restype = C.c_int
        lib.lsb_graph_solve_workspace_size.argtypes = [i64, i64, C.POINTER(GraphParams), C.POINTER(sz)]
        lib.lsb_graph_solve_workspace_size.restype = C.c_int
        lib.lsb_graph_solve.argtypes = [i64, vp, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, vp, vp,
                                        C.POINTER(GraphParams), vp, vp, vp, sz, C.POINTER(GraphStats), C.c_char_p,
                                        sz, vp]
        lib.lsb_graph_solve.restype = C.c_int
        _lib = lib
        return lib


def default_params() -> Params:
    p = Params()
    load().lsb_params_default(C.byref(p))
    return p


def default_raster_params() -> RasterParams:
    p = RasterParams()
    load().lsb_raster_params_default(C.byref(p))
    return p


def default_graph_params() -> GraphParams:
    p = GraphParams()
    load().lsb_graph_params_default(C.byref(p))
    return p


def check(rc: int, err) -> None:
    if rc == LSB_OK:
        return
    msg = err.value.decode(errors="replace") if err is not None else ""
    if rc == LSB_ERR_ARGUMENT:
        raise ValueError(msg)
    raise NativeError(rc, msg)
