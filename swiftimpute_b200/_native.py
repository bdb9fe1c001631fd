"""ctypes binding of the C ABI declared in ``include/swiftimpute_b200.h``.

The library is the in-tree ``swiftimpute_b200/lib/libswiftimpute_b200.so``.
There is no fallback: if the library is missing or fails to load, every entry
point raises :class:`NativeLibraryError`.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_uint32, c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libswiftimpute_b200.so"

SI_OK = 0
STATUS_NAMES = {
    0: "SI_OK", 1: "SI_ERR_INVALID_ARG", 2: "SI_ERR_CUDA", 3: "SI_ERR_OUT_OF_MEMORY",
    4: "SI_ERR_UNSUPPORTED", 5: "SI_ERR_STATE", 6: "SI_ERR_TIMEOUT", 7: "SI_ERR_BUDGET",
    8: "SI_ERR_CANCELLED",
}
SEL_AUTO, SEL_WARP, SEL_INSERTION, SEL_FIRST_PAIRS, SEL_TARGET = 0, 1, 2, 3, 4
TRANS_MATRIX0, TRANS_PER_GAP = 0, 1
SAMPLE_ARGMAX, SAMPLE_PHILOX = 0, 1
PBWT_STORE_INDEX, PBWT_ROW_HASHES = 1, 2
GENO_MISSING = 3
IMPUTE_RESELECT = 1
IMPUTE_FULL_CHAIN = 2
IMPUTE_CODES_2BIT = 4
IMPUTE_HAPS_BITS = 8


class NativeLibraryError(RuntimeError):
    """The CUDA library could not be loaded; there is no CPU fallback."""


class SIError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class ImputeParams(ctypes.Structure):
    """Mirror of ``si_impute_params``."""
    _fields_ = [
        ("num_states", c_uint32),
        ("ne", c_uint32),
        ("rho_rate", c_double),
        ("theta", c_double),
        ("transition_mode", c_int32),
        ("selection_kind", c_int32),
        ("sampling", c_int32),
        ("flags", c_uint32),
        ("tie_eps", c_double),
        ("seed", c_uint64),
        ("sample_id_base", c_uint64),
        ("checkpoint_interval", c_uint32),
        ("block_threads", c_uint32),
        ("reserved", c_uint64 * 4),
    ]


INDEX_GLOBAL, INDEX_REGION = 0, 1
PLAN_AUTOTUNE = 1


class Region(ctypes.Structure):
    """Mirror of ``si_region``."""
    _fields_ = [("m_begin", c_uint32), ("m_end", c_uint32), ("num_states", c_uint32), ("index_origin", c_int32)]


class Job(ctypes.Structure):
    """Mirror of ``si_job``."""
    _fields_ = [("region", c_uint32), ("reserved", c_uint32), ("geno_offset", c_uint64), ("out_offset", c_uint64),
                ("sample_id", c_uint64)]


# (name, restype, argtypes) for every symbol the header declares.
class ServeConfig(ctypes.Structure):
    """Mirror of ``si_serve_config``."""
    _fields_ = [("max_batch_cells", c_uint64), ("max_wait_us", c_uint32), ("max_queue", c_uint32),
                ("max_batch_requests", c_uint32), ("reserved", c_uint32)]


class Request(ctypes.Structure):
    """Mirror of ``si_request``."""
    _fields_ = [("m_begin", c_uint32), ("m_end", c_uint32), ("num_states", c_uint32), ("index_origin", c_int32),
                ("n_samples", c_uint32), ("reserved", c_uint32), ("sample_id_base", c_uint64),
                ("codes", c_void_p), ("dosage", c_void_p), ("haps", c_void_p), ("hap_prob", c_void_p)]


class ServeStatistics(ctypes.Structure):
    """Mirror of ``si_serve_statistics``."""
    _fields_ = [("submitted", c_uint64), ("completed", c_uint64), ("failed", c_uint64), ("cancelled", c_uint64),
                ("batches", c_uint64), ("cells", c_uint64), ("latency_p50_ms", ctypes.c_double),
                ("latency_p99_ms", ctypes.c_double), ("latency_max_ms", ctypes.c_double),
                ("busy_ms", ctypes.c_double), ("wall_ms", ctypes.c_double)]


SIGNATURES = [
    ("si_abi_version", c_int, []),
    ("si_status_string", c_char_p, [c_int]),
    ("si_ctx_create", c_int, [c_int, c_uint64, POINTER(c_void_p)]),
    ("si_ctx_destroy", c_int, [c_void_p]),
    ("si_last_error", c_char_p, [c_void_p]),
    ("si_ctx_memory", c_int, [c_void_p, POINTER(c_uint64), POINTER(c_uint64)]),
    ("si_panel_upload_u8", c_int, [c_void_p, c_void_p, c_uint32, c_uint32]),
    ("si_panel_exception_count", c_int, [c_void_p, POINTER(c_uint64)]),
    ("si_pbwt_stored_bytes", c_int, [c_void_p, POINTER(c_uint64)]),
    ("si_pbwt_save", c_int, [c_void_p, c_void_p, c_uint64]),
    ("si_pbwt_load", c_int, [c_void_p, c_void_p, c_uint64]),
    ("si_panel_upload_packed", c_int, [c_void_p, c_void_p, c_uint32, c_uint32, c_uint32]),
    ("si_panel_set_map", c_int, [c_void_p, c_void_p, c_void_p]),
    ("si_pbwt_build", c_int, [c_void_p, c_uint32]),
    ("si_pbwt_get_prefix_rows", c_int, [c_void_p, c_uint32, c_uint32, c_void_p]),
    ("si_pbwt_row_hashes", c_int, [c_void_p, c_void_p]),
    ("si_pbwt_last_ms", c_int, [c_void_p, POINTER(c_float)]),
    ("si_select_states", c_int, [c_void_p, c_uint32, c_int32, c_uint32, c_uint32, c_void_p]),
    ("si_select_states_target", c_int, [c_void_p, c_uint32, c_void_p, c_uint32, c_void_p]),
    ("si_impute_params_default", c_int, [POINTER(ImputeParams)]),
    ("si_impute", c_int, [c_void_p, POINTER(ImputeParams), c_void_p, c_uint32, c_void_p, c_void_p, c_void_p]),
    ("si_impute_gl", c_int, [c_void_p, POINTER(ImputeParams), c_void_p, c_uint32, c_void_p, c_void_p, c_void_p]),
    ("si_impute_device", c_int,
     [c_void_p, POINTER(ImputeParams), c_void_p, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("si_impute_jobs_device", c_int,
     [c_void_p, POINTER(ImputeParams), POINTER(Region), c_uint32, POINTER(Job), c_uint32, c_void_p, c_void_p,
      c_void_p, c_void_p, c_void_p]),
    ("si_impute_device_noalloc", c_int,
     [c_void_p, POINTER(ImputeParams), c_void_p, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("si_last_timings", c_int, [c_void_p, POINTER(c_float)]),
    ("si_last_kernel_ms", c_int, [c_void_p, POINTER(c_float)]),
    ("si_plan_create", c_int,
     [c_void_p, POINTER(ImputeParams), POINTER(Region), c_uint32, POINTER(Job), c_uint32, c_uint32, c_void_p,
      c_void_p, c_void_p, c_void_p, c_uint32, POINTER(c_void_p)]),
    ("si_plan_launch", c_int, [c_void_p, c_void_p]),
    ("si_plan_graph_launch", c_int, [c_void_p, c_void_p]),
    ("si_plan_check", c_int, [c_void_p]),
    ("si_plan_info", c_int, [c_void_p, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_float)]),
    ("si_plan_destroy", c_int, [c_void_p]),
    ("si_serve_start", c_int, [c_void_p, POINTER(ImputeParams), POINTER(ServeConfig), POINTER(c_void_p)]),
    ("si_serve_submit", c_int, [c_void_p, POINTER(Request), POINTER(c_uint64)]),
    ("si_serve_poll", c_int, [c_void_p, c_uint64, POINTER(c_int), POINTER(c_int)]),
    ("si_serve_wait", c_int, [c_void_p, c_uint64, c_uint32, POINTER(c_int)]),
    ("si_serve_cancel", c_int, [c_void_p, c_uint64]),
    ("si_serve_stats", c_int, [c_void_p, POINTER(ServeStatistics)]),
    ("si_serve_stop", c_int, [c_void_p]),
]

_lib = None


def load() -> ctypes.CDLL:
    """Load the library once; raise NativeLibraryError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise NativeLibraryError(
            f"{LIB_PATH} not found: build it with `python -m swiftimpute_b200.build` "
            "(there is no CPU fallback)")
    try:
        lib = ctypes.CDLL(str(LIB_PATH))
    except OSError as e:  # pragma: no cover - depends on the host
        raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def default_params(**overrides) -> ImputeParams:
    p = ImputeParams()
    load().si_impute_params_default(ctypes.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p
