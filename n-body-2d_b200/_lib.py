"""ctypes binding of libnbody_b200.so (declared in include/nbody_b200.h).

The library is the product path: if it is missing or fails to load, every
call here raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libnbody_b200.so"

NB_OK = 0
NB_ERR_INVALID = 1
NB_ERR_CUDA = 2
NB_ERR_CAPACITY = 3
NB_ERR_TIMEOUT = 4
NB_ERR_NOMEM = 5
NB_ERR_NOTFOUND = 6

NB_MODE_FP64 = 0
NB_MODE_SPLIT = 1
NB_MODE_ALLPAIRS = 2
NB_FLAG_QUADRUPOLE = 1
NB_FLAG_LEARNED = 2
NB_FLAG_CPU_LAW = 4
NB_MLP_PARAMS = 5123  # include/nbody_b200.h
NB_STATIC_SORT_MAX_BODIES = 262144  # include/nbody_b200.h

# Every symbol include/nbody_b200.h declares.
EXPORTS = (
    "nb_params_default", "nb_create", "nb_destroy", "nb_step", "nb_sync", "nb_set_timestep",
    "nb_upload", "nb_download", "nb_accelerations", "nb_debug_morton", "nb_debug_state",
    "nb_debug_tree", "nb_get_stats", "nb_last_error", "nb_status_string",
    "nb_allpairs_accelerations", "nb_phase_times", "nb_phase_name", "nb_morton_sort_static",
    "nb_set_mlp_weights", "nb_mlp_samples", "nb_mlp_forward", "nb_mlp_loss_grad", "nb_mlp_train",
    "nb_batch_create", "nb_autotune", "nb_render", "nb_download_async", "nb_download_wait",
    "nb_debug_wait_timeout", "nb_upload_async", "nb_debug_interactions", "nb_debug_groups",
    "nb_debug_sort_passes",
)


class NbView(C.Structure):
    _fields_ = [
        ("x", C.c_double),
        ("y", C.c_double),
        ("width", C.c_double),
        ("height", C.c_double),
        ("res_x", C.c_uint32),
        ("res_y", C.c_uint32),
        ("point_diameter", C.c_float),
        ("reserved", C.c_uint32),
    ]


class NbParams(C.Structure):
    _fields_ = [
        ("G", C.c_double),
        ("timestep", C.c_double),
        ("theta", C.c_double),
        ("epsilon_squared", C.c_double),
        ("mode", C.c_int32),
        ("leaf_size", C.c_int32),
        ("device", C.c_int32),
        ("flags", C.c_int32),
        ("bmax_ratio", C.c_double),
        ("band_theta", C.c_double),
        ("bodies_per_lane", C.c_int32),
        ("reserved", C.c_int32),
    ]


class NbStats(C.Structure):
    _fields_ = [
        ("steps", C.c_uint64),
        ("n", C.c_uint64),
        ("tree_nodes", C.c_uint64),
        ("cell_interactions", C.c_uint64),
        ("body_interactions", C.c_uint64),
        ("ms_last_step", C.c_double),
        ("root_width", C.c_double),
        ("kernels_per_step", C.c_uint64),
    ]


class NbMlpTrainParams(C.Structure):
    _fields_ = [
        ("epochs", C.c_uint32),
        ("batch", C.c_uint32),
        ("lr", C.c_float),
        ("seed", C.c_uint64),
    ]


class NbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib: C.CDLL | None = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)


def load() -> C.CDLL:
    """Loads the library once; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() (nvcc) first")
    lib = C.CDLL(str(LIB_PATH))
    lib.nb_params_default.argtypes = [C.POINTER(NbParams)]
    lib.nb_create.argtypes = [C.POINTER(NbParams), C.c_uint64, _P, _P, _P, C.POINTER(_P)]
    lib.nb_destroy.argtypes = [_P]
    lib.nb_step.argtypes = [_P, C.c_uint32]
    lib.nb_sync.argtypes = [_P]
    lib.nb_set_timestep.argtypes = [_P, C.c_double]
    lib.nb_upload.argtypes = [_P, _P, _P, _P]
    lib.nb_upload_async.argtypes = [_P, _P, _P, _P]
    lib.nb_download.argtypes = [_P, _P, _P]
    lib.nb_accelerations.argtypes = [_P, _P]
    lib.nb_debug_morton.argtypes = [_P, _P, _P, _P]
    lib.nb_debug_state.argtypes = [_P, _P, _P, _P, _P]
    lib.nb_debug_tree.argtypes = [_P, _P, _P, _P, _P, _P, _P]
    lib.nb_get_stats.argtypes = [_P, C.POINTER(NbStats)]
    lib.nb_debug_interactions.argtypes = [_P, _P, _P, _P]
    lib.nb_debug_groups.argtypes = [_P, _P, _P, C.c_uint64, _P]
    lib.nb_debug_sort_passes.argtypes = [_P, C.c_int32, _P]
    lib.nb_last_error.argtypes = [_P]
    lib.nb_last_error.restype = C.c_char_p
    lib.nb_status_string.argtypes = [C.c_int]
    lib.nb_status_string.restype = C.c_char_p
    lib.nb_morton_sort_static.argtypes = [_P, C.c_uint64, _P, _P, _P, _P]
    lib.nb_batch_create.argtypes = [C.POINTER(NbParams), C.c_uint32, _P, _P, _P, _P,
                                    C.POINTER(_P)]
    lib.nb_autotune.argtypes = [_P, C.c_uint32, _P, _P]
    lib.nb_render.argtypes = [_P, C.POINTER(NbView), _P]
    lib.nb_download_async.argtypes = [_P, _P, _P]
    lib.nb_download_wait.argtypes = [_P]
    lib.nb_debug_wait_timeout.argtypes = [C.c_int32]
    lib.nb_set_mlp_weights.argtypes = [_P, _P]
    lib.nb_mlp_samples.argtypes = [_P, C.c_uint64, C.c_uint64, C.c_uint64, _P, _P, _P]
    lib.nb_mlp_forward.argtypes = [C.c_int32, _P, C.c_uint64, _P, _P]
    lib.nb_mlp_loss_grad.argtypes = [C.c_int32, _P, C.c_uint64, _P, _P, _P, _P]
    lib.nb_mlp_train.argtypes = [C.c_int32, C.c_uint64, _P, _P, C.POINTER(NbMlpTrainParams), _P, _P]
    lib.nb_phase_times.argtypes = [_P, _P, C.c_int]
    lib.nb_phase_name.argtypes = [C.c_int]
    lib.nb_phase_name.restype = C.c_char_p
    lib.nb_allpairs_accelerations.argtypes = [C.c_int32, C.c_uint64, _P, _P, C.c_uint64, _P,
                                              C.c_double, _P]
    for name in EXPORTS:
        if name not in ("nb_last_error", "nb_status_string", "nb_phase_name"):
            getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays passed to libnbody_b200 must be C-contiguous")
    return a.ctypes.data


def check(status: int, ctx: int | None = None) -> None:
    if status == NB_OK:
        return
    lib = load()
    msg = lib.nb_status_string(status).decode()
    if ctx:
        detail = lib.nb_last_error(ctx).decode()
        if detail:
            msg = f"{msg}: {detail}"
    raise NbError(status, msg)
