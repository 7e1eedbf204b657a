"""ctypes binding of ``libgasp_b200.so`` (the C ABI declared in include/gasp.h).

The library is built in-tree by ``gpu_2dising_b200.build.build()``; importing
this module raises ``ImportError`` when it is missing -- there is no fallback
implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libgasp_b200.so")

GASP_OK = 0
GASP_ERR_INVALID = 1
GASP_ERR_CUDA = 2
GASP_ERR_NO_DEVICE = 3
GASP_ERR_ALLOC = 4
GASP_ERR_IO = 5
GASP_ERR_FORMAT = 6
GASP_ERR_CALLBACK = 7
GASP_ERR_UNSUPPORTED = 8
GASP_ERR_TIMEOUT = 9

OPT_SWEEP_VARIANT = 1
OPT_WARPS_PER_CTA = 2
OPT_TAIL_REPLICAS = 3

BATCH_PLAIN = 0
BATCH_GRAPH = 1
BATCH_MULTI = 2

RNG_XORWOW = 0
RNG_MWC64X = 1

MODE_EXACT = 0
MODE_TRACE_CPU = 1

# Every symbol include/gasp.h declares (checked by tests/test_abi.py).
EXPORTED = (
    "gasp_status_string", "gasp_last_error", "gasp_version", "gasp_init_device",
    "gasp_select_gpu_method", "gasp_acceptance_table", "gasp_max_shared_L",
    "gasp_set_stream", "gasp_init_grid", "gasp_free_grid", "gasp_grids_upload",
    "gasp_grids_download", "gasp_grids_upload_inputs",
    "gasp_grids_upload_inputs_noalloc", "gasp_grids_shape", "gasp_grids_set_option", "gasp_init_rand",
    "gasp_init_rand_mode", "gasp_mwc64x_seed_states", "gasp_acceptance_thresholds",
    "gasp_mwc64x_lane_multipliers", "gasp_rng_read_states", "gasp_free_rand",
    "gasp_sweep", "gasp_sweep_trace_cpu", "gasp_magnetisation", "gasp_largest_cluster", "gasp_pack_frame",
    "gasp_frame_bytes", "gasp_mc_driver_gpu", "gasp_mc_driver_gpu_ex",
    "gasp_init_grids_uniform", "gasp_init_grids_from_file", "gasp_init_grids_from_array",
    "gasp_init_fates", "gasp_read_input_grid", "gasp_write_ising_grids",
    "gasp_write_packed_frame", "gasp_bootstrap_errbar", "gasp_committor_from_fates",
    "gasp_read_frame", "gasp_write_input_grid", "gasp_create_ising_grids_hdf5",
    "gasp_write_ising_grids_hdf5", "gasp_checkpoint_save", "gasp_checkpoint_info",
    "gasp_checkpoint_load",
    "gasp_batch_create", "gasp_batch_free", "gasp_batch_swarm", "gasp_batch_autotune",
    "gasp_batch_layout",
    "gasp_cnn_param_count", "gasp_cnn_create", "gasp_cnn_free", "gasp_cnn_set_params",
    "gasp_cnn_set_fused",
    "gasp_cnn_get_params", "gasp_cnn_predict", "gasp_cnn_predict_ex", "gasp_cnn_gradients",
    "gasp_cnn_train_step",
)


class GaspError(RuntimeError):
    """A non-zero status from the native library."""

    def __init__(self, status, what=""):
        self.status = status
        lib = _lib
        text = lib.gasp_status_string(status).decode() if lib else str(status)
        detail = lib.gasp_last_error().decode() if lib else ""
        super().__init__(f"{what}: {text} ({detail})" if what else f"{text} ({detail})")


# ---- C types mirroring include/gasp.h -------------------------------------
class SamplerT(C.Structure):
    _fields_ = [("tot_nsweeps", C.c_int), ("mag_output_int", C.c_int),
                ("grid_output_int", C.c_int)]


class FunctionT(C.Structure):
    _fields_ = [("itask", C.c_int), ("dn_thr", C.c_double), ("up_thr", C.c_double),
                ("ninputs", C.c_int), ("initial_spin", C.c_int), ("cv", C.c_char_p),
                ("result", C.POINTER(C.c_float)), ("filename", C.c_char_p)]


class GpuRunT(C.Structure):
    _fields_ = [("d_state", C.c_void_p), ("threadsPerBlock", C.c_int), ("gpu_method", C.c_int)]


class GpuGridsT(C.Structure):
    _fields_ = [("L", C.c_int), ("ngrids", C.c_int), ("ising_grids", C.POINTER(C.c_int)),
                ("d_grids", C.c_void_p)]


class GroupT(C.Structure):
    _fields_ = [("L", C.c_int), ("ngrids", C.c_int), ("beta", C.c_double), ("h", C.c_double)]


GRID_OUTPUT_FN = C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int,
                             C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_char_p,
                             C.c_double, C.c_double, C.c_char_p)
PACKED_OUTPUT_FN = C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint8), C.c_size_t,
                               C.c_int, C.POINTER(C.c_float), C.c_void_p)


class DriverOptsT(C.Structure):
    _fields_ = [("verbosity", C.c_int), ("compact", C.c_int),
                ("packed_out", PACKED_OUTPUT_FN), ("packed_user", C.c_void_p),
                ("elapsed_s", C.POINTER(C.c_double)), ("attempts", C.POINTER(C.c_longlong)),
                ("first_up", C.POINTER(C.c_int))]


_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")


def _bind(lib):
    P = C.c_void_p
    I = C.c_int
    sig = {
        "gasp_status_string": (C.c_char_p, [I]),
        "gasp_last_error": (C.c_char_p, []),
        "gasp_version": (C.c_char_p, []),
        "gasp_init_device": (I, [I, I, C.POINTER(I), C.POINTER(I)]),
        "gasp_select_gpu_method": (I, [I, I, I, I, C.POINTER(I)]),
        "gasp_acceptance_table": (I, [C.c_double, C.c_double, _f32p]),
        "gasp_max_shared_L": (I, [I, C.POINTER(I)]),
        "gasp_set_stream": (I, [P]),
        "gasp_init_grid": (I, [I, I, I, P, C.POINTER(P)]),
        "gasp_free_grid": (I, [P]),
        "gasp_grids_upload": (I, [P, _i32p]),
        "gasp_grids_download": (I, [P, _i32p]),
        "gasp_grids_upload_inputs": (I, [P, _i32p, I]),
        "gasp_grids_upload_inputs_noalloc": (I, [P, _i32p, I]),
        "gasp_grids_shape": (I, [P, C.POINTER(I), C.POINTER(I)]),
        "gasp_grids_set_option": (I, [P, I, I]),
        "gasp_init_rand": (I, [I, I, C.c_ulonglong, C.POINTER(P)]),
        "gasp_init_rand_mode": (I, [I, I, C.c_ulonglong, I, C.POINTER(P)]),
        "gasp_mwc64x_seed_states": (I, [C.c_ulonglong, I, I,
                                        np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")]),
        "gasp_acceptance_thresholds": (I, [P, C.c_double, C.c_double,
                                           np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS"),
                                           C.POINTER(I)]),
        "gasp_mwc64x_lane_multipliers": (I, [np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS"),
                                             np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")]),
        "gasp_rng_read_states": (I, [P, np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS"),
                                     C.c_longlong]),
        "gasp_free_rand": (I, [P]),
        "gasp_sweep": (I, [P, P, C.c_double, C.c_double, I, I]),
        "gasp_sweep_trace_cpu": (I, [P, _f64p, C.c_double, C.c_double, I]),
        "gasp_magnetisation": (I, [P, _f32p]),
        "gasp_largest_cluster": (I, [P, I, _f32p]),
        "gasp_pack_frame": (I, [P, _u8p]),
        "gasp_frame_bytes": (C.c_size_t, [I, I]),
        "gasp_mc_driver_gpu": (I, [GpuGridsT, C.c_double, C.c_double, P, SamplerT, FunctionT,
                                   GpuRunT, GRID_OUTPUT_FN]),
        "gasp_mc_driver_gpu_ex": (I, [GpuGridsT, C.c_double, C.c_double, P, SamplerT,
                                      FunctionT, GpuRunT, GRID_OUTPUT_FN,
                                      C.POINTER(DriverOptsT)]),
        "gasp_init_grids_uniform": (I, [I, I, I, _i32p]),
        "gasp_init_grids_from_file": (I, [C.c_char_p, I, I, _i32p]),
        "gasp_init_grids_from_array": (I, [I, I, I, _i32p, _i32p]),
        "gasp_init_fates": (I, [I, _i32p]),
        "gasp_read_input_grid": (I, [C.c_char_p, I, I, _i32p]),
        "gasp_write_ising_grids": (I, [I, I, _i32p, I, P, P, C.c_char_p, C.c_double,
                                       C.c_double, C.c_char_p]),
        "gasp_write_packed_frame": (I, [C.c_char_p, I, I, I, _u8p, C.c_size_t]),
        "gasp_read_frame": (I, [C.c_char_p, I, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_int), C.c_void_p, C.c_longlong]),
        "gasp_write_input_grid": (I, [C.c_char_p, I, _i32p]),
        "gasp_create_ising_grids_hdf5": (I, [I, I, I, C.c_double, C.c_double, I, C.c_char_p]),
        "gasp_write_ising_grids_hdf5": (I, [I, I, _i32p, I, P, P, C.c_char_p, C.c_double,
                                            C.c_double, C.c_char_p]),
        "gasp_checkpoint_save": (I, [C.c_char_p, P, P, C.c_void_p, I]),
        "gasp_checkpoint_info": (I, [C.c_char_p] + [C.POINTER(C.c_int)] * 5),
        "gasp_checkpoint_load": (I, [C.c_char_p, P, P, C.c_void_p, C.POINTER(C.c_int)]),
        "gasp_bootstrap_errbar": (C.c_double, [I, I, _i32p]),
        "gasp_committor_from_fates": (I, [I, I, _i32p, _f32p]),
        "gasp_batch_create": (I, [C.POINTER(GroupT), I, C.c_ulonglong, I, C.POINTER(P)]),
        "gasp_batch_free": (I, [P]),
        "gasp_batch_swarm": (I, [P, I, I, C.c_double, I, _i32p, C.POINTER(C.c_longlong),
                                 C.POINTER(C.c_double)]),
        "gasp_batch_autotune": (I, [P, I, _i32p]),
        "gasp_batch_layout": (I, [P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "gasp_cnn_param_count": (I, []),
        "gasp_cnn_create": (I, [I, I, C.POINTER(P)]),
        "gasp_cnn_free": (I, [P]),
        "gasp_cnn_set_params": (I, [P, _f32p]),
        "gasp_cnn_set_fused": (I, [P, I]),
        "gasp_cnn_get_params": (I, [P, _f32p]),
        "gasp_cnn_predict": (I, [P, _i8p, I, _f32p]),
        "gasp_cnn_predict_ex": (I, [P, _i8p, I, _f32p, C.c_void_p]),
        "gasp_cnn_gradients": (I, [P, _i8p, _f32p, I, C.POINTER(C.c_float), _f32p]),
        "gasp_cnn_train_step": (I, [P, _i8p, _f32p, I, C.c_float, C.POINTER(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib():
    """The loaded native library; raises ImportError if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"gasp-b200 native library missing: {LIB_PATH}. "
                "Build it with gpu_2dising_b200.build.build().")
        _lib = _bind(C.CDLL(LIB_PATH))
    return _lib


def check(status, what=""):
    if status != GASP_OK:
        raise GaspError(status, what)
    return status
