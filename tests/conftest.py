import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")
REF_DIR = os.path.join(REPO, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # Build the native library and the oracle when they are missing.
    need = [os.path.join(REPO, "gpu_2dising_b200", "libgasp_b200.so"),
            os.path.join(REPO, "oracle", "liboracle.so")]
    if not all(os.path.exists(p) for p in need):
        from gpu_2dising_b200.build import build
        build()


def ref_lib_path(name):
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None


@pytest.fixture(scope="session")
def ref_cpu():
    """The reference CPU code compiled unmodified (skips if not built)."""
    import ctypes as C
    import numpy as np
    p = ref_lib_path("libref_cpu.so")
    if p is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    lib = C.CDLL(p)
    i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    lib.ref_driver_cpu.argtypes = [C.c_int, C.c_int, C.c_ulong, C.c_double, C.c_double, C.c_int,
                                   C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                   i32, C.c_void_p, f32, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
    lib.ref_driver_cpu.restype = C.c_int
    lib.ref_precompute_probs_cpu.argtypes = [C.c_double, C.c_double, f64]
    lib.ref_sweep_cpu.argtypes = [C.c_int, i32, C.c_int, C.c_double, C.c_double, C.c_int]
    lib.ref_magnetisation_cpu.argtypes = [C.c_int, i32, C.c_int]
    lib.ref_magnetisation_cpu.restype = C.c_float
    lib.compute_largest_cluster_cpu.argtypes = [C.c_int, i32, C.c_int, C.c_int, f32]
    lib.ref_bootstrap_errbar.argtypes = [C.c_int, C.c_int, i32]
    lib.ref_bootstrap_errbar.restype = C.c_double
    lib.ref_init_grids_from_array.argtypes = [C.c_int, C.c_int, C.c_int, i32, i32]
    lib.ref_genrand_int32.restype = C.c_ulong
    lib.ref_genrand_real3.restype = C.c_double
    lib.ref_init_genrand.argtypes = [C.c_ulong]
    return lib


@pytest.fixture(scope="session")
def ref_gpu():
    """The reference GPU kernels compiled for sm_100a (skips if not built)."""
    import ctypes as C
    import numpy as np
    p = ref_lib_path("libref_gpu.so")
    if p is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    lib = C.CDLL(p)
    i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    lib.refgpu_run_kernels.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                       C.c_double, C.c_double, C.c_int, C.c_int, i32, f32]
    lib.refgpu_uniform_stream.argtypes = [C.c_ulonglong, C.c_int, C.c_int, f32]
    lib.refgpu_run_driver.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                      C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_double, C.c_double, C.c_int, i32, C.c_void_p, f32,
                                      C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.refgpu_run_driver_cv.argtypes = lib.refgpu_run_driver.argtypes + [C.c_char_p, C.c_int,
                                                                          C.c_void_p]
    lib.refgpu_largest_cluster.argtypes = [C.c_int, C.c_int, C.c_int, i32, f32]
    return lib


def has_gpu():
    try:
        r = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=20)
        return r.returncode == 0 and "GPU" in r.stdout
    except Exception:
        return False
