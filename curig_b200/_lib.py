"""ctypes binding of libcurafft.so (the B200 gridder's C ABI, include/curig.h).

The argument types of the four reference entry points are those of the
reference's own binding (python/curagridder/curagridder.py:50-70): C-contiguous
float64 / complex128 ndpointers, so wrong dtypes or layouts raise
ctypes.ArgumentError exactly as they do there.  There is no fallback: if the
library is missing, importing this module raises RuntimeError (as the
reference's loader does, curagridder.py:24-28).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_double, c_int, c_int64, c_void_p

import numpy as np

# CURIG_LIB selects another build of the library, e.g. the bounds-checked
# libcurafft_check.so (curig_b200/csrc/build.py --check)
LIB_PATH = os.environ.get("CURIG_LIB") or os.path.join(os.path.dirname(os.path.abspath(__file__)), "libcurafft.so")

try:
    lib = ctypes.CDLL(LIB_PATH)
except OSError as exc:  # pragma: no cover - exercised when the build is missing
    raise RuntimeError(
        f"Failed to load the curig_b200 CUDA library {LIB_PATH}: {exc}. "
        "Build it with `python curig_b200/csrc/build.py`.") from exc

_f64 = np.ctypeslib.ndpointer(np.double, flags="C")
_c128 = np.ctypeslib.ndpointer(np.complex128, flags="C")

# reference ABI (include/cugridder.h:12-21)
ms2dirty_1 = lib.ms2dirty_1
ms2dirty_1.argtypes = [c_int, c_int, c_int, c_double, c_double, _f64, _c128, _c128, c_double,
                       c_double, c_int]
ms2dirty_1.restype = c_int
ms2dirty_2 = lib.ms2dirty_2
ms2dirty_2.argtypes = [c_int, c_int, c_int, c_double, c_double, _f64, _c128, _f64, _c128, c_double,
                       c_double, c_int]
ms2dirty_2.restype = c_int
dirty2ms_1 = lib.dirty2ms_1
dirty2ms_1.argtypes = ms2dirty_1.argtypes
dirty2ms_1.restype = c_int
dirty2ms_2 = lib.dirty2ms_2
dirty2ms_2.argtypes = ms2dirty_2.argtypes
dirty2ms_2.restype = c_int


class CurigOpts(ctypes.Structure):
    _fields_ = [("precision", c_int), ("window", c_int), ("bin_xy", c_int), ("sub", c_int),
                ("smem_budget", c_int64), ("stream", c_void_p), ("accumulate", c_int), ("w_term", c_int),
                ("grid_x", c_int), ("grid_y", c_int), ("bin_z", c_int), ("slabs", c_int), ("sparse", c_int)]


def make_opts(precision: int = 0, window: int = 0, bin_xy: int = 0, sub: int = 0,
              smem_budget: int = 0, stream: int | None = None, accumulate: int = 0, w_term: int = 0,
              grid_x: int = 0, grid_y: int = 0, bin_z: int = 0, slabs: int = 0, sparse: int = 0) -> CurigOpts:
    return CurigOpts(precision, window, bin_xy, sub, smem_budget, stream or None, accumulate, w_term,
                     grid_x, grid_y, bin_z, slabs, sparse)


_P = c_void_p
lib.curig_ms2dirty.argtypes = [c_int64, c_int, c_int, c_int, c_double, c_double, _P, _P, _P, _P, _P,
                               c_double, c_double, c_int, ctypes.POINTER(CurigOpts)]
lib.curig_ms2dirty.restype = c_int
lib.curig_dirty2ms.argtypes = lib.curig_ms2dirty.argtypes
lib.curig_dirty2ms.restype = c_int
lib.curig_makeplan.argtypes = [c_int, c_int, c_int, c_double, c_double, c_double, c_double, c_int,
                               ctypes.POINTER(CurigOpts), ctypes.POINTER(c_void_p)]
lib.curig_makeplan.restype = c_int
lib.curig_setpts.argtypes = [c_void_p, c_int64, c_int, _P, _P]
lib.curig_setpts.restype = c_int
lib.curig_setpts_uvw.argtypes = [c_void_p, c_int64, c_int, _P, _P, _P, c_int, _P]
lib.curig_setpts_uvw.restype = c_int
lib.curig_execute.argtypes = [c_void_p, _P, _P, _P]
lib.curig_execute.restype = c_int
lib.curig_execute_dir.argtypes = [c_void_p, c_int, _P, _P, _P]
lib.curig_execute_dir.restype = c_int
lib.curig_set_timing.argtypes = [c_int]
lib.curig_set_timing.restype = None
lib.curig_plan_timings.argtypes = [c_void_p, ctypes.POINTER(c_double), c_int]
lib.curig_plan_timings.restype = c_int
lib.curig_plan_status.argtypes = [c_void_p]
lib.curig_plan_status.restype = c_int
lib.curig_launch_count.argtypes = []
lib.curig_launch_count.restype = c_int64
lib.curig_destroy.argtypes = [c_void_p]
lib.curig_destroy.restype = c_int
lib.curig_plan_info.argtypes = [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_double)]
lib.curig_plan_info.restype = c_int
lib.curig_plan_error.argtypes = [c_void_p, ctypes.POINTER(c_double)]
lib.curig_plan_error.restype = c_int
lib.curig_set_window.argtypes = [c_int, c_int, _P, c_double]
lib.curig_set_window.restype = c_int
lib.curig_clear_windows.argtypes = []
lib.curig_clear_windows.restype = None
lib.curig_last_error.argtypes = []
lib.curig_last_error.restype = ctypes.c_char_p
lib.curig_release_memory.argtypes = []
lib.curig_release_memory.restype = c_int
lib.curig_grid_params.argtypes = [c_int, c_int, c_double, c_double, c_double, c_double, c_double,
                                  c_double, ctypes.POINTER(c_int), ctypes.POINTER(c_double)]
lib.curig_grid_params.restype = c_int
lib.curig_psi_hat.argtypes = [c_int, c_double, c_double, ctypes.POINTER(c_double)]
lib.curig_psi_hat.restype = c_int
lib.curig_window_nparams.argtypes = []
lib.curig_window_nparams.restype = c_int
lib.curig_train_window.argtypes = [c_int, c_double, c_int, c_double, _P, _P]
lib.curig_train_window.restype = c_int
lib.curig_train_window_mc.argtypes = [c_int, c_double, c_int, c_double, ctypes.c_uint64, _P, _P]
lib.curig_train_window_mc.restype = c_int
lib.curig_window_loss_grad.argtypes = [c_int, c_double, _P, _P, _P]
lib.curig_window_loss_grad.restype = c_int
lib.curig_window_table.argtypes = [c_int, c_double, _P, c_int, _P]
lib.curig_window_loss_grad_static.argtypes = [c_int, c_double, _P, _P, _P]
lib.curig_window_loss_grad_static.restype = c_int
lib.curig_window_table.restype = c_int
lib.curig_default_opts.argtypes = [ctypes.POINTER(CurigOpts)]
lib.curig_nufft_makeplan.argtypes = [c_int, c_int, c_int, c_int, c_double, c_int, c_double,
                                     ctypes.POINTER(CurigOpts), ctypes.POINTER(c_void_p)]
lib.curig_nufft_makeplan.restype = c_int
lib.curig_nufft_setpts.argtypes = [c_void_p, c_int64, _P, _P]
lib.curig_nufft_setpts.restype = c_int
lib.curig_nufft_execute.argtypes = [c_void_p, _P, _P]
lib.curig_nufft_execute.restype = c_int
lib.curig_nufft_destroy.argtypes = [c_void_p]
lib.curig_nufft_destroy.restype = c_int
lib.curig_default_opts.restype = None
lib.curig_nufft3d_makeplan.argtypes = [c_int, c_int, c_int, c_int, c_double, c_int, c_double,
                                       ctypes.POINTER(CurigOpts), ctypes.POINTER(c_void_p)]
lib.curig_nufft3d_makeplan.restype = c_int
lib.curig_nufft3d_setpts.argtypes = [c_void_p, c_int64, _P, _P, _P]
lib.curig_nufft3d_setpts.restype = c_int
lib.curig_nufft_setpts3.argtypes = [c_void_p, c_int64, _P, c_int64, _P]
lib.curig_nufft_setpts3.restype = c_int
lib.curig_nufft_info3.argtypes = [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_double)]
lib.curig_nufft_info3.restype = c_int
lib.curig_test_tile_wait.argtypes = [c_int64, c_int]
lib.curig_test_tile_wait.restype = None
lib.curig_test_gather_scratch.argtypes = [c_int]
lib.curig_test_gather_scratch.restype = None

ERRORS = {
    1: "generic error", 2: "bad upsampling factor", 3: "invalid argument", 4: "CUDA error",
    5: "cuFFT error", 6: "out of device memory", 7: "NaN/Inf input", 8: "unsupported option",
    9: "no learned window reaches the requested epsilon",
}


class CurigError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib.curig_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != 0:
        raise CurigError(code, where)


def ptr(a) -> int | None:
    """Data pointer of a numpy array or torch tensor (None passes through)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
