"""Device-pointer plan API (curig_makeplan / curig_setpts / curig_execute),
the Python face of the reference's gridder_setting / gridder_execution /
gridder_destroy life cycle (src/astro/cugridder.cu:105-307).

Arrays are CUDA tensors (torch) or raw device pointers; torch is used only to
hold device memory and to pass its current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

MS2DIRTY = 1
DIRTY2MS = 2
PRECISIONS = {"fp64": 0, "f64": 0, "float64": 0, "fp32": 1, "f32": 1, "float32": 1}
WINDOWS = {"es": 0, "learned": 1}


def _stream_handle(stream):
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:  # pragma: no cover
            pass
        return None
    return getattr(stream, "cuda_stream", stream)


def set_timing(on: bool) -> None:
    """Record per-stage CUDA events in every plan (off by default)."""
    _lib.lib.curig_set_timing(1 if on else 0)


def launch_count() -> int:
    """Kernels launched by libcurafft.so in this process."""
    return int(_lib.lib.curig_launch_count())


class GridderPlan:
    """One ms2dirty (kind=1) or dirty2ms (kind=2) transform with fixed image
    geometry; set points once, execute many times."""

    def __init__(self, kind, nxdirty, nydirty, pixsize_x, pixsize_y, epsilon, sigma=2.0, sign=-1,
                 precision="fp64", window="es", stream=None, bin_xy=0, sub=0, smem_budget=0,
                 accumulate=0, w_term=0, grid_x=0, grid_y=0, bin_z=0, sparse=0):
        self.kind = kind
        self.nxdirty, self.nydirty = int(nxdirty), int(nydirty)
        self.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self.window = WINDOWS[window] if isinstance(window, str) else int(window)
        self._stream = _stream_handle(stream)
        self._opts = _lib.make_opts(self.precision, self.window, bin_xy, sub, smem_budget, self._stream,
                                    accumulate, w_term, grid_x, grid_y, bin_z, sparse=sparse)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.curig_makeplan(kind, self.nxdirty, self.nydirty, float(pixsize_x),
                                           float(pixsize_y), float(epsilon), float(sigma), int(sign),
                                           ctypes.byref(self._opts), ctypes.byref(h)), "makeplan")
        self._h = h
        self._keep = None

    def setpts(self, uvw, freq):
        """uvw: device float64 [nrow, 3] (tensor or (pointer, nrow)); freq: host array [nchan]."""
        freq = np.ascontiguousarray(np.atleast_1d(freq), dtype=np.float64)
        if isinstance(uvw, tuple):
            p, nrow = uvw
        else:
            if uvw.dtype.__str__() not in ("torch.float64",) or not uvw.is_contiguous() or uvw.shape[-1] != 3:
                raise TypeError("uvw must be a contiguous float64 CUDA tensor [nrow, 3]")
            p, nrow = uvw.data_ptr(), uvw.shape[0]
        self._keep = (uvw, freq)
        self.nrow, self.nchan = int(nrow), int(freq.shape[0])
        _lib.check(_lib.lib.curig_setpts(self._h, self.nrow, self.nchan, p, freq.ctypes.data), "setpts")

    def execute(self, vis, wgt, dirty):
        """ms2dirty: reads vis [nrow, nchan] (+ wgt), writes dirty [nx, ny];
        dirty2ms: reads dirty, writes vis.  Device tensors or pointers."""
        _lib.check(_lib.lib.curig_execute(self._h, _lib.ptr(vis), _lib.ptr(wgt), _lib.ptr(dirty)),
                   "execute")

    def execute_dir(self, kind, vis, wgt, dirty):
        """Execute in direction ``kind`` (1 ms2dirty, 2 dirty2ms) with the same points."""
        _lib.check(_lib.lib.curig_execute_dir(self._h, int(kind), _lib.ptr(vis), _lib.ptr(wgt),
                                              _lib.ptr(dirty)), "execute")

    def status(self) -> None:
        """Wait for the plan's stream and raise CurigError if its kernels flagged
        a failure since set points (an interpolator tile load that did not
        complete within its bounded wait, or an index check of the
        bounds-checked build)."""
        _lib.check(_lib.lib.curig_plan_status(self._h), "plan_status")

    def timings(self) -> dict:
        """Stage durations (ms) of the last setpts / executes (needs set_timing(True))."""
        out = (ctypes.c_double * 11)()
        _lib.check(_lib.lib.curig_plan_timings(self._h, out, 11), "plan_timings")
        keys = ["setpts", "binning", "vis_prep", "grid_zero", "spread", "fft_m2d", "correct_m2d",
                "correct_d2m", "fft_d2m", "interp", "vis_out"]
        return {k: out[i] for i, k in enumerate(keys)}

    def info(self) -> dict:
        ii = (ctypes.c_int * 8)()
        dd = (ctypes.c_double * 6)()
        _lib.check(_lib.lib.curig_plan_info(self._h, ii, dd), "plan_info")
        keys = ["nf1", "nf2", "nf3", "kw", "bin_xy", "bin_z", "nbins", "window"]
        out = {k: ii[i] for i, k in enumerate(keys)}
        out.update(beta=dd[0], gamma=dd[1], h=dd[2], w_center=dd[3], w_half=dd[4], nm1_center=dd[5])
        return out

    def error_estimate(self) -> dict:
        """Estimated relative L2 error of this plan's results against the FP64
        direct transform, with its parts (curig_plan_error)."""
        e = (ctypes.c_double * 4)()
        _lib.check(_lib.lib.curig_plan_error(self._h, e), "plan_error")
        return {"total": e[0], "window": e[1], "arithmetic": e[2], "accumulation": e[3]}

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib.curig_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass
