"""Generic NUFFT of types 1 and 2 in one or two dimensions (device arrays),
built on the w-free gridder of this library (curig_nufft_* in include/curig.h).

Type 1: fk[k] = sum_j c_j exp(i iflag k.x_j), modes k = index - n/2;
type 2: c_j = sum_k fk[k] exp(i iflag k.x_j).  Points in radians (periodic).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .plan import PRECISIONS, _stream_handle


class Nufft:
    """One type-1 or type-2 transform with n_modes = (n1,) or (n1, n2)."""

    def __init__(self, nufft_type, n_modes, epsilon, iflag=1, sigma=2.0, precision="fp64", stream=None):
        n_modes = tuple(int(n) for n in n_modes)
        if len(n_modes) not in (1, 2):
            raise ValueError("n_modes must have one or two entries")
        self.type, self.n_modes = int(nufft_type), n_modes
        self.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self._opts = _lib.make_opts(self.precision, stream=_stream_handle(stream))
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.curig_nufft_makeplan(self.type, len(n_modes), n_modes[0],
                                                 n_modes[1] if len(n_modes) == 2 else 1, float(epsilon),
                                                 int(iflag), float(sigma), ctypes.byref(self._opts),
                                                 ctypes.byref(h)), "nufft_makeplan")
        self._h = h
        self._keep = None

    def setpts(self, x, y=None):
        """x (and y): contiguous float64 CUDA tensors of the m point coordinates."""
        if len(self.n_modes) == 2 and y is None:
            raise ValueError("two-dimensional transform needs y")
        self._keep = (x, y)
        self.m = int(x.shape[0])
        _lib.check(_lib.lib.curig_nufft_setpts(self._h, self.m, _lib.ptr(x), _lib.ptr(y)), "nufft_setpts")

    def execute(self, c, fk):
        """Type 1 reads c [m], writes fk (n_modes); type 2 reads fk, writes c."""
        _lib.check(_lib.lib.curig_nufft_execute(self._h, _lib.ptr(c), _lib.ptr(fk)), "nufft_execute")

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib.curig_nufft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass
