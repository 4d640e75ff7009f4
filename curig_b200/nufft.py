"""Generic NUFFT of types 1 and 2 in one or two dimensions and of type 3 in
one dimension (device arrays); types 1 and 2 run on the w-free gridder of this
library, type 3 spreads onto its own grid and evaluates it with a type 2
(curig_nufft_* in include/curig.h).

Type 1: fk[k] = sum_j c_j exp(i iflag k.x_j), modes k = index - n/2;
type 2: c_j = sum_k fk[k] exp(i iflag k.x_j).  Points in radians (periodic).
Type 3: f_k = sum_j c_j exp(i iflag s_k x_j), any real points and frequencies.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .plan import PRECISIONS, _stream_handle


class Nufft:
    """One type-1 or type-2 transform with n_modes = (n1,), (n1, n2) or (n1, n2, n3)."""

    def __init__(self, nufft_type, n_modes, epsilon, iflag=1, sigma=2.0, precision="fp64", stream=None):
        n_modes = tuple(int(n) for n in n_modes)
        if len(n_modes) not in (1, 2, 3):
            raise ValueError("n_modes must have one to three entries")
        self.type, self.n_modes = int(nufft_type), n_modes
        self.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self._opts = _lib.make_opts(self.precision, stream=_stream_handle(stream))
        h = ctypes.c_void_p()
        if len(n_modes) == 3:
            _lib.check(_lib.lib.curig_nufft3d_makeplan(self.type, *n_modes, float(epsilon), int(iflag), float(sigma),
                                                       ctypes.byref(self._opts), ctypes.byref(h)), "nufft3d_makeplan")
        else:
            _lib.check(_lib.lib.curig_nufft_makeplan(self.type, len(n_modes), n_modes[0],
                                                     n_modes[1] if len(n_modes) == 2 else 1, float(epsilon),
                                                     int(iflag), float(sigma), ctypes.byref(self._opts),
                                                     ctypes.byref(h)), "nufft_makeplan")
        self._h = h
        self._keep = None

    def setpts(self, x, y=None, z=None):
        """x (y, z): contiguous float64 CUDA tensors of the m point coordinates."""
        if len(self.n_modes) >= 2 and y is None or len(self.n_modes) == 3 and z is None:
            raise ValueError(f"{len(self.n_modes)}-dimensional transform needs {len(self.n_modes)} coordinates")
        self._keep = (x, y, z)
        self.m = int(x.shape[0])
        if len(self.n_modes) == 3:
            _lib.check(_lib.lib.curig_nufft3d_setpts(self._h, self.m, _lib.ptr(x), _lib.ptr(y), _lib.ptr(z)),
                       "nufft3d_setpts")
        else:
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


class Nufft3:
    """Type-3 NUFFT in one dimension: f_k = sum_j c_j exp(i iflag s_k x_j) for
    points x[m] with strengths c and frequencies s[n] (curig_nufft_setpts3)."""

    def __init__(self, epsilon, iflag=1, sigma=2.0, precision="fp64", stream=None):
        self.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self._opts = _lib.make_opts(self.precision, stream=_stream_handle(stream))
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.curig_nufft_makeplan(3, 1, 1, 1, float(epsilon), int(iflag), float(sigma),
                                                 ctypes.byref(self._opts), ctypes.byref(h)), "nufft_makeplan")
        self._h = h
        self._keep = None

    def setpts(self, x, s):
        """x [m] points and s [n] frequencies: contiguous float64 CUDA tensors."""
        self._keep = (x, s)
        self.m, self.n = int(x.shape[0]), int(s.shape[0])
        _lib.check(_lib.lib.curig_nufft_setpts3(self._h, self.m, _lib.ptr(x), self.n, _lib.ptr(s)), "nufft_setpts3")

    def info(self):
        nf = ctypes.c_int()
        d = (ctypes.c_double * 6)()
        _lib.check(_lib.lib.curig_nufft_info3(self._h, ctypes.byref(nf), d), "nufft_info3")
        return {"nf": nf.value, "i_center": d[0], "i_half": d[1], "o_center": d[2], "o_half": d[3],
                "gamma": d[4], "h": d[5]}

    def execute(self, c, f):
        """Reads the strengths c [m], writes f [n]."""
        _lib.check(_lib.lib.curig_nufft_execute(self._h, _lib.ptr(c), _lib.ptr(f)), "nufft_execute")

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib.curig_nufft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass
