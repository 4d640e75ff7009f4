"""Reference-flavour Python API (python/curagridder/curagridder.py:69-128).

vis2dirty / dirty2vis call the same C entry points with the same arguments as
the reference (sign +1, sigma default 1.25, freq[0], fov in degrees), filling
the caller's array in place and returning it.  With more than one channel the
call goes through curig_ms2dirty / curig_dirty2ms, which transform all
channels in one pass (the reference reads only channel 0's frequency).
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _nchan(ms):
    return 1 if ms.ndim == 1 else ms.shape[1]


def vis2dirty(uvw, freq, ms, wgt, dirty, fov, epsilon=1e-6, sigma=1.25):
    """Dirty image [nxdirty, nydirty] (complex128, written into ``dirty``)."""
    nrow = uvw.shape[0]
    nxdirty, nydirty = dirty.shape[0], dirty.shape[1]
    sign = 1
    if _nchan(ms) > 1:
        return _multichannel(1, uvw, freq, ms, wgt, dirty, fov, epsilon, sigma, sign)
    if wgt is None:
        st = _lib.ms2dirty_1(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, dirty, epsilon, sigma, sign)
    else:
        st = _lib.ms2dirty_2(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, wgt, dirty, epsilon, sigma,
                             sign)
    _lib.check(st, "ms2dirty")
    return dirty


def dirty2vis(uvw, freq, ms, wgt, dirty, fov, epsilon=1e-6, sigma=1.25):
    """Visibilities [nrow(, nchan)] (complex128, written into ``ms``)."""
    nrow = uvw.shape[0]
    nxdirty, nydirty = dirty.shape[0], dirty.shape[1]
    sign = 1
    if _nchan(ms) > 1:
        return _multichannel(2, uvw, freq, ms, wgt, dirty, fov, epsilon, sigma, sign)
    if wgt is None:
        st = _lib.dirty2ms_1(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, dirty, epsilon, sigma, sign)
    else:
        st = _lib.dirty2ms_2(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, wgt, dirty, epsilon, sigma,
                             sign)
    _lib.check(st, "dirty2ms")
    return ms


def _multichannel(kind, uvw, freq, ms, wgt, dirty, fov, epsilon, sigma, sign):
    nrow, nchan = ms.shape
    nx, ny = dirty.shape
    psx = fov / 180.0 * np.pi / nx
    psy = fov / 180.0 * np.pi / ny
    freq = np.ascontiguousarray(freq[:nchan], dtype=np.float64)
    for a, t in ((uvw, np.float64), (ms, np.complex128), (dirty, np.complex128)):
        if a.dtype != t or not a.flags.c_contiguous:
            raise TypeError("uvw, ms and dirty must be C-contiguous float64 / complex128")
    if wgt is not None and (wgt.dtype != np.float64 or not wgt.flags.c_contiguous):
        raise TypeError("wgt must be C-contiguous float64")
    opts = _lib.make_opts(precision=0)
    f = _lib.lib.curig_ms2dirty if kind == 1 else _lib.lib.curig_dirty2ms
    st = f(nrow, nchan, nx, ny, psx, psy, freq.ctypes.data, uvw.ctypes.data, ms.ctypes.data,
           None if wgt is None else wgt.ctypes.data, dirty.ctypes.data, epsilon, sigma, sign, opts)
    _lib.check(st, "ms2dirty" if kind == 1 else "dirty2ms")
    return dirty if kind == 1 else ms
