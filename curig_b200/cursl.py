"""Nifty-gridder-compatible Python API, the RASCIL-facing surface
(python/curagridder/cursl.py:55-118 of the reference, names and argument
order kept).

The reference accepts nx, ny, rad_pix_y and do_wstacking and ignores them
(fov = rad_pix_x * nxdirty, sigma = 2, improved w-stacking always).  Here they
have the Nifty gridder's meaning:

* rad_pix_x, rad_pix_y: pixel sizes along the two image axes;
* nx, ny: the oversampled grid (even, >= nxdirty / nydirty); 0 keeps the
  reference's sigma = 2 sizing, and the kernel width follows the smaller
  oversampling ratio otherwise;
* do_wstacking=False: w is ignored (2-D gridding, no n - 1 term, no 1/n).

With nx = ny = 0, do_wstacking=True and rad_pix_y = rad_pix_x * nxdirty /
nydirty the result is the reference's.  As there: sign -1, ms2dirty returns
the real part of the dirty image, dirty2ms takes a real image and returns
complex visibilities (nrow, nchan); a wrong dtype raises ctypes.ArgumentError.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _as_2d(a, nrow):
    return None if a is None else a.reshape(nrow, -1)


def _check(name, a, dtype):
    if a is not None and (a.dtype != dtype or not a.flags.c_contiguous):
        raise ctypes.ArgumentError(f"{name}: expected a C-contiguous {np.dtype(dtype).name} array")


def _opts(nx, ny, do_wstacking):
    nx, ny = int(nx or 0), int(ny or 0)
    if (nx > 0) != (ny > 0):
        raise ValueError("nx and ny must both be given (> 0) or both be 0")
    return _lib.make_opts(precision=0, w_term=0 if do_wstacking else 1, grid_x=nx, grid_y=ny)


def ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, rad_pix_x, rad_pix_y, nx, ny, epsilon,
             do_wstacking, *args):
    """Real dirty image [nxdirty, nydirty] of visibilities ms [nrow(, nchan)]."""
    _check("uvw", uvw, np.float64)
    _check("ms", ms, np.complex128)
    _check("wgt", wgt, np.float64)
    nrow = uvw.shape[0]
    ms2, wgt2 = _as_2d(ms, nrow), _as_2d(wgt, nrow)
    nchan = ms2.shape[1]
    freq = np.ascontiguousarray(np.atleast_1d(freq)[:nchan], dtype=np.float64)
    dirty = np.zeros((nxdirty, nydirty), dtype=np.complex128)
    st = _lib.lib.curig_ms2dirty(nrow, nchan, nxdirty, nydirty, float(rad_pix_x), float(rad_pix_y),
                                 freq.ctypes.data, uvw.ctypes.data, ms2.ctypes.data,
                                 None if wgt2 is None else wgt2.ctypes.data, dirty.ctypes.data,
                                 float(epsilon), 2.0, -1, _opts(nx, ny, do_wstacking))
    _lib.check(st, "ms2dirty")
    return dirty.real


def dirty2ms(uvw, freq, dirty, wgt, rad_pix_x, rad_pix_y, nx, ny, epsilon, do_wstacking, *args):
    """Complex visibilities (nrow, nchan) of the real dirty image [nxdirty, nydirty]."""
    _check("uvw", uvw, np.float64)
    _check("wgt", wgt, np.float64)
    nrow = uvw.shape[0]
    nxdirty, nydirty = dirty.shape[0], dirty.shape[1]
    wgt2 = _as_2d(wgt, nrow)
    nchan = len(np.atleast_1d(freq)) if wgt2 is None else wgt2.shape[1]
    freq = np.ascontiguousarray(np.atleast_1d(freq)[:nchan], dtype=np.float64)
    dirty1 = np.zeros((nxdirty, nydirty), dtype=np.complex128)
    dirty1.real = dirty
    ms = np.zeros((nrow, nchan), dtype=np.complex128)
    st = _lib.lib.curig_dirty2ms(nrow, nchan, nxdirty, nydirty, float(rad_pix_x), float(rad_pix_y),
                                 freq.ctypes.data, uvw.ctypes.data, ms.ctypes.data,
                                 None if wgt2 is None else wgt2.ctypes.data, dirty1.ctypes.data,
                                 float(epsilon), 2.0, -1, _opts(nx, ny, do_wstacking))
    _lib.check(st, "dirty2ms")
    return ms
