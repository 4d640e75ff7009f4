"""Nifty-gridder-compatible Python API, the RASCIL-facing surface
(python/curagridder/cursl.py:55-118).

As in the reference: sigma = 2, sign = -1, fov = rad_pix_x * nxdirty * 180/pi
(so the y pixel size is fov/nydirty, not rad_pix_y), ms2dirty returns the real
part of the dirty image, dirty2ms takes a real image and returns complex
visibilities shaped (nrow, 1).  nx, ny, do_wstacking and the extra arguments
are accepted and ignored, as there (improved w-stacking is always on).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .curagridder import _multichannel


def ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, rad_pix_x, rad_pix_y, nx, ny, epsilon,
             do_wstacking, *args):
    """Real dirty image [nxdirty, nydirty] of visibilities ms [nrow(, nchan)]."""
    nrow = uvw.shape[0]
    sigma = 2
    fov = rad_pix_x * nxdirty * 180 / np.pi
    dirty = np.zeros((nxdirty, nydirty), dtype=np.complex128)
    sign = -1
    if ms.ndim == 2 and ms.shape[1] > 1:
        _multichannel(1, uvw, freq, ms, wgt, dirty, fov, epsilon, sigma, sign)
        return dirty.real
    if wgt is None:
        st = _lib.ms2dirty_1(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, dirty, epsilon, sigma, sign)
    else:
        st = _lib.ms2dirty_2(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, wgt, dirty, epsilon, sigma,
                             sign)
    _lib.check(st, "ms2dirty")
    dirty = np.reshape(dirty, [nxdirty, nydirty])
    return dirty.real


def dirty2ms(uvw, freq, dirty, wgt, rad_pix_x, rad_pix_y, nx, ny, epsilon, do_wstacking, *args):
    """Complex visibilities (nrow, 1) of the real dirty image [nxdirty, nydirty]."""
    nrow = uvw.shape[0]
    nxdirty, nydirty = dirty.shape[0], dirty.shape[1]
    sigma = 2
    fov = rad_pix_x * nxdirty * 180 / np.pi
    sign = -1
    dirty1 = np.zeros(dirty.shape, dtype=np.complex128)
    dirty1.real = dirty
    nchan = len(freq) if wgt is None or wgt.ndim == 1 else wgt.shape[1]
    if nchan > 1:
        ms = np.zeros((nrow, nchan), dtype=np.complex128)
        return _multichannel(2, uvw, np.asarray(freq), ms, wgt, dirty1, fov, epsilon, sigma, sign)
    ms = np.zeros((nrow, 1), dtype=np.complex128)
    if wgt is None:
        st = _lib.dirty2ms_1(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, dirty1, epsilon, sigma, sign)
    else:
        st = _lib.dirty2ms_2(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, wgt, dirty1, epsilon, sigma,
                             sign)
    _lib.check(st, "dirty2ms")
    return ms
