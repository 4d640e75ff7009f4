"""ctypes front-end of the FP64 explicit-DFT oracle (oracle/dft.c).

TEST INFRASTRUCTURE ONLY.  Restates python/curagridder/test_wst.py:15-32 and
python/curagridder/explicit_test.py:32-54 of the reference (complex results;
the Nifty-flavour callers take ``.real`` of the gridder output).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import build_dft

_lib = None


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build",
                            "liboracle_dft.so")
        if not os.path.exists(path):
            path = build_dft()
        _lib = ctypes.CDLL(path)
        P = ctypes.c_void_p
        for name in ("oracle_ms2dirty_dft", "oracle_dirty2ms_dft"):
            f = getattr(_lib, name)
            f.restype = None
            f.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_double, ctypes.c_double, P, P, P, P, ctypes.c_int,
                          ctypes.c_int64, P, P]
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def pixel_n(nx, ny, pixsize_x, pixsize_y, pix=None):
    """n(l, m) = sqrt(1 - l^2 - m^2) of the pixels as dft.c computes it
    (integer centres nx/2, ny/2; n - 1 = -e / (sqrt(1 - e) + 1)), full
    [nx][ny] or the flat pixels in ``pix``."""
    p = np.arange(nx * ny, dtype=np.int64) if pix is None else np.asarray(pix, dtype=np.int64)
    x = (p // ny - nx // 2).astype(np.float64) * pixsize_x
    y = (p % ny - ny // 2).astype(np.float64) * pixsize_y
    e = x * x + y * y
    n = -e / (np.sqrt(1.0 - e) + 1.0) + 1.0
    return n.reshape(nx, ny) if pix is None else n


def _without_w(uvw):
    uvw = np.array(uvw, dtype=np.float64, copy=True)
    uvw[:, 2] = 0.0
    return uvw


def ms2dirty_dft(uvw, freqs, vis, wgt, nx, ny, pixsize_x, pixsize_y, sign, pix=None, apply_w=True):
    """Complex dirty values: full [nx][ny] image, or the flat pixels listed in ``pix``.
    apply_w=False: the Nifty gridder's w-free form (n - 1 = 0, n = 1): w set to
    zero and the 1/n of the w form undone."""
    if not apply_w:
        out = ms2dirty_dft(_without_w(uvw), freqs, vis, wgt, nx, ny, pixsize_x, pixsize_y, sign, pix)
        return out * pixel_n(nx, ny, pixsize_x, pixsize_y, pix)
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    freqs = np.ascontiguousarray(np.atleast_1d(freqs), dtype=np.float64)
    nrow, nchan = uvw.shape[0], freqs.shape[0]
    vis = np.ascontiguousarray(vis, dtype=np.complex128).reshape(nrow, nchan)
    wgt = None if wgt is None else np.ascontiguousarray(wgt, dtype=np.float64).reshape(nrow, nchan)
    if pix is None:
        out = np.empty((nx, ny), dtype=np.complex128)
        npix = nx * ny
    else:
        pix = np.ascontiguousarray(pix, dtype=np.int64)
        out = np.empty(pix.shape[0], dtype=np.complex128)
        npix = pix.shape[0]
    _load().oracle_ms2dirty_dft(nrow, nchan, nx, ny, pixsize_x, pixsize_y, _ptr(freqs),
                                _ptr(uvw), _ptr(vis), _ptr(wgt), int(sign), npix, _ptr(pix),
                                _ptr(out))
    return out


def dirty2ms_dft(uvw, freqs, dirty, wgt, pixsize_x, pixsize_y, sign, idx=None, apply_w=True):
    """Complex visibilities [nrow][nchan], or the flat (row*nchan+chan) ones in ``idx``.
    apply_w=False: the w-free form (w = 0, no division by n)."""
    if not apply_w:
        d = np.asarray(dirty, dtype=np.complex128)
        return dirty2ms_dft(_without_w(uvw), freqs, d * pixel_n(d.shape[0], d.shape[1], pixsize_x, pixsize_y),
                            wgt, pixsize_x, pixsize_y, sign, idx)
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    freqs = np.ascontiguousarray(np.atleast_1d(freqs), dtype=np.float64)
    nrow, nchan = uvw.shape[0], freqs.shape[0]
    dirty = np.ascontiguousarray(dirty, dtype=np.complex128)
    nx, ny = dirty.shape
    wgt = None if wgt is None else np.ascontiguousarray(wgt, dtype=np.float64).reshape(nrow, nchan)
    if idx is None:
        out = np.empty((nrow, nchan), dtype=np.complex128)
        nvis = nrow * nchan
    else:
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        out = np.empty(idx.shape[0], dtype=np.complex128)
        nvis = idx.shape[0]
    _load().oracle_dirty2ms_dft(nrow, nchan, nx, ny, pixsize_x, pixsize_y, _ptr(freqs),
                                _ptr(uvw), _ptr(dirty), _ptr(wgt), int(sign), nvis, _ptr(idx),
                                _ptr(out))
    return out
