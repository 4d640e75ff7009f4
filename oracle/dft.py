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


def ms2dirty_dft(uvw, freqs, vis, wgt, nx, ny, pixsize_x, pixsize_y, sign, pix=None):
    """Complex dirty values: full [nx][ny] image, or the flat pixels listed in ``pix``."""
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


def dirty2ms_dft(uvw, freqs, dirty, wgt, pixsize_x, pixsize_y, sign, idx=None):
    """Complex visibilities [nrow][nchan], or the flat (row*nchan+chan) ones in ``idx``."""
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
