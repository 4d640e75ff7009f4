"""Failure paths on the GPU without a GPU fault.

The interpolator stages interior tiles with TMA box loads and waits on an
mbarrier for at most a bounded number of polls; when the wait runs out, the
CTA raises an error flag and leaves, and the one-shot call returns status 4
with a "timed out" message.  Here the wait is made to run out on purpose: the
test hook arms the barrier without issuing the load (nothing is in flight when
the CTA leaves) and shortens the poll limit.  A normal call afterwards must
succeed and be correct, so the context stays usable."""
import ctypes

import numpy as np
import pytest

from conftest import disk_inputs, l2err
from oracle import dft

pytestmark = pytest.mark.gpu


def _dirty2ms(L, uvw, freq, img, wgt, n, psx, eps):
    nrow = uvw.shape[0]
    vis = np.zeros((nrow, 1), dtype=np.complex64)
    opts = L.make_opts(precision=1)
    st = L.lib.curig_dirty2ms(nrow, 1, n, n, psx, psx, freq.ctypes.data, uvw.ctypes.data, vis.ctypes.data,
                              wgt.ctypes.data, img.ctypes.data, eps, 2.0, -1, ctypes.byref(opts))
    return st, vis


def test_tile_load_wait_runs_out_and_context_survives():
    import curig_b200._lib as L
    n, fov, eps = 256, 2.0, 1e-5
    freq, uvw, _, wgt = disk_inputs(20000, 1, n, fov, max_pix=110.0, seed=3)
    uvw = np.ascontiguousarray(uvw)
    wgt = np.ascontiguousarray(wgt.astype(np.float32))
    rng = np.random.default_rng(4)
    img = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    psx = fov * np.pi / 180 / n
    L.lib.curig_test_tile_wait(64, 1)           # loads never issued, 64 polls
    try:
        st, _ = _dirty2ms(L, uvw, freq, img, wgt, n, psx, eps)
    finally:
        L.lib.curig_test_tile_wait(0, 0)
    assert st == 4, st
    assert "timed out" in L.lib.curig_last_error().decode()
    st, vis = _dirty2ms(L, uvw, freq, img, wgt, n, psx, eps)
    assert st == 0, L.lib.curig_last_error()
    ref = dft.dirty2ms_dft(uvw, freq, img.astype(np.complex128), wgt.astype(np.float64), psx, psx, -1)
    assert l2err(ref, vis) < 10 * eps
