"""Failure paths on the GPU without a GPU fault: a bounded wait made to run
out, and allocations beyond the device's memory.

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


def test_grid_beyond_device_memory_is_reported_and_context_survives():
    """Out of memory on the host's side of the call: a plan whose explicit
    oversampled grid (131072^2 FP64 cells, one plane: 275 GB) cannot be
    allocated returns status 6 from set points, before any kernel touches the
    grid; the plan is released and a normal plan afterwards is correct."""
    import torch

    import curig_b200._lib as L
    from curig_b200 import GridderPlan
    freq, uvw, ms, wgt = disk_inputs(500, 1, 64, 2.0, max_pix=25.0, seed=7)
    psx = 2.0 * np.pi / 180 / 64
    d_uvw = torch.from_numpy(np.ascontiguousarray(uvw)).cuda()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    big = GridderPlan(1, 64, 64, psx, psx, 1e-6, 2.0, -1, precision="fp64", window="es", w_term=1,
                      grid_x=131072, grid_y=131072)
    with pytest.raises(L.CurigError) as err:
        big.setpts(d_uvw, freq)
    assert err.value.code == 6, str(err.value)
    big.close()
    torch.cuda.synchronize()
    # the failed request leaves no device memory held (other processes need it)
    assert torch.cuda.mem_get_info()[0] > free0 - (1 << 30), (free0, torch.cuda.mem_get_info()[0])
    ok = GridderPlan(1, 64, 64, psx, psx, 1e-6, 2.0, -1, precision="fp64", window="es")
    ok.setpts(d_uvw, freq)
    d = torch.empty((64, 64), dtype=torch.complex128, device="cuda")
    ok.execute(torch.from_numpy(np.ascontiguousarray(ms)).cuda(), torch.from_numpy(np.ascontiguousarray(wgt)).cuda(), d)
    torch.cuda.synchronize()
    ok.close()
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, 64, 64, psx, psx, -1)
    assert l2err(ref, d.cpu().numpy()) < 1e-5


def test_one_shot_call_beyond_device_memory_then_a_normal_call():
    """The same through the one-shot ABI (host buffers): status 6 for the
    275 GB grid, then the same call with the default grid is correct."""
    import curig_b200._lib as L
    freq, uvw, ms, wgt = disk_inputs(500, 1, 64, 2.0, max_pix=25.0, seed=8)
    uvw = np.ascontiguousarray(uvw)
    ms, wgt = np.ascontiguousarray(ms), np.ascontiguousarray(wgt)
    psx = 2.0 * np.pi / 180 / 64
    out = np.zeros((64, 64), dtype=np.complex128)

    def call(opts):
        return L.lib.curig_ms2dirty(500, 1, 64, 64, psx, psx, freq.ctypes.data, uvw.ctypes.data, ms.ctypes.data,
                                    wgt.ctypes.data, out.ctypes.data, 1e-6, 2.0, -1, ctypes.byref(opts))

    import torch
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert call(L.make_opts(w_term=1, grid_x=131072, grid_y=131072)) == 6
    assert "memory" in L.lib.curig_last_error().decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] > free0 - (1 << 30), (free0, torch.cuda.mem_get_info()[0])
    st = call(L.make_opts())
    assert st == 0, L.lib.curig_last_error()
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, 64, 64, psx, psx, -1)
    assert l2err(ref, out) < 1e-5


def test_plan_api_reports_the_timed_out_tile_load():
    """The plan API leaves the device status to the caller: after a dirty2ms
    whose tile-load wait ran out, GridderPlan.status() raises status 4, and
    the next set points + execute are correct."""
    import torch

    import curig_b200._lib as L
    from curig_b200 import GridderPlan
    n, fov, eps = 256, 2.0, 1e-5
    freq, uvw, _, wgt = disk_inputs(20000, 1, n, fov, max_pix=110.0, seed=3)
    psx = fov * np.pi / 180 / n
    rng = np.random.default_rng(5)
    img = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    d_uvw = torch.from_numpy(np.ascontiguousarray(uvw)).cuda()
    d_wgt = torch.from_numpy(np.ascontiguousarray(wgt.astype(np.float32))).cuda()
    d_img = torch.from_numpy(img).cuda()
    p = GridderPlan(2, n, n, psx, psx, eps, 2.0, -1, precision="fp32", window="es")
    d_vis = torch.empty((20000, 1), dtype=torch.complex64, device="cuda")
    L.lib.curig_test_tile_wait(64, 1)            # loads never issued, 64 polls (taken at set points)
    try:
        p.setpts(d_uvw, freq)
        p.status()                               # nothing flagged yet
        p.execute(d_vis, d_wgt, d_img)
        with pytest.raises(L.CurigError) as err:
            p.status()
    finally:
        L.lib.curig_test_tile_wait(0, 0)
    assert err.value.code == 4 and "timed out" in str(err.value)
    p.setpts(d_uvw, freq)                        # set points clears the flags, regular wait
    p.execute(d_vis, d_wgt, d_img)
    p.status()
    vis = d_vis.cpu().numpy()
    p.close()
    ref = dft.dirty2ms_dft(uvw, freq, img.astype(np.complex128), wgt, psx, psx, -1)
    assert l2err(ref, vis) < 10 * eps
