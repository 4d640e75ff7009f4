"""Row-slab pipeline of the one-shot calls (curig_ms2dirty / curig_dirty2ms,
curig_opts.slabs): the sort key is slab-major, each slab's visibilities are
gathered and spread (ms2dirty) or interpolated and returned (dirty2ms) on
their own, so results must equal the single-slab call up to the order of the
grid's floating-point additions, and match the direct transform."""
import ctypes

import numpy as np
import pytest

from conftest import disk_inputs, l2err
from oracle import dft


def _call(kind, uvw, freq, vis, wgt, dirty, psx, eps, precision, slabs, window=0):
    from curig_b200 import _lib
    opts = _lib.make_opts(precision=1 if precision == "fp32" else 0, window=window, slabs=slabs)
    nrow, nchan = vis.shape
    nx, ny = dirty.shape
    f = _lib.lib.curig_ms2dirty if kind == 1 else _lib.lib.curig_dirty2ms
    st = f(nrow, nchan, nx, ny, psx, psx, np.ascontiguousarray(freq).ctypes.data, uvw.ctypes.data,
           vis.ctypes.data, None if wgt is None else wgt.ctypes.data, dirty.ctypes.data, eps, 2.0, -1,
           ctypes.byref(opts))
    _lib.check(st, "one-shot")


def _inputs(nrow, nchan, nx, precision, seed, with_wgt=True):
    freq, uvw, ms, wgt = disk_inputs(nrow, nchan, nx, 2.0, f0=0.9e9, fmax=1.1e9, max_pix=0.4 * nx, wmax=300,
                                     seed=seed)
    cdt, rdt = (np.complex64, np.float32) if precision == "fp32" else (np.complex128, np.float64)
    ms = np.ascontiguousarray(ms.astype(cdt))
    wgt = np.ascontiguousarray(wgt.astype(rdt)) if with_wgt else None
    img = np.random.default_rng(seed + 1).standard_normal((nx, nx)) + 1j * np.random.default_rng(seed + 2) \
        .standard_normal((nx, nx))
    return freq, np.ascontiguousarray(uvw), ms, wgt, np.ascontiguousarray(img.astype(cdt))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,eps,tol_same,tol_dft", [("fp64", 1e-9, 1e-12, 1e-8), ("fp32", 1e-5, 5e-6, 2e-5)])
@pytest.mark.parametrize("slabs", [2, 3, 8])
@pytest.mark.parametrize("with_wgt", [True, False])
def test_slabs_match_one_slab_and_dft(precision, eps, tol_same, tol_dft, slabs, with_wgt):
    nx = 128
    psx = 2.0 * np.pi / 180 / nx
    freq, uvw, ms, wgt, img = _inputs(20011, 3, nx, precision, 60 + slabs, with_wgt)
    d1 = np.zeros((nx, nx), dtype=ms.dtype)
    dk = np.zeros_like(d1)
    _call(1, uvw, freq, ms, wgt, d1, psx, eps, precision, 1)
    _call(1, uvw, freq, ms, wgt, dk, psx, eps, precision, slabs)
    assert l2err(d1, dk) < tol_same
    pix = np.random.default_rng(5).integers(0, nx * nx, 400)
    w64 = None if wgt is None else wgt.astype(np.float64)
    ref = dft.ms2dirty_dft(uvw, freq, ms.astype(np.complex128), w64, nx, nx, psx, psx, -1, pix=pix)
    assert l2err(ref, dk.ravel()[pix]) < tol_dft
    v1 = np.zeros_like(ms)
    vk = np.zeros_like(ms)
    _call(2, uvw, freq, v1, wgt, img, psx, eps, precision, 1)
    _call(2, uvw, freq, vk, wgt, img, psx, eps, precision, slabs)
    assert l2err(v1, vk) < tol_same
    idx = np.random.default_rng(6).integers(0, ms.size, 300)
    refv = dft.dirty2ms_dft(uvw, freq, img.astype(np.complex128), w64, psx, psx, -1, idx=idx)
    assert l2err(refv, vk.ravel()[idx]) < tol_dft


@pytest.mark.gpu
def test_more_slabs_than_rows():
    nx = 32
    psx = 1.0 * np.pi / 180 / nx
    freq, uvw, ms, wgt, img = _inputs(3, 2, nx, "fp64", 70)
    d1 = np.zeros((nx, nx), dtype=np.complex128)
    d8 = np.zeros_like(d1)
    _call(1, uvw, freq, ms, wgt, d1, psx, 1e-8, "fp64", 1)
    _call(1, uvw, freq, ms, wgt, d8, psx, 1e-8, "fp64", 8)
    assert l2err(d1, d8) < 1e-13
    v1 = np.zeros_like(ms)
    v8 = np.zeros_like(ms)
    _call(2, uvw, freq, v1, wgt, img, psx, 1e-8, "fp64", 1)
    _call(2, uvw, freq, v8, wgt, img, psx, 1e-8, "fp64", 8)
    assert l2err(v1, v8) < 1e-13


@pytest.mark.gpu
def test_automatic_slabs_at_a_larger_size():
    """6e6 FP32 visibilities with weights (72 MB): the automatic choice is two
    slabs; both directions against the single-slab call."""
    nx = 256
    psx = 2.0 * np.pi / 180 / nx
    freq, uvw, ms, wgt, img = _inputs(1_500_000, 4, nx, "fp32", 80)
    d1 = np.zeros((nx, nx), dtype=np.complex64)
    d0 = np.zeros_like(d1)
    _call(1, uvw, freq, ms, wgt, d1, psx, 1e-5, "fp32", 1)
    _call(1, uvw, freq, ms, wgt, d0, psx, 1e-5, "fp32", 0)
    assert l2err(d1, d0) < 5e-6
    v1 = np.zeros_like(ms)
    v0 = np.zeros_like(ms)
    _call(2, uvw, freq, v1, wgt, img, psx, 1e-5, "fp32", 1)
    _call(2, uvw, freq, v0, wgt, img, psx, 1e-5, "fp32", 0)
    assert l2err(v1, v0) < 1e-6


def test_slab_count_outside_range_is_rejected():
    from curig_b200 import _lib
    freq = np.array([1e9])
    uvw = np.zeros((4, 3))
    ms = np.zeros((4, 1), dtype=np.complex128)
    dirty = np.zeros((8, 8), dtype=np.complex128)
    for bad in (-1, 9):
        opts = _lib.make_opts(slabs=bad)
        st = _lib.lib.curig_ms2dirty(4, 1, 8, 8, 1e-3, 1e-3, freq.ctypes.data, uvw.ctypes.data, ms.ctypes.data,
                                     None, dirty.ctypes.data, 1e-6, 2.0, 1, ctypes.byref(opts))
        assert st == 3


@pytest.mark.gpu
def test_slabs_on_a_caller_stream_and_from_several_threads():
    """Three-slab one-shot calls on a caller-supplied CUDA stream, and from four
    host threads at once (each on its per-thread default stream): the same
    results as one-slab calls made one after another."""
    import threading

    import torch
    from curig_b200 import _lib
    nx = 96
    psx = 2.0 * np.pi / 180 / nx
    cases = [_inputs(12007, 2, nx, "fp64", 90 + k) for k in range(4)]

    def run(k, slabs, stream=None):
        freq, uvw, ms, wgt, img = cases[k]
        opts = _lib.make_opts(slabs=slabs, stream=stream)
        d = np.zeros((nx, nx), dtype=np.complex128)
        v = np.zeros_like(ms)
        for kind, vis, dirty in ((1, ms, d), (2, v, img)):
            f = _lib.lib.curig_ms2dirty if kind == 1 else _lib.lib.curig_dirty2ms
            st = f(ms.shape[0], ms.shape[1], nx, nx, psx, psx, np.ascontiguousarray(freq).ctypes.data,
                   uvw.ctypes.data, vis.ctypes.data, wgt.ctypes.data, dirty.ctypes.data, 1e-9, 2.0, -1,
                   ctypes.byref(opts))
            _lib.check(st, "one-shot")
        return d, v

    seq = [run(k, 1) for k in range(4)]
    s = torch.cuda.Stream()
    d, v = run(0, 3, s.cuda_stream)
    assert l2err(seq[0][0], d) < 1e-12 and l2err(seq[0][1], v) < 1e-12
    par = [None] * 4

    def worker(k):
        par[k] = run(k, 3)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for (d1, v1), (d3, v3) in zip(seq, par):
        assert l2err(d1, d3) < 1e-12 and l2err(v1, v3) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("fp32", 2e-6)])
@pytest.mark.parametrize("slabs", [1, 3])
def test_weighted_gather_with_and_without_scratch(precision, tol, slabs):
    """ms2dirty forms vis * wgt in input order into a scratch from the pool and
    gathers that into bin order; without the scratch (allocation failure, or
    the test hook) it gathers vis and wgt in one pass.  Both paths give the
    same image up to the rounding order of the two products."""
    from curig_b200 import _lib
    nx, nchan = 128, 4
    freq, uvw, ms, wgt, _ = _inputs(20000, nchan, nx, precision, seed=41)
    psx = 2.0 * np.pi / 180 / nx
    eps = 1e-9 if precision == "fp64" else 1e-5
    cdt = ms.dtype
    out = []
    try:
        for on in (1, 0):
            _lib.lib.curig_test_gather_scratch(on)
            dirty = np.zeros((nx, nx), dtype=cdt)
            _call(1, uvw, freq, ms, wgt, dirty, psx, eps, precision, slabs)
            out.append(dirty)
    finally:
        _lib.lib.curig_test_gather_scratch(1)
    assert l2err(out[0], out[1]) < tol
    assert np.linalg.norm(out[0]) > 0
