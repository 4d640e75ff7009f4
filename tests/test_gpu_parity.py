"""GPU parity: the CUDA path against the oracle (FP64 DFT and the NUFFT
restatement of the reference), the reference library's own recorded outputs,
and the reference's adjointness test, all through the C ABI."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, disk_inputs, l2err, wst_inputs
from oracle import dft, nufft
from oracle import params as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def C():
    import curig_b200
    return curig_b200


# ---------------------------------------------------------------- reference ABI vs oracle
CASES = [  # nrow, nx, ny, fov, eps, sign, wgt
    (100, 30, 128, 10, 5e-7, -1, True), (27, 16, 64, 20, 5e-3, -1, False),
    (100, 128, 250, 1, 5e-12, -1, True), (200, 64, 64, 2, 1e-6, 1, True),
    (2, 30, 64, 10, 5e-5, -1, True), (500, 96, 80, 5, 1e-9, 1, False),
    (300, 64, 64, 20, 2e-1, -1, True)]


@pytest.mark.parametrize("nrow,nx,ny,fov,eps,sign,use_wgt", CASES)
def test_reference_abi_matches_oracle(C, nrow, nx, ny, fov, eps, sign, use_wgt):
    freq, uvw, ms, dirty, wgt = wst_inputs(nrow, 1, nx, ny, fov, wgt=use_wgt)
    xps, yps = P.pixel_sizes(fov, nx, ny)
    out = np.zeros((nx, ny), dtype=np.complex128)
    if sign == 1:
        C.vis2dirty(uvw, freq, ms, wgt, out, fov, eps, 2.0)
        got_d = out
    else:
        got_d = None
        import curig_b200._lib as L
        st = (L.ms2dirty_2(nrow, nx, ny, fov, freq[0], uvw, ms, wgt, out, eps, 2.0, sign) if use_wgt
              else L.ms2dirty_1(nrow, nx, ny, fov, freq[0], uvw, ms, out, eps, 2.0, sign))
        assert st == 0
        got_d = out
    ref_nu = nufft.ms2dirty(uvw, freq, ms, wgt, nx, ny, fov, eps, 2.0, sign)
    ref_ex = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, xps, yps, sign)
    # same algorithm, same sizes: agreement far below eps (FP64 rounding only)
    assert l2err(ref_nu, got_d) < 1e-10
    assert l2err(ref_ex, got_d) < max(10 * eps, 1e-12)
    vis = np.zeros((nrow, 1), dtype=np.complex128)
    cd = dirty.astype(np.complex128)
    import curig_b200._lib as L
    st = (L.dirty2ms_2(nrow, nx, ny, fov, freq[0], uvw, vis, wgt, cd, eps, 2.0, sign) if use_wgt
          else L.dirty2ms_1(nrow, nx, ny, fov, freq[0], uvw, vis, cd, eps, 2.0, sign))
    assert st == 0
    ref_nu = nufft.dirty2ms(uvw, freq, dirty, wgt, nx, ny, fov, eps, 2.0, sign)
    ref_ex = dft.dirty2ms_dft(uvw, freq, dirty, wgt, xps, yps, sign)
    assert l2err(ref_nu, vis) < 1e-10
    assert l2err(ref_ex, vis) < max(10 * eps, 1e-12)


# ---------------------------------------------------------------- the reference's own test
@pytest.mark.parametrize("nrow", (2, 27, 100))
@pytest.mark.parametrize("nxdirty", (30, 128, 16))
@pytest.mark.parametrize("nydirty", (128, 250, 64))
@pytest.mark.parametrize("fov", (1, 10, 20))
@pytest.mark.parametrize("epsilon", (2e-1, 5e-3, 5e-5, 5e-7, 5e-12))
@pytest.mark.parametrize("use_wgt", (False, True))
def test_against_wdft(C, nrow, nxdirty, nydirty, fov, epsilon, use_wgt):
    """python/curagridder/test_wst.py:36-83: adjointness at rtol 1e-12 (asserted
    there) plus the L2 error against the explicit DFT (printed there, asserted here)."""
    freq, uvw, ms, dirty, wgt = wst_inputs(nrow, 1, nxdirty, nydirty, fov, wgt=use_wgt)
    xpixsize = fov * np.pi / 180 / nxdirty
    ypixsize = fov * np.pi / 180 / nydirty
    dirty2 = C.ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, xpixsize, ypixsize, 0, 0, epsilon, True, 4)
    ms2 = C.dirty2ms(uvw, freq, dirty, wgt, xpixsize, ypixsize, 0, 0, epsilon, True, 4)
    np.testing.assert_allclose(np.vdot(ms, ms2).real, np.vdot(dirty2, dirty), rtol=1e-12)
    msw = ms * wgt if use_wgt else ms
    truth = dft.ms2dirty_dft(uvw, freq, msw, None, nxdirty, nydirty, xpixsize, ypixsize, -1).real
    assert l2err(truth, dirty2) < max(10 * epsilon, 1e-12)


# ---------------------------------------------------------------- recorded reference outputs
def _reflib():
    # single-call fixtures (inputs stored); the 4096^2 ones are in test_configs_at_size.py
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "reflib_*.npz"))
                  if not os.path.basename(p).startswith("reflib_cfg2_"))


@pytest.mark.parametrize("path", _reflib(), ids=os.path.basename)
def test_matches_reference_library_outputs(C, path):
    g = np.load(path)
    import curig_b200._lib as L
    nx, ny = int(g["nx"]), int(g["ny"])
    uvw, freq, ms, dirty = g["uvw"], g["freq"], g["ms"], g["dirty"]
    wgt = g["wgt"] if g["wgt"].size else None
    fov, eps, sigma, sign = float(g["fov"]), float(g["eps"]), float(g["sigma"]), int(g["sign"])
    out = np.zeros((nx, ny), dtype=np.complex128)
    vis = np.zeros((uvw.shape[0], 1), dtype=np.complex128)
    n = uvw.shape[0]
    if wgt is None:
        assert L.ms2dirty_1(n, nx, ny, fov, freq[0], uvw, ms, out, eps, sigma, sign) == 0
        assert L.dirty2ms_1(n, nx, ny, fov, freq[0], uvw, vis, dirty, eps, sigma, sign) == 0
    else:
        assert L.ms2dirty_2(n, nx, ny, fov, freq[0], uvw, ms, wgt, out, eps, sigma, sign) == 0
        assert L.dirty2ms_2(n, nx, ny, fov, freq[0], uvw, vis, wgt, dirty, eps, sigma, sign) == 0
    # the reference differs from us only by rounding (same sizes, kernel and quadrature)
    tol = max(1e-9, 1e-3 * eps)
    assert l2err(g["ms2dirty"], out) < tol
    assert l2err(g["dirty2ms"], vis) < tol


# ---------------------------------------------------------------- 256^2, 2000 vis, eps 1e-6
def test_disk2000_256_against_reference_truth(C):
    g = np.load(os.path.join(GOLDEN, "refdft_disk2000_256x256.npz"))
    xps = float(g["xpixsize"])
    d = C.ms2dirty(g["uvw"], g["freq"], g["ms"], g["wgt"], 256, 256, xps, xps, 0, 0, 1e-6, True)
    assert l2err(g["gridder_sign_m1"], d) < 1e-5


# ---------------------------------------------------------------- multi-channel, FP32, plan API
def _plan_run(kind, nx, ny, psx, psy, eps, sign, uvw, freq, vis=None, wgt=None, dirty=None,
              precision="fp64", window="es", accumulate=0, sub=0, sparse=0):
    import torch
    from curig_b200 import GridderPlan
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    rt = torch.float64 if precision == "fp64" else torch.float32
    p = GridderPlan(kind, nx, ny, psx, psy, eps, 2.0, sign, precision=precision, window=window,
                    accumulate=accumulate, sub=sub, sparse=sparse)
    d_uvw = torch.from_numpy(np.ascontiguousarray(uvw)).cuda()
    p.setpts(d_uvw, freq)
    nrow, nchan = uvw.shape[0], len(freq)
    d_wgt = None if wgt is None else torch.from_numpy(np.ascontiguousarray(wgt)).to(rt).cuda()
    if kind == 1:
        d_vis = torch.from_numpy(np.ascontiguousarray(vis)).to(dt).cuda()
        d_dirty = torch.empty((nx, ny), dtype=dt, device="cuda")
        p.execute(d_vis, d_wgt, d_dirty)
        torch.cuda.synchronize()
        out = d_dirty.cpu().numpy()
    else:
        d_dirty = torch.from_numpy(np.ascontiguousarray(dirty)).to(dt).cuda()
        d_vis = torch.empty((nrow, nchan), dtype=dt, device="cuda")
        p.execute(d_vis, d_wgt, d_dirty)
        torch.cuda.synchronize()
        out = d_vis.cpu().numpy()
    info = p.info()
    p.close()
    return out, info


# sparse: 0 the default split (chunks below 128 (FP32) or 64 (FP64) visibilities
# straight to the grid, one warp per visibility), -1 every chunk through a tile, 1 << 30 no tile
@pytest.mark.parametrize("sparse", [0, -1, 1 << 30])
@pytest.mark.parametrize("accumulate", [0, 1, 2, 3])
@pytest.mark.parametrize("precision,eps,tol", [("fp64", 1e-9, 1e-8), ("fp64", 1e-5, 1e-4),
                                               ("fp32", 1e-5, 2e-5), ("fp32", 1e-4, 2e-4)])
def test_multichannel_plan_vs_dft(C, precision, eps, tol, accumulate, sparse):
    freq, uvw, ms, wgt = disk_inputs(3000, 4, 128, 2.0, f0=0.9e9, fmax=1.1e9, max_pix=60, wmax=300)
    psx = psy = 2.0 * np.pi / 180 / 128
    d, info = _plan_run(1, 128, 128, psx, psy, eps, -1, uvw, freq, vis=ms, wgt=wgt, precision=precision,
                        accumulate=accumulate, sparse=sparse)
    pix = np.random.default_rng(1).integers(0, 128 * 128, 600)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, 128, 128, psx, psy, -1, pix=pix)
    assert l2err(ref, d.ravel()[pix]) < tol
    img = np.random.default_rng(2).standard_normal((128, 128)) + 0j
    v, _ = _plan_run(2, 128, 128, psx, psy, eps, -1, uvw, freq, dirty=img, wgt=wgt, precision=precision)
    idx = np.random.default_rng(3).integers(0, uvw.shape[0] * len(freq), 300)
    refv = dft.dirty2ms_dft(uvw, freq, img, wgt, psx, psy, -1, idx=idx)
    assert l2err(refv, v.ravel()[idx]) < tol


def test_plan_repeated_execute_is_stable(C):
    import torch
    from curig_b200 import GridderPlan
    freq, uvw, ms, wgt = disk_inputs(5000, 2, 96, 3.0)
    psx = 3.0 * np.pi / 180 / 96
    p = GridderPlan(1, 96, 96, psx, psx, 1e-6, 2.0, 1, precision="fp64")
    p.setpts(torch.from_numpy(uvw).cuda(), freq)
    v = torch.from_numpy(ms).cuda()
    w = torch.from_numpy(wgt).cuda()
    outs = []
    for _ in range(3):
        d = torch.empty((96, 96), dtype=torch.complex128, device="cuda")
        p.execute(v, w, d)
        outs.append(d.cpu().numpy())
    assert l2err(outs[0], outs[1]) < 1e-13 and l2err(outs[0], outs[2]) < 1e-13


def test_odd_image_sizes_vs_dft(C):
    freq, uvw, ms, wgt = disk_inputs(400, 1, 33, 4.0, max_pix=12)
    psx, psy = 4.0 * np.pi / 180 / 33, 4.0 * np.pi / 180 / 21
    d, _ = _plan_run(1, 33, 21, psx, psy, 1e-8, 1, uvw, freq, vis=ms, wgt=wgt)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, 33, 21, psx, psy, 1)
    assert l2err(ref, d) < 1e-7


def test_nonfinite_uvw_is_rejected(C):
    import curig_b200._lib as L
    freq, uvw, ms, dirty, wgt = wst_inputs(20, 1, 16, 16, 2)
    uvw[3, 1] = np.nan
    out = np.zeros((16, 16), dtype=np.complex128)
    assert L.ms2dirty_1(20, 16, 16, 2.0, 1e9, uvw, ms, out, 1e-6, 2.0, 1) == 7
    uvw[3, 1] = 0.0
    uvw[5, 2] = np.inf
    assert L.ms2dirty_1(20, 16, 16, 2.0, 1e9, uvw, ms, out, 1e-6, 2.0, 1) == 7


def test_bad_sigma_is_rejected(C):
    import curig_b200._lib as L
    freq, uvw, ms, dirty, wgt = wst_inputs(20, 1, 16, 16, 2)
    out = np.zeros((16, 16), dtype=np.complex128)
    assert L.ms2dirty_1(20, 16, 16, 2.0, 1e9, uvw, ms, out, 1e-6, 1.0, 1) == 2


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_fixed_point_accumulation_matches_float(C, precision):
    """Integer (fixed-point) tile accumulation against the floating-point one on
    a dense case (many visibilities per cell)."""
    freq, uvw, ms, wgt = disk_inputs(200000, 2, 64, 2.0, max_pix=24, wmax=300)
    psx = 2.0 * np.pi / 180 / 64
    d0, _ = _plan_run(1, 64, 64, psx, psx, 1e-6, 1, uvw, freq, vis=ms, wgt=wgt, precision=precision,
                      accumulate=3)
    d2, _ = _plan_run(1, 64, 64, psx, psx, 1e-6, 1, uvw, freq, vis=ms, wgt=wgt, precision=precision,
                      accumulate=1)
    assert l2err(d0, d2) < (2e-6 if precision == "fp32" else 1e-12)


@pytest.mark.parametrize("sub,tol", [(0, 3e-6), (4096, 3e-6), (256, 3e-6), (16384, 3e-6), (65536, 8e-6)])
def test_one_word_fixed_point_matches_exact(C, sub, tol):
    """One-word int32 tile accumulation (22-bit terms) against the exact two-word
    one on a dense case (about 4e5 visibilities in a few bins, chunks of up to
    the chunk size; 0 = the default, 16384 for one-word tiles): nothing may
    overflow and the error stays at the 22-bit rounding level.  A requested
    chunk of 65536 puts a whole bin in one chunk; its box bound binds and the
    rounding step grows with it."""
    freq, uvw, ms, wgt = disk_inputs(200000, 2, 64, 2.0, max_pix=24, wmax=300)
    psx = 2.0 * np.pi / 180 / 64
    d0, _ = _plan_run(1, 64, 64, psx, psx, 1e-6, 1, uvw, freq, vis=ms, wgt=wgt, precision="fp32",
                      accumulate=3)
    d1, _ = _plan_run(1, 64, 64, psx, psx, 1e-6, 1, uvw, freq, vis=ms, wgt=wgt, precision="fp32",
                      accumulate=2, sub=sub)
    assert l2err(d0, d1) < tol


@pytest.mark.parametrize("n", [4000, 16000])
def test_one_word_fixed_point_all_in_one_cell(C, n):
    """Every visibility at the same uv point (4000; 16000, one bin below the
    one-word chunk size of 16384, which the binning still cuts into chunks of at
    most 4096 because they all share one start-cell residue class): the box
    bound must scale each chunk so that no int32 cell sum overflows, and the
    rounding error (growing with the visibilities per chunk) stays below
    epsilon."""
    rng = np.random.default_rng(7)
    uvw = np.tile(np.array([[120.0, -80.0, 15.0]]), (n, 1))
    freq = np.array([1.0e9])
    ms = (rng.standard_normal((n, 1)) + 1j * rng.standard_normal((n, 1))).astype(np.complex128)
    wgt = np.ones((n, 1))
    psx = 1.0 * np.pi / 180 / 64
    d3, _ = _plan_run(1, 64, 64, psx, psx, 1e-5, -1, uvw, freq, vis=ms, wgt=wgt, precision="fp32", accumulate=3)
    d2, _ = _plan_run(1, 64, 64, psx, psx, 1e-5, -1, uvw, freq, vis=ms, wgt=wgt, precision="fp32", accumulate=2)
    assert l2err(d3, d2) < 1e-5


def test_fp64_fixed_point_all_in_one_cell_wide_range(C):
    """FP64 three-word int32 tiles: a 4000-visibility chunk at one uv point with
    magnitudes over sixteen decades (the chunk scale follows the largest; the
    high words of one cell take every term) against double atomics."""
    rng = np.random.default_rng(8)
    n = 4000
    uvw = np.tile(np.array([[120.0, -80.0, 15.0]]), (n, 1))
    freq = np.array([1.0e9])
    mag = 10.0 ** rng.uniform(-8, 8, (n, 1))
    ms = mag * (rng.standard_normal((n, 1)) + 1j * rng.standard_normal((n, 1)))
    wgt = np.ones((n, 1))
    psx = 1.0 * np.pi / 180 / 64
    d0, _ = _plan_run(1, 64, 64, psx, psx, 1e-9, -1, uvw, freq, vis=ms, wgt=wgt, accumulate=0)
    d1, _ = _plan_run(1, 64, 64, psx, psx, 1e-9, -1, uvw, freq, vis=ms, wgt=wgt, accumulate=1)
    assert l2err(d1, d0) < 1e-13


def test_bad_accumulate_option_is_rejected(C):
    from curig_b200 import GridderPlan
    from curig_b200._lib import CurigError
    with pytest.raises(CurigError):
        GridderPlan(1, 32, 32, 1e-4, 1e-4, 1e-5, precision="fp32", accumulate=4)
