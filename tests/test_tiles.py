"""Tile geometry paths against the DFT: w-plane slabs (bin_z, tiles that wrap the
w axis), odd bin edges (the tile's column shift varies from bin to bin), and
small bins (many wrapping tiles: plain tile loads and cell-by-cell flushes)."""
import numpy as np
import pytest

from conftest import disk_inputs, l2err


def _run(precision, eps, accumulate=0, **tile):
    import torch
    from curig_b200 import GridderPlan
    from oracle import dft
    nx, ny = 96, 80
    freq, uvw, ms, wgt = disk_inputs(4000, 2, nx, 3.0, f0=0.95e9, fmax=1.05e9, max_pix=40, wmax=800, seed=13)
    psx, psy = 3.0 * np.pi / 180 / nx, 3.0 * np.pi / 180 / ny
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    rdt = torch.float64 if precision == "fp64" else torch.float32
    p = GridderPlan(1, nx, ny, psx, psy, eps, precision=precision, accumulate=accumulate, **tile)
    p.setpts(torch.from_numpy(uvw).cuda(), freq)
    info = p.info()
    v = torch.from_numpy(ms).to(cdt).cuda()
    w = torch.from_numpy(wgt).to(rdt).cuda()
    d = torch.empty((nx, ny), dtype=cdt, device="cuda")
    p.execute_dir(1, v, w, d)
    img = np.random.default_rng(14).standard_normal((nx, ny)) + 0j
    vo = torch.empty_like(v)
    p.execute_dir(2, vo, w, torch.from_numpy(img).to(cdt).cuda())
    torch.cuda.synchronize()
    p.close()
    pix = np.random.default_rng(15).integers(0, nx * ny, 400)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, psx, psy, -1, pix=pix)
    idx = np.random.default_rng(16).integers(0, ms.size, 400)
    vref = dft.dirty2ms_dft(uvw, freq, img, wgt, psx, psy, -1, idx=idx)
    return (l2err(ref, d.cpu().numpy().ravel()[pix]), l2err(vref, vo.cpu().numpy().ravel()[idx]), info)


@pytest.mark.gpu
@pytest.mark.parametrize("bin_z", [1, 2, 4, 8])
@pytest.mark.parametrize("precision,eps,accumulate", [("fp64", 1e-9, 0), ("fp32", 1e-5, 2), ("fp32", 1e-5, 3)])
def test_w_slabs_match_dft(bin_z, precision, eps, accumulate):
    e1, e2, info = _run(precision, eps, accumulate, bin_z=bin_z)
    assert info["bin_z"] == bin_z and info["nf3"] > bin_z
    tol = 10 * eps if precision == "fp64" else 3e-5
    assert e1 < tol and e2 < tol


@pytest.mark.gpu
@pytest.mark.parametrize("bin_xy", [3, 7, 11, 15])
@pytest.mark.parametrize("precision,eps", [("fp64", 1e-7), ("fp32", 1e-5)])
def test_odd_and_small_bins_match_dft(bin_xy, precision, eps):
    """(A requested bin must fit the shared-memory budget: FP64 at kw = 8.)"""
    e1, e2, info = _run(precision, eps, bin_xy=bin_xy)
    assert info["bin_xy"] == bin_xy
    tol = 10 * eps if precision == "fp64" else 3e-5
    assert e1 < tol and e2 < tol


@pytest.mark.gpu
def test_bin_z_beyond_planes_is_rejected():
    from curig_b200._lib import CurigError
    with pytest.raises(CurigError):
        _run("fp64", 1e-6, bin_z=10000)
