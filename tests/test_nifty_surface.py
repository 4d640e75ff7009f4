"""The Nifty-gridder surface in full (curig_b200.cursl): separate pixel sizes,
explicit oversampled grid sizes nx / ny, and do_wstacking=False (w ignored),
against the oracle DFT (oracle/dft.py, apply_w=False restating the Nifty
gridder's w-free explicit form: n - 1 = 0, n = 1)."""
import numpy as np
import pytest

from conftest import disk_inputs, l2err


def test_cursl_rejects_half_given_grid():
    import curig_b200 as C
    uvw = np.zeros((4, 3))
    ms = np.zeros((4, 1), dtype=np.complex128)
    with pytest.raises(ValueError):
        C.ms2dirty(uvw, np.array([1e9]), ms, None, 8, 8, 1e-3, 1e-3, 32, 0, 1e-6, True)


@pytest.mark.gpu
@pytest.mark.parametrize("eps,tol", [(1e-6, 1e-5), (1e-10, 1e-9)])
def test_no_wstacking_matches_w_free_dft(eps, tol):
    import curig_b200 as C
    from oracle import dft
    nx, ny = 64, 48
    freq, uvw, ms, wgt = disk_inputs(500, 2, nx, 4.0, max_pix=20, wmax=500, seed=3)
    psx, psy = 4.0 * np.pi / 180 / nx, 3.0 * np.pi / 180 / ny
    d = C.ms2dirty(uvw, freq, ms, wgt, nx, ny, psx, psy, 0, 0, eps, False)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, psx, psy, -1, apply_w=False).real
    assert l2err(ref, d) < tol
    img = np.random.default_rng(4).standard_normal((nx, ny))
    v = C.dirty2ms(uvw, freq, img, wgt, psx, psy, 0, 0, eps, False)
    vref = dft.dirty2ms_dft(uvw, freq, img + 0j, wgt, psx, psy, -1, apply_w=False)
    assert l2err(vref, v) < tol
    # the w term matters here: with w-stacking the answer differs from the w-free one
    dw = C.ms2dirty(uvw, freq, ms, wgt, nx, ny, psx, psy, 0, 0, eps, True)
    assert l2err(ref, dw) > 100 * tol


@pytest.mark.gpu
@pytest.mark.parametrize("grid,wst", [((160, 120), True), ((128, 96), True), ((200, 150), False),
                                      ((96, 72), True)])
def test_explicit_oversampled_grid(grid, wst):
    """nx, ny set the grid (sigma = min(nx/nxdirty, ny/nydirty) for the kernel rule)."""
    import curig_b200 as C
    from oracle import dft
    nx, ny = 64, 48
    freq, uvw, ms, wgt = disk_inputs(400, 1, nx, 3.0, max_pix=20, wmax=300, seed=5)
    psx, psy = 3.0 * np.pi / 180 / nx, 3.0 * np.pi / 180 / ny
    eps = 1e-7
    d = C.ms2dirty(uvw, freq, ms, wgt, nx, ny, psx, psy, grid[0], grid[1], eps, wst)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, psx, psy, -1, apply_w=wst).real
    assert l2err(ref, d) < 20 * eps


@pytest.mark.gpu
def test_separate_pixel_sizes_with_wstacking():
    import curig_b200 as C
    from oracle import dft
    nx, ny = 80, 40
    freq, uvw, ms, wgt = disk_inputs(300, 3, nx, 5.0, f0=0.9e9, fmax=1.1e9, max_pix=25, wmax=400, seed=6)
    psx, psy = 5.0 * np.pi / 180 / nx, 2.0 * np.pi / 180 / ny
    d = C.ms2dirty(uvw, freq, ms, wgt, nx, ny, psx, psy, 0, 0, 1e-8, True)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, psx, psy, -1).real
    assert l2err(ref, d) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("precision,eps,tol", [("fp64", 1e-10, 1e-12), ("fp32", 1e-5, 1e-5)])
def test_no_w_plan_adjointness_and_dft(precision, eps, tol):
    """Plan API with w_term=1: the two directions are adjoint and match the DFT."""
    import torch
    from curig_b200 import GridderPlan
    from oracle import dft
    nx = ny = 64
    freq, uvw, ms, wgt = disk_inputs(3000, 2, nx, 2.0, max_pix=25, wmax=300, seed=7)
    psx = 2.0 * np.pi / 180 / nx
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    rdt = torch.float64 if precision == "fp64" else torch.float32
    p = GridderPlan(1, nx, ny, psx, psx, eps, precision=precision, w_term=1)
    p.setpts(torch.from_numpy(uvw).cuda(), freq)
    v = torch.from_numpy(ms).to(cdt).cuda()
    w = torch.from_numpy(wgt).to(rdt).cuda()
    d = torch.empty((nx, ny), dtype=cdt, device="cuda")
    p.execute_dir(1, v, w, d)
    y = torch.from_numpy(np.random.default_rng(8).standard_normal((nx, ny)) + 0j).to(cdt).cuda()
    vo = torch.empty_like(v)
    p.execute_dir(2, vo, w, y)
    torch.cuda.synchronize()
    lhs = complex(torch.vdot(d.reshape(-1), y.reshape(-1)))
    rhs = complex(torch.vdot(v.reshape(-1), vo.reshape(-1)))
    assert abs(lhs - rhs) <= tol * abs(lhs) * 10
    pix = np.random.default_rng(9).integers(0, nx * ny, 300)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, psx, psx, -1, pix=pix, apply_w=False)
    assert l2err(ref, d.cpu().numpy().ravel()[pix]) < max(10 * eps, tol)
    p.close()


@pytest.mark.gpu
def test_bad_grid_requests_are_rejected():
    import curig_b200 as C
    from curig_b200._lib import CurigError
    freq, uvw, ms, wgt = disk_inputs(10, 1, 32, 2.0, seed=1)
    psx = 2.0 * np.pi / 180 / 32
    for nxg, nyg in ((31, 64), (16, 64), (64, 30)):        # odd, smaller than the image
        with pytest.raises(CurigError):
            C.ms2dirty(uvw, freq, ms, wgt, 32, 32, psx, psx, nxg, nyg, 1e-6, True)
