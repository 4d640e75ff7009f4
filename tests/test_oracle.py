"""CPU tests: the oracle is pinned against the reference's own truth functions
(golden vectors from tests/golden/make_golden.py), its parameter rules against
the reference's documented sizes, and its NUFFT restatement against the DFT."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, l2err, wst_inputs
from oracle import dft, nufft
from oracle import params as P


@pytest.mark.parametrize("n", [2, 3, 10, 22, 27, 64, 88])
def test_gauss_legendre_matches_numpy(n):
    x, w = P.gauss_legendre(n)
    xr, wr = np.polynomial.legendre.leggauss(n)
    assert np.max(np.abs(x - xr)) < 1e-14
    assert np.max(np.abs(w - wr)) < 1e-13


def _brute235(n):
    m = max(n, 2)
    m += m % 2
    while True:
        k = m
        for f in (2, 3, 5):
            while k % f == 0:
                k //= f
        if k == 1:
            return m
        m += 2


@pytest.mark.parametrize("n", list(range(0, 80)) + [97, 511, 1000, 4097, 8191])
def test_next235_matches_definition(n):
    assert P.next235even(n) == _brute235(n)


@pytest.mark.parametrize("eps,kw,beta", [(2e-1, 2, 4.4), (5e-3, 4, 9.52), (1e-4, 5, 11.5),
                                         (1e-5, 6, 13.8), (1e-6, 7, 16.1), (5e-12, 13, 29.9)])
def test_kernel_width_rule(eps, kw, beta):
    o = P.setup_conv_opts(eps, 2.0)
    assert o.kw == kw
    assert abs(o.beta - beta) < 1e-12


def test_config_sizes():
    """Sizes the survey derives for the 256^2 and 4096^2 configurations."""
    # 256x256, fov 2 deg, eps 1e-6, w +-200 m at 1 GHz
    w = 200 * 1e9 / P.SPEEDOFLIGHT * 2 * np.pi
    prm = P.gridder_params(256, 256, 2.0, None, None, 1e-6, 2.0, 1, w_range=(-w, w))
    assert (prm.nf1, prm.nf2, prm.nf3, prm.opts.kw) == (512, 512, 16, 7)
    # 4096x4096, fov 3 deg, w +-1000 m at 1.1 GHz
    w = 1000 * 1.1e9 / P.SPEEDOFLIGHT * 2 * np.pi
    for eps, kw, nf3 in [(1e-4, 5, 16), (1e-5, 6, 18), (1e-6, 7, 18)]:
        prm = P.gridder_params(4096, 4096, 3.0, None, None, eps, 2.0, 1, w_range=(-w, w))
        assert (prm.nf1, prm.nf3, prm.opts.kw) == (8192, nf3, kw)


def _golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "refdft_*.npz")))


@pytest.mark.parametrize("path", _golden_files(), ids=os.path.basename)
def test_oracle_dft_matches_reference_truth(path):
    """oracle/dft.c against the reference's numpy explicit_gridder /
    explicit_degridder outputs (test_wst.py:15-32, test_ws.py, explicit_test.py:32-54)."""
    g = np.load(path)
    uvw, freq, ms = g["uvw"], g["freq"], g["ms"]
    wgt = g["wgt"] if g["wgt"].size else None
    nx, ny = g["gridder_sign_m1"].shape
    msw = ms * wgt if wgt is not None else ms
    xps, yps = float(g["xpixsize"]), float(g["ypixsize"])
    got = dft.ms2dirty_dft(uvw, freq, msw, None, nx, ny, xps, yps, -1)
    assert l2err(g["gridder_sign_m1"], got.real) < 1e-12
    if "gridder_sign_p1" in g:
        got = dft.ms2dirty_dft(uvw, freq, msw, None, nx, ny, xps, yps, +1)
        assert l2err(g["gridder_sign_p1"], got.real) < 1e-12
    if "degridder_sign_m1" in g:
        got = dft.dirty2ms_dft(uvw, freq, g["dirty"], None, xps, yps, -1)
        assert l2err(g["degridder_sign_m1"], got.ravel()) < 1e-12


@pytest.mark.parametrize("nrow,nx,ny,fov,eps,sign", [
    (100, 30, 128, 10, 5e-7, -1), (27, 16, 64, 20, 5e-3, -1), (100, 128, 64, 1, 5e-5, 1),
    (200, 64, 64, 2, 1e-10, 1), (60, 32, 32, 10, 2e-1, -1)])
def test_oracle_nufft_vs_dft(nrow, nx, ny, fov, eps, sign):
    freq, uvw, ms, dirty, wgt = wst_inputs(nrow, 1, nx, ny, fov)
    xps, yps = P.pixel_sizes(fov, nx, ny)
    d_nu = nufft.ms2dirty(uvw, freq, ms, wgt, nx, ny, fov, eps, 2.0, sign)
    d_ex = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, xps, yps, sign)
    tol = max(10 * eps, 1e-13)
    assert l2err(d_ex, d_nu) < tol
    v_nu = nufft.dirty2ms(uvw, freq, dirty, wgt, nx, ny, fov, eps, 2.0, sign)
    v_ex = dft.dirty2ms_dft(uvw, freq, dirty, wgt, xps, yps, sign)
    assert l2err(v_ex, v_nu) < tol
    # adjointness as asserted by test_wst.py:77
    lhs = np.vdot(ms, v_nu).real
    rhs = np.vdot(d_nu.real, dirty)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_oracle_multichannel_is_sum_of_channels():
    freq, uvw, ms, dirty, wgt = wst_inputs(80, 3, 32, 48, 5)
    xps, yps = P.pixel_sizes(5, 32, 48)
    d_all = nufft.ms2dirty(uvw, freq, ms, wgt, 32, 48, 5, 1e-9, 2.0, -1)
    d_ex = dft.ms2dirty_dft(uvw, freq, ms, wgt, 32, 48, xps, yps, -1)
    assert l2err(d_ex, d_all) < 1e-8


def _reflib_files():
    # single-call fixtures (inputs stored); the 4096^2 ones are in test_configs_at_size.py
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "reflib_*.npz"))
                  if not os.path.basename(p).startswith("reflib_cfg2_"))


@pytest.mark.parametrize("path", _reflib_files(), ids=os.path.basename)
def test_oracle_nufft_matches_reference_library(path):
    """The numpy restatement against outputs recorded from the reference's own
    libcurafft.so on a B200 (tests/golden/make_ref_golden.py): same algorithm,
    same sizes, so agreement is at FP64 rounding level, far below eps."""
    g = np.load(path)
    assert list(g["status"]) == [0, 0]
    nx, ny = int(g["nx"]), int(g["ny"])
    wgt = g["wgt"] if g["wgt"].size else None
    args = (nx, ny, float(g["fov"]), float(g["eps"]), float(g["sigma"]), int(g["sign"]))
    d = nufft.ms2dirty(g["uvw"], g["freq"], g["ms"], wgt, *args)
    v = nufft.dirty2ms(g["uvw"], g["freq"], g["dirty"], wgt, *args)
    assert l2err(g["ms2dirty"], d) < 1e-11
    assert l2err(g["dirty2ms"], v) < 1e-11


@pytest.mark.parametrize("nchan,sign,use_wgt", [(1, -1, True), (3, 1, False), (4, -1, True)])
def test_torch_dft_matches_c_oracle(nchan, sign, use_wgt):
    """oracle/dft_torch.py (the size-scale checker) against oracle/dft.c, on the CPU."""
    from oracle import dft_torch
    freq, uvw, ms, dirty, wgt = wst_inputs(150, nchan, 48, 40, 10.0, wgt=use_wgt)
    psx, psy = 10 * np.pi / 180 / 48, 10 * np.pi / 180 / 40
    rng = np.random.default_rng(1)
    pix = rng.integers(0, 48 * 40, 300)
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, 48, 40, psx, psy, sign, pix=pix)
    got = dft_torch.ms2dirty_dft(uvw, freq, ms, wgt, 48, 40, psx, psy, sign, pix, chunk=64)
    assert l2err(ref, got) < 1e-12
    d = dirty + 1j * rng.standard_normal(dirty.shape)
    idx = rng.integers(0, 150 * nchan, 200)
    ref = dft.dirty2ms_dft(uvw, freq, d, wgt, psx, psy, sign, idx=idx)
    got = dft_torch.dirty2ms_dft(uvw, freq, d, wgt, psx, psy, sign, idx, chunk=500)
    assert l2err(ref, got) < 1e-12


@pytest.mark.parametrize("path", _golden_files()[1:], ids=os.path.basename)
def test_numpy_explicit_path_matches_reference_truth(path):
    """oracle/explicit_numpy.py (the reference's CPU path as bench.py times it)
    against the reference's own explicit_gridder / explicit_degridder outputs."""
    from oracle import explicit_numpy as X
    g = np.load(path)
    uvw, freq, ms = g["uvw"], g["freq"], g["ms"]
    wgt = g["wgt"] if g["wgt"].size else None
    nx, ny = g["gridder_sign_m1"].shape
    msw = ms * wgt if wgt is not None else ms
    xps, yps = float(g["xpixsize"]), float(g["ypixsize"])
    assert l2err(g["gridder_sign_m1"], X.explicit_gridder(uvw, freq, msw, nx, ny, xps, yps)) < 1e-12
    if "degridder_sign_m1" in g:
        got = X.explicit_degridder(uvw, freq, g["dirty"], xps, yps, -1)
        assert l2err(g["degridder_sign_m1"], got) < 1e-12
