import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
SPEEDOFLIGHT = 299792458.0


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def l2err(ref, got):
    ref = np.asarray(ref)
    got = np.asarray(got)
    return float(np.sqrt(np.sum(np.abs(ref - got) ** 2) / np.sum(np.abs(ref) ** 2)))


def wst_inputs(nrow, nchan, nx, ny, fov, seed=42, wgt=True):
    """Inputs drawn as in the reference's python/curagridder/test_wst.py:55-62."""
    rng = np.random.RandomState(seed)
    f0 = 1e9
    freq = f0 + np.arange(nchan) * (f0 / nchan)
    uvw = (rng.rand(nrow, 3) - 0.5) / (f0 / SPEEDOFLIGHT)
    ms = rng.rand(nrow, nchan) - 0.5 + 1j * (rng.rand(nrow, nchan) - 0.5)
    dirty = rng.rand(nx, ny) - 0.5
    w = rng.rand(nrow, nchan) if wgt else None
    return freq, uvw, ms, dirty, w


def disk_inputs(nrow, nchan, nx, fov_deg, f0=1.0e9, fmax=None, max_pix=120.0, wmax=200.0, seed=0,
                gaussian=False):
    """Uniform-disk (or truncated-Gaussian) u,v with max|u| fov/lambda = max_pix
    pixels at the highest frequency, w uniform in +-wmax metres, complex normal
    visibilities, weights uniform in (0.5, 1]."""
    rng = np.random.default_rng(seed)
    c = SPEEDOFLIGHT
    fmax = fmax or f0
    freq = np.linspace(f0, fmax, nchan) if nchan > 1 else np.array([f0])
    R = max_pix * (c / freq.max()) / (fov_deg * np.pi / 180)
    if gaussian:
        r = np.abs(rng.standard_normal(nrow)) * 0.3 * R
        bad = r > R
        while bad.any():
            r[bad] = np.abs(rng.standard_normal(bad.sum())) * 0.3 * R
            bad = r > R
    else:
        r = R * np.sqrt(rng.random(nrow))
    th = 2 * np.pi * rng.random(nrow)
    w = rng.uniform(-wmax, wmax, nrow)
    uvw = np.stack([r * np.cos(th), r * np.sin(th), w], axis=1)
    ms = rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))
    wgt = (1.0 - rng.random((nrow, nchan))) * 0.5 + 0.5
    return freq, uvw, ms, wgt


def gaussian_uv_inputs(nrow, nchan=16, npix=4096, fov_deg=3.0, seed=0, fmin=0.9e9, fmax=1.1e9, wmax=1000.0):
    """The 4096^2 configuration's visibilities, drawn with numpy (the same
    values on every machine with this numpy): channels linear in
    [fmin, fmax]; (u, v) from an isotropic Gaussian of sigma = 0.3 R, draws
    beyond R drawn again, R * fov / lambda_min = 0.47 npix pixels; w uniform
    in +-wmax metres; complex-normal visibilities [nrow][nchan]; weights
    uniform in (0.5, 1]."""
    rng = np.random.default_rng(seed)
    freq = np.linspace(fmin, fmax, nchan) if nchan > 1 else np.array([1.0e9])
    R = 0.47 * npix * (SPEEDOFLIGHT / freq.max()) / (fov_deg * np.pi / 180)
    uv = rng.standard_normal((nrow, 2)) * (0.3 * R)
    for _ in range(64):
        bad = np.flatnonzero((uv * uv).sum(1) > R * R)
        if bad.size == 0:
            break
        uv[bad] = rng.standard_normal((bad.size, 2)) * (0.3 * R)
    w = rng.uniform(-wmax, wmax, (nrow, 1))
    uvw = np.ascontiguousarray(np.concatenate([uv, w], 1))
    vis = np.empty((nrow, nchan), dtype=np.complex128)
    vis.real = rng.standard_normal((nrow, nchan))
    vis.imag = rng.standard_normal((nrow, nchan))
    wgt = 1.0 - 0.5 * rng.random((nrow, nchan))
    return freq, uvw, vis, wgt


def gaussian_image(npix, seed=1):
    """Complex-normal dirty image [npix][npix] (numpy, seeded)."""
    rng = np.random.default_rng(seed)
    img = np.empty((npix, npix), dtype=np.complex128)
    img.real = rng.standard_normal((npix, npix))
    img.imag = rng.standard_normal((npix, npix))
    return img


def input_checksum(*arrays):
    """Order-sensitive checksum of the inputs (detects a change of generator)."""
    s = 0.0
    for a in arrays:
        f = np.ascontiguousarray(a).view(np.float64).reshape(-1)
        k = np.arange(1, f.size + 1, dtype=np.float64) % 997.0
        s += float(np.dot(f, k))
    return s
