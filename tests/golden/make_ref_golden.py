"""Record golden outputs of the reference library itself.

Runs on a machine with a B200: loads oracle/_ref/libcurafft_ref.so (the
reference's libcurafft.so built for sm_100a from its own sources by
oracle/Makefile.ref) through the same ctypes signatures as the reference's
python/curagridder/curagridder.py:50-70, calls ms2dirty_2 / dirty2ms_2 (and the
_1 forms) on seeded inputs, and writes reflib_*.npz (inputs + outputs) to the
directory given on the command line.  The files are then committed under
tests/golden/ and pin both the oracle's NUFFT restatement and the product.

    python tests/golden/make_ref_golden.py <output directory>
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
C = 299792458.0


def load():
    lib = ctypes.cdll.LoadLibrary(os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so"))
    f64 = np.ctypeslib.ndpointer(np.double, flags="C")
    c128 = np.ctypeslib.ndpointer(np.complex128, flags="C")
    ci, cd = ctypes.c_int, ctypes.c_double
    for name, wgt in (("ms2dirty_1", False), ("ms2dirty_2", True), ("dirty2ms_1", False),
                      ("dirty2ms_2", True)):
        f = getattr(lib, name)
        f.argtypes = [ci, ci, ci, cd, cd, f64, c128] + ([f64] if wgt else []) + [c128, cd, cd, ci]
        f.restype = ci
    return lib


def wst_case(nrow, nx, ny, seed=42):
    rng = np.random.RandomState(seed)
    f0 = 1e9
    uvw = (rng.rand(nrow, 3) - 0.5) / (f0 / C)
    ms = rng.rand(nrow, 1) - 0.5 + 1j * (rng.rand(nrow, 1) - 0.5)
    dirty = rng.rand(nx, ny) - 0.5 + 0j
    wgt = rng.rand(nrow, 1)
    return np.array([f0]), uvw, ms, dirty, wgt


def disk_case(nrow, nx, fov, seed=0):
    rng = np.random.default_rng(seed)
    f0 = 1e9
    R = 120.0 * (C / f0) / (fov * np.pi / 180)
    r = R * np.sqrt(rng.random(nrow))
    th = 2 * np.pi * rng.random(nrow)
    w = rng.uniform(-200.0, 200.0, nrow)
    uvw = np.stack([r * np.cos(th), r * np.sin(th), w], axis=1)
    ms = (rng.standard_normal(nrow) + 1j * rng.standard_normal(nrow))[:, None]
    wgt = ((1.0 - rng.random(nrow)) * 0.5 + 0.5)[:, None]
    dirty = rng.standard_normal((nx, nx)) + 0j
    return np.array([f0]), uvw, ms, dirty, wgt


CASES = [  # name, generator, nx, ny, fov, eps, sigma, sign, use_wgt
    ("wst_n100_30x128_fov10_e5e-7", lambda: wst_case(100, 30, 128), 30, 128, 10.0, 5e-7, 2.0, -1, True),
    ("wst_n27_16x64_fov20_e5e-3", lambda: wst_case(27, 16, 64), 16, 64, 20.0, 5e-3, 2.0, -1, False),
    ("wst_n100_128x250_fov1_e5e-12", lambda: wst_case(100, 128, 250), 128, 250, 1.0, 5e-12, 2.0, -1, True),
    ("ws_n200_64x64_fov2_e1e-6_sp1", lambda: wst_case(200, 64, 64), 64, 64, 2.0, 1e-6, 2.0, 1, True),
    ("ws_n200_64x48_fov5_e1e-6_s125", lambda: wst_case(200, 64, 48), 64, 48, 5.0, 1e-6, 1.25, 1, False),
    ("disk2000_256x256_fov2_e1e-6", lambda: disk_case(2000, 256, 2.0), 256, 256, 2.0, 1e-6, 2.0, -1, True),
]


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    lib = load()
    for name, gen, nx, ny, fov, eps, sigma, sign, use_wgt in CASES:
        freq, uvw, ms, dirty, wgt = gen()
        uvw = np.ascontiguousarray(uvw)
        out_d = np.zeros((nx, ny), dtype=np.complex128)
        out_v = np.zeros((uvw.shape[0], 1), dtype=np.complex128)
        if use_wgt:
            s1 = lib.ms2dirty_2(uvw.shape[0], nx, ny, fov, freq[0], uvw, ms, wgt, out_d, eps, sigma, sign)
            s2 = lib.dirty2ms_2(uvw.shape[0], nx, ny, fov, freq[0], uvw, out_v, wgt, dirty, eps, sigma, sign)
        else:
            s1 = lib.ms2dirty_1(uvw.shape[0], nx, ny, fov, freq[0], uvw, ms, out_d, eps, sigma, sign)
            s2 = lib.dirty2ms_1(uvw.shape[0], nx, ny, fov, freq[0], uvw, out_v, dirty, eps, sigma, sign)
        np.savez_compressed(os.path.join(outdir, f"reflib_{name}.npz"), uvw=uvw, freq=freq, ms=ms,
                            dirty=dirty, wgt=wgt if use_wgt else np.zeros(0), nx=nx, ny=ny, fov=fov,
                            eps=eps, sigma=sigma, sign=sign, status=np.array([s1, s2]),
                            ms2dirty=out_d, dirty2ms=out_v)
        print(name, "status", s1, s2, "|dirty|", float(np.abs(out_d).max()), flush=True)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_ref_golden.py <output directory>")
    main(sys.argv[1])
