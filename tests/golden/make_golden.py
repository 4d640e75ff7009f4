"""Generate golden vectors from the reference's own Python truth functions.

Run here (the reference tree is only needed at generation time):
    python tests/golden/make_golden.py <reference source tree>

The reference's test modules import its ctypes library at module level and run
tests on import, so the truth functions are taken out of the source with
``ast`` and executed alone:
  * python/curagridder/test_wst.py  explicit_gridder        (sign -1, real)
  * python/curagridder/test_ws.py   explicit_gridder        (sign +1, real)
  * python/curagridder/explicit_test.py explicit_degridder  (sign -1, complex)
Inputs follow test_wst.py:55-62 (np.random.seed(42), f0 = 1 GHz,
u,v,w uniform in +-0.5 c/f0) plus one larger case with the 256x256 /
2000-visibility shape (seeded uniform-disk u,v, w in +-200 m).
"""
from __future__ import annotations

import ast
import os
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))


def load_functions(path, names):
    src = open(path).read()
    tree = ast.parse(src)
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    mod = ast.Module(body=body, type_ignores=[])
    ns = {"np": np}
    exec(compile(mod, path, "exec"), ns)
    return {n: ns[n] for n in names}


def main(ref):
    py = os.path.join(ref, "python", "curagridder")
    wst = load_functions(os.path.join(py, "test_wst.py"), ["explicit_gridder"])
    ws = load_functions(os.path.join(py, "test_ws.py"), ["explicit_gridder"])
    ex = load_functions(os.path.join(py, "explicit_test.py"), ["explicit_degridder"])
    c = 299792458.0
    cases = [  # (nrow, nxdirty, nydirty, fov_deg, use_wgt) from the test_wst.py:36-42 grid
        (27, 30, 128, 10, True),
        (100, 16, 64, 20, False),
        (100, 128, 250, 1, True),
    ]
    for (nrow, nx, ny, fov, use_wgt) in cases:
        np.random.seed(42)
        nchan = 1
        f0 = 1e9
        freq = f0 + np.arange(nchan) * (f0 / nchan)
        uvw = (np.random.rand(nrow, 3) - 0.5) / (f0 / c)
        ms = np.random.rand(nrow, nchan) - 0.5 + 1j * (np.random.rand(nrow, nchan) - 0.5)
        dirty = np.random.rand(nx, ny) - 0.5
        wgt = np.random.rand(nrow, nchan) if use_wgt else None
        xps = fov * np.pi / 180 / nx
        yps = fov * np.pi / 180 / ny
        msw = ms * wgt if use_wgt else ms
        g_m = wst["explicit_gridder"](uvw, freq, msw, nx, ny, xps, yps)
        g_p = ws["explicit_gridder"](uvw, freq, msw, nx, ny, xps, yps)
        d_m = ex["explicit_degridder"](uvw, freq, dirty, xps, yps, nrow, nchan, -1)
        name = f"refdft_n{nrow}_{nx}x{ny}_fov{fov}.npz"
        np.savez_compressed(os.path.join(OUT, name), uvw=uvw, freq=freq, ms=ms, dirty=dirty,
                            wgt=np.zeros(0) if wgt is None else wgt, fov=fov,
                            xpixsize=xps, ypixsize=yps, gridder_sign_m1=g_m,
                            gridder_sign_p1=g_p, degridder_sign_m1=d_m)
        print("wrote", name)
    # 256x256, 2000 visibilities, fov 2 deg, 1 GHz: uniform disk with
    # max|u| * fov / lambda = 120 pixels, w uniform in +-200 m, seed 0.
    rng = np.random.default_rng(0)
    nrow, nx, ny, fov, f0 = 2000, 256, 256, 2.0, 1.0e9
    lam = c / f0
    R = 120.0 * lam / (fov * np.pi / 180)
    r = R * np.sqrt(rng.random(nrow))
    th = 2 * np.pi * rng.random(nrow)
    w = rng.uniform(-200.0, 200.0, nrow)
    uvw = np.stack([r * np.cos(th), r * np.sin(th), w], axis=1)
    ms = (rng.standard_normal(nrow) + 1j * rng.standard_normal(nrow))[:, None]
    wgt = (1.0 - rng.random(nrow))[:, None] * 0.5 + 0.5       # uniform (0.5, 1]
    xps = fov * np.pi / 180 / nx
    yps = fov * np.pi / 180 / ny
    g_m = wst["explicit_gridder"](uvw, np.array([f0]), ms * wgt, nx, ny, xps, yps)
    np.savez_compressed(os.path.join(OUT, "refdft_disk2000_256x256.npz"), uvw=uvw,
                        freq=np.array([f0]), ms=ms, wgt=wgt, fov=fov, xpixsize=xps,
                        ypixsize=yps, gridder_sign_m1=g_m)
    print("wrote refdft_disk2000_256x256.npz")


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("CURIG_REFERENCE"):
        sys.exit("usage: make_golden.py <reference source tree> (or set CURIG_REFERENCE)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["CURIG_REFERENCE"])
