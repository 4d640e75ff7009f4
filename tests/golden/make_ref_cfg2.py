"""Record the reference library's outputs at the 4096^2 configuration.

Runs on a machine with a B200: the reference's libcurafft.so (built for
sm_100a from its own sources by oracle/Makefile.ref into oracle/_ref/) is
called through its one-shot ABI (ms2dirty_2 / dirty2ms_2, FP64, host buffers,
one frequency per call, src/astro/cugridder.cu:587-612), once per channel as
its Python package does (python/curagridder/curagridder.py:92 passes freq[0]).
ms2dirty is summed over channels; dirty2ms is evaluated per channel.  Only
values at seeded sample indices are stored (2,000 pixels of the summed dirty
image, 2,000 visibilities), with the full-image L2 norm and an input checksum;
the inputs themselves are regenerated by tests/conftest.gaussian_uv_inputs.

    python tests/golden/make_ref_cfg2.py <output directory> [nrow]

Workload: nrow rows (default 2e6) x 16 channels (0.9-1.1 GHz), 4096^2, fov 3
deg, sigma 2, sign -1, epsilon in {1e-4, 1e-5, 1e-6}; the dirty2ms input is
tests/conftest.gaussian_image(4096, seed=1).
"""
from __future__ import annotations

import ctypes
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import gaussian_image, gaussian_uv_inputs, input_checksum  # noqa: E402

NPIX, FOV, NCHAN = 4096, 3.0, 16
EPSILONS = (1e-4, 1e-5, 1e-6)


def samples(nrow, nchan=NCHAN, npix=NPIX):
    """Seeded sample indices: 2,000 distinct pixels and 2,000 distinct visibilities."""
    rng = np.random.default_rng(5)
    pix = np.sort(rng.choice(npix * npix, 2000, replace=False)).astype(np.int64)
    vidx = np.sort(rng.choice(nrow * nchan, 2000, replace=False)).astype(np.int64)
    return pix, vidx


def bind(path):
    lib = ctypes.CDLL(path)
    P, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    for name in ("ms2dirty_2", "dirty2ms_2"):
        f = getattr(lib, name)
        f.argtypes = [ci, ci, ci, cd, cd, P, P, P, P, cd, cd, ci]
        f.restype = ci
    return lib


def main(outdir, nrow):
    os.makedirs(outdir, exist_ok=True)
    lib = bind(os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so"))
    freq, uvw, vis, wgt = gaussian_uv_inputs(nrow, NCHAN, NPIX, FOV, seed=0)
    img = gaussian_image(NPIX, seed=1)
    pix, vidx = samples(nrow)
    vrow, vch = vidx // NCHAN, vidx % NCHAN
    res = {"nrow": nrow, "nchan": NCHAN, "npix": NPIX, "fov": FOV, "pix": pix, "vidx": vidx,
           "epsilons": np.array(EPSILONS), "checksum": input_checksum(uvw, vis, wgt),
           "image_checksum": input_checksum(img)}
    uvw = np.ascontiguousarray(uvw)
    for k, eps in enumerate(EPSILONS):
        t0 = time.time()
        acc = np.zeros((NPIX, NPIX), dtype=np.complex128)
        out = np.zeros((NPIX, NPIX), dtype=np.complex128)
        vals = np.zeros(vidx.size, dtype=np.complex128)
        status = []
        for c in range(NCHAN):
            vc = np.ascontiguousarray(vis[:, c])
            wc = np.ascontiguousarray(wgt[:, c])
            st = lib.ms2dirty_2(nrow, NPIX, NPIX, FOV, float(freq[c]), uvw.ctypes.data, vc.ctypes.data,
                                wc.ctypes.data, out.ctypes.data, eps, 2.0, -1)
            status.append(st)
            acc += out
            vo = np.zeros(nrow, dtype=np.complex128)
            st = lib.dirty2ms_2(nrow, NPIX, NPIX, FOV, float(freq[c]), uvw.ctypes.data, vo.ctypes.data,
                                wc.ctypes.data, img.ctypes.data, eps, 2.0, -1)
            status.append(st)
            sel = vch == c
            vals[sel] = vo[vrow[sel]]
        res[f"status_{k}"] = np.array(status)
        res[f"ms2dirty_{k}"] = acc.reshape(-1)[pix]
        res[f"ms2dirty_norm_{k}"] = float(np.linalg.norm(acc))
        res[f"dirty2ms_{k}"] = vals
        print(f"eps {eps:g}: statuses {sorted(set(status))}, |dirty| {res[f'ms2dirty_norm_{k}']:.6e}, "
              f"{time.time() - t0:.1f} s", flush=True)
    path = os.path.join(outdir, f"reflib_cfg2_{nrow}x{NCHAN}_{NPIX}.npz")
    np.savez_compressed(path, **res)
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_ref_cfg2.py <output directory> [nrow]")
    main(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 2_000_000)
