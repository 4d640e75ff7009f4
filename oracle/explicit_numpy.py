"""The reference's CPU path for this transform, in numpy: its explicit FP64
gridder and degridder.

TEST AND BASELINE INFRASTRUCTURE ONLY.  A restatement of
python/curagridder/test_wst.py:15-32 (explicit_gridder) and
python/curagridder/explicit_test.py:32-54 (explicit_degridder) with the same
numpy evaluation pattern -- one visibility at a time, each a handful of
whole-image array operations (phase, complex exponential, accumulate) in a
single Python process -- so that timing it measures what running the
reference's own CPU code costs.  The reference's Python modules cannot be
imported where the benchmark runs (they load the reference's GPU library at
import), so the functions are restated here.

Conventions: pixel (ix, iy) at l = (ix - nx/2) psx, m = (iy - ny/2) psy
(half-integer centres for odd sizes, as np.arange(n) - n/2 gives);
n - 1 = -e / (sqrt(1 - e) + 1), e = l^2 + m^2.
"""
from __future__ import annotations

import numpy as np

SPEEDOFLIGHT = 299792458.0


def _lmn(nx, ny, psx, psy):
    l, m = np.meshgrid((np.arange(nx) - nx / 2) * psx, (np.arange(ny) - ny / 2) * psy, indexing="ij")
    e = l * l + m * m
    nm1 = -e / (np.sqrt(1.0 - e) + 1.0)
    return l, m, nm1, nm1 + 1.0


def explicit_gridder(uvw, freq, ms, nx, ny, psx, psy):
    """Real dirty image [nx][ny] = Re sum ms e^{2 pi i f/c (l u + m v - w (n-1))} / n."""
    l, m, nm1, n = _lmn(nx, ny, psx, psy)
    out = np.zeros((nx, ny))
    for r in range(ms.shape[0]):
        u, v, w = uvw[r]
        for c in range(ms.shape[1]):
            ph = (freq[c] / SPEEDOFLIGHT) * (l * u + m * v - w * nm1)
            out += (ms[r, c] * np.exp(2j * np.pi * ph)).real
    return out / n


def explicit_degridder(uvw, freq, dirty, psx, psy, sign):
    """Visibilities [nrow * nchan] = sum dirty / n e^{-2 pi i f/c (l u + m v + sign w (n-1))}."""
    nx, ny = dirty.shape
    l, m, nm1, n = _lmn(nx, ny, psx, psy)
    img = dirty.astype(np.complex128) / n
    nchan = len(freq)
    out = np.zeros(uvw.shape[0] * nchan, dtype=np.complex128)
    for r in range(uvw.shape[0]):
        u, v, w = uvw[r]
        for c in range(nchan):
            ph = -(freq[c] / SPEEDOFLIGHT) * (l * u + m * v + sign * w * nm1)
            out[r * nchan + c] = np.sum(img * np.exp(2j * np.pi * ph))
    return out
