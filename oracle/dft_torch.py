"""FP64 explicit DFT in torch, for checks at the full configuration sizes.

TEST INFRASTRUCTURE ONLY -- a checker, never the product.  The same formulas
as oracle/dft.c (the reference's truth functions,
python/curagridder/test_wst.py:15-32 and explicit_test.py:32-54), in the same
operation order, evaluated with torch on any device: on a GPU it checks
2,000 sampled pixels (or visibilities) of a transform of 1e7-1.6e8
visibilities in seconds, which the C/OpenMP oracle cannot.  Pinned to
oracle/dft.c by tests/test_oracle.py (CPU, 1e-12).

  ms2dirty:  dirty[p] = sum_j wgt_j vis_j exp(+2 pi i f/c (l u + m v + sign w (n-1))) / n
  dirty2ms:  vis_j = wgt_j sum_p dirty[p] / n exp(-2 pi i f/c (l u + m v + sign w (n-1)))
Pixel (ix, iy) sits at l = (ix - nx/2) psx, m = (iy - ny/2) psy (integer halves),
n - 1 = -e / (sqrt(1 - e) + 1), e = l^2 + m^2.
"""
from __future__ import annotations

import math

import numpy as np

SPEEDOFLIGHT = 299792458.0


def _pixels(torch, pix, nx, ny, psx, psy, dev):
    p = torch.as_tensor(np.asarray(pix, dtype=np.int64), device=dev)
    x = (p // ny - nx // 2).to(torch.float64) * psx
    y = (p % ny - ny // 2).to(torch.float64) * psy
    e = x * x + y * y
    nm1 = -e / (torch.sqrt(1.0 - e) + 1.0)
    return x, y, nm1, nm1 + 1.0


def ms2dirty_dft(uvw, freq, vis, wgt, nx, ny, psx, psy, sign, pix, chunk=1 << 16):
    """Complex dirty values at the flat pixels ``pix`` (numpy complex128).
    uvw [nrow][3] float64, vis [nrow][nchan] complex, wgt same shape or None:
    torch tensors on one device (or numpy arrays, moved to the CPU device)."""
    import torch
    uvw = torch.as_tensor(uvw)
    dev = uvw.device
    uvw = uvw.to(torch.float64)
    vis = torch.as_tensor(vis, device=dev).to(torch.complex128)
    nrow = uvw.shape[0]
    nchan = len(freq)
    vis = vis.reshape(nrow, nchan)
    if wgt is not None:
        wgt = torch.as_tensor(wgt, device=dev).to(torch.float64).reshape(nrow, nchan)
    l, m, nm1, n = _pixels(torch, pix, nx, ny, psx, psy, dev)
    acc = torch.zeros(l.shape[0], dtype=torch.complex128, device=dev)
    for r0 in range(0, nrow, chunk):
        r1 = min(nrow, r0 + chunk)
        u, v, w = uvw[r0:r1, 0], uvw[r0:r1, 1], uvw[r0:r1, 2]
        base = torch.outer(l, u) + torch.outer(m, v) + float(sign) * torch.outer(nm1, w)
        z = vis[r0:r1]
        if wgt is not None:
            z = z * wgt[r0:r1]
        for c in range(nchan):
            ph = 2.0 * math.pi * ((float(freq[c]) / SPEEDOFLIGHT) * base)
            e = torch.complex(torch.cos(ph), torch.sin(ph))
            acc += e @ z[:, c]
            del ph, e
        del base
    return (acc / n).cpu().numpy()


def dirty2ms_dft(uvw, freq, dirty, wgt, psx, psy, sign, idx, chunk=1 << 15):
    """Complex visibilities at the flat (row * nchan + chan) indices ``idx``."""
    import torch
    uvw = torch.as_tensor(uvw)
    dev = uvw.device
    uvw = uvw.to(torch.float64)
    dirty = torch.as_tensor(dirty, device=dev).to(torch.complex128)
    nx, ny = dirty.shape
    nrow = uvw.shape[0]
    nchan = len(freq)
    j = torch.as_tensor(np.asarray(idx, dtype=np.int64), device=dev)
    r, c = j // nchan, j % nchan
    foc = torch.as_tensor(np.asarray(freq, dtype=np.float64), device=dev)[c] / SPEEDOFLIGHT
    u, v, w = uvw[r, 0], uvw[r, 1], uvw[r, 2]
    flat = dirty.reshape(-1)
    acc = torch.zeros(j.shape[0], dtype=torch.complex128, device=dev)
    npix = nx * ny
    for p0 in range(0, npix, chunk):
        p1 = min(npix, p0 + chunk)
        l, m, nm1, n = _pixels(torch, np.arange(p0, p1), nx, ny, psx, psy, dev)
        base = torch.outer(u, l) + torch.outer(v, m) + float(sign) * torch.outer(w, nm1)
        ph = -2.0 * math.pi * (foc[:, None] * base)
        e = torch.complex(torch.cos(ph), torch.sin(ph))
        acc += e @ (flat[p0:p1] / n)
        del base, ph, e
    if wgt is not None:
        wt = torch.as_tensor(wgt, device=dev).to(torch.float64).reshape(-1)[j]
        acc = acc * wt
    return acc.cpu().numpy()
