"""Oracle: numpy restatement of CuRIG's improved-w-stacking NUFFT pipeline.

TEST INFRASTRUCTURE ONLY (the checker; never imported by ``curig_b200``).

Follows the reference step by step, in FP64, with the same kernel width, ES
beta, grid sizes, w-plane count, gamma, h and kernel Fourier transforms, so it
agrees with the reference library far more tightly than either agrees with the
exact DFT.  Sizes must stay small (pure numpy; M * kw^3 scatter updates).

ms2dirty (src/astro/ra_exec.cu:141-323):
  effective coords       precomp.cu:48-79     u,v,w *= f/c (w also * sign), * 2 pi
  pixel scaling          cugridder.cu:249-250 u *= pixsize_x, v *= pixsize_y
  vis * wgt              ra_exec.cu:98-104
  c *= e^{i o_c w}       cuft.cu:19-51
  w' = (w-i_c)/gamma     cuft.cu:53-92
  ES spreading           conv.cu:144-228 (x <- v, y <- u, z <- w'; cugridder.cu:188)
  2-D FFT per plane, +1  cuft.cu:127-143
  w-DFT over planes      cuft.cu:520-572
  /(psi1 psi2)           deconv.cu:236-276
  e^{i(n-1-o_c) i_c}/psi3 deconv.cu:371-417
  / n                    ra_exec.cu:22-52
dirty2ms (ra_exec.cu:325-435) runs the adjoint chain; weights multiply (not
divide) at the end (utils.cu:185-192 launches the multiply kernel).

Extension beyond the reference (which handles one channel per call): a list of
channels is folded into one transform with the w range taken over all channels;
for a single channel this is exactly the reference pipeline.
"""
from __future__ import annotations

import numpy as np

from .params import (M_1_2PI, PI, SPEEDOFLIGHT, GridderParams, gridder_params,
                     psi_hat_grid, psi_hat_w)


def _eff_coords(uvw, freqs, P: GridderParams):
    """Spreading coordinates (x, y, z) in grid units plus w_eff per (row, chan)."""
    uvw = np.asarray(uvw, dtype=np.float64)
    freqs = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
    foc = freqs / SPEEDOFLIGHT
    u = (uvw[:, 0:1] * foc[None, :]) * (2 * PI)
    v = (uvw[:, 1:2] * foc[None, :]) * (2 * PI)
    w = (uvw[:, 2:3] * (foc * P.sign)[None, :]) * (2 * PI)
    us = u * P.pixsize_x
    vs = v * P.pixsize_y
    wp = (w - P.i_center) / P.gamma
    gx = (vs * M_1_2PI + 0.5) * P.nf1
    gy = (us * M_1_2PI + 0.5) * P.nf2
    gz = (wp * M_1_2PI + 0.5) * P.nf3
    return gx.ravel(), gy.ravel(), gz.ravel(), w.ravel(), wp.ravel()


def _taps(g, nf, opts, window):
    """Start cell, wrapped indices [M, kw] and kernel values [M, kw] along one axis."""
    kw = opts.kw
    start = np.ceil(g - kw / 2.0)
    off = (start - g)[:, None] + np.arange(kw)[None, :]
    if window is None:
        val = np.zeros_like(off)
        m = np.abs(off) < kw / 2.0
        val[m] = np.exp(opts.beta * np.sqrt(1.0 - opts.c * off[m] * off[m]))
    else:
        val = window(off)
    idx = (start.astype(np.int64)[:, None] + np.arange(kw)[None, :]) % nf
    return idx, val


def _pixel_tables(P: GridderParams):
    """Per-pixel FFTW indices, n, n-1 (naive form, as the reference), k' and the
    correction factors, for the [nx][ny] dirty layout."""
    nx, ny = P.nxdirty, P.nydirty
    ix = np.arange(nx)[:, None]
    iy = np.arange(ny)[None, :]
    w2 = np.where(ix >= nx // 2, ix - nx // 2, P.nf2 + ix - nx // 2)
    w1 = np.where(iy >= ny // 2, iy - ny // 2, P.nf1 + iy - ny // 2)
    ax = np.abs(ix - nx // 2) * P.pixsize_x
    ay = np.abs(iy - ny // 2) * P.pixsize_y
    k = np.sqrt(1.0 - ax ** 2 - ay ** 2) - 1                      # precomp.cu:220
    kp = (k - P.o_center) * P.gamma * P.h                         # cuft.cu:73
    lx = (ix - nx // 2) * P.pixsize_x
    my = (iy - ny // 2) * P.pixsize_y
    n = np.sqrt(1.0 - lx ** 2 - my ** 2)                          # ra_exec.cu:31
    nm1 = np.sqrt(1.0 - lx ** 2 - my ** 2) - 1                    # deconv.cu:390
    return w1, w2, kp, n, nm1


def ms2dirty(uvw, freqs, vis, wgt, nxdirty, nydirty, fov_deg=None, eps=1e-6, sigma=2.0,
             sign=1, pixsize_x=None, pixsize_y=None, window=None, params=None):
    """Complex dirty image [nx][ny] of vis [nrow][nchan] (wgt same shape or None)."""
    P = params or gridder_params(nxdirty, nydirty, fov_deg, uvw, freqs, eps, sigma, sign,
                                 pixsize_x, pixsize_y)
    opts = P.opts
    gx, gy, gz, w, _ = _eff_coords(uvw, freqs, P)
    c = np.asarray(vis, dtype=np.complex128).ravel().copy()
    if wgt is not None:
        c = c * np.asarray(wgt, dtype=np.float64).ravel()
    c = c * np.exp(1j * (P.o_center * w))
    ixs, kx = _taps(gx, P.nf1, opts, window)
    iys, ky = _taps(gy, P.nf2, opts, window)
    izs, kz = _taps(gz, P.nf3, opts, window)
    grid = np.zeros((P.nf3, P.nf2, P.nf1), dtype=np.complex128)
    kw = opts.kw
    for a in range(kw):
        for b in range(kw):
            cz = c * kz[:, a] * ky[:, b]
            for d in range(kw):
                np.add.at(grid, (izs[:, a], iys[:, b], ixs[:, d]), cz * kx[:, d])
    grid = np.fft.ifft2(grid, axes=(1, 2)) * (P.nf1 * P.nf2)       # cuFFT sign +1
    w1, w2, kp, n, nm1 = _pixel_tables(P)
    planes = grid[:, w2, w1]                                       # [nf3][nx][ny]
    p = np.arange(P.nf3) - P.nf3 // 2
    out = np.einsum('pxy,pxy->xy', planes, np.exp(1j * kp[None] * p[:, None, None]))
    psi1 = psi_hat_grid(P.nf1, opts, window)
    psi2 = psi_hat_grid(P.nf2, opts, window)
    ix = np.arange(P.nxdirty)[:, None]
    iy = np.arange(P.nydirty)[None, :]
    out = out / (psi1[np.abs(iy - P.nydirty // 2)] * psi2[np.abs(ix - P.nxdirty // 2)])
    psi3 = psi_hat_w(kp, opts, window)
    out = out * np.exp(1j * ((nm1 - P.o_center) * P.i_center)) / psi3
    return out / n


def dirty2ms(uvw, freqs, dirty, wgt, nxdirty, nydirty, fov_deg=None, eps=1e-6, sigma=2.0,
             sign=1, pixsize_x=None, pixsize_y=None, window=None, params=None):
    """Complex visibilities [nrow][nchan] of the complex dirty image [nx][ny]."""
    P = params or gridder_params(nxdirty, nydirty, fov_deg, uvw, freqs, eps, sigma, sign,
                                 pixsize_x, pixsize_y)
    opts = P.opts
    nrow = np.asarray(uvw).shape[0]
    nchan = np.atleast_1d(freqs).shape[0]
    fk = np.asarray(dirty, dtype=np.complex128).reshape(nxdirty, nydirty)
    w1, w2, kp, n, nm1 = _pixel_tables(P)
    fk = fk / n
    psi3 = psi_hat_w(kp, opts, window)
    fk = fk * np.exp(-1j * ((nm1 - P.o_center) * P.i_center)) / psi3
    psi1 = psi_hat_grid(P.nf1, opts, window)
    psi2 = psi_hat_grid(P.nf2, opts, window)
    ix = np.arange(nxdirty)[:, None]
    iy = np.arange(nydirty)[None, :]
    fk = fk / (psi1[np.abs(iy - nydirty // 2)] * psi2[np.abs(ix - nxdirty // 2)])
    grid = np.zeros((P.nf3, P.nf2, P.nf1), dtype=np.complex128)
    p = np.arange(P.nf3) - P.nf3 // 2
    grid[:, w2, w1] = fk[None] * np.exp(-1j * kp[None] * p[:, None, None])
    grid = np.fft.fft2(grid, axes=(1, 2))                          # cuFFT sign -1
    gx, gy, gz, w, wp = _eff_coords(uvw, freqs, P)
    ixs, kx = _taps(gx, P.nf1, opts, window)
    iys, ky = _taps(gy, P.nf2, opts, window)
    izs, kz = _taps(gz, P.nf3, opts, window)
    c = np.zeros(gx.shape[0], dtype=np.complex128)
    kw = opts.kw
    for a in range(kw):
        for b in range(kw):
            for d in range(kw):
                c += grid[izs[:, a], iys[:, b], ixs[:, d]] * (kz[:, a] * ky[:, b] * kx[:, d])
    if wgt is not None:
        c = c * np.asarray(wgt, dtype=np.float64).ravel()
    c = c * np.exp(-1j * ((wp * P.gamma + P.i_center) * P.o_center))  # ra_exec.cu:56-64
    return c.reshape(nrow, nchan)
