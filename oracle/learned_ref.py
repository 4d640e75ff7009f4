"""Oracle for the learned window: CPU (torch, FP64, autograd) restatement of
the training objective and of the window, for checking the GPU forward and
backward kernels of curig_b200/csrc/learned.cu.

TEST INFRASTRUCTURE ONLY (the checker; never imported by curig_b200).

Objective (per axis): S(f, xi) = sum_d phi(t_d) e^{2 pi i xi t_d} with
t_d = ceil(f - W/2) + d - f over f = (i + 1/2)/64, xi in linspace(-1/(2 sigma),
1/(2 sigma), 64); psi(xi) = int phi(t) cos(2 pi xi t) dt by a 96-point
Gauss-Legendre rule on [-W/2, W/2]; L = sqrt(mean |S/psi - 1|^2).  The
quadrature correction restates src/fourier/deconv.cu:13-197 of the reference;
the rest has no reference counterpart.
"""
from __future__ import annotations

import math

import numpy as np
import torch

H = 32
NF, NXI, NQ = 64, 64, 96


def es_beta(W: int, sigma: float = 2.0) -> float:
    if sigma == 2.0:
        return {2: 2.20, 3: 2.26, 4: 2.38}.get(W, 2.30) * W
    return 0.97 * math.pi * (1 - 1 / (2 * sigma)) * W


def unpack(p):
    o = 0
    out = []
    for shape in ((H,), (H,), (H, H), (H,), (H, H), (H,), (H,), (1,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def window(p, t, W, beta):
    W1, b1, W2, b2, W3, b3, Wo, bo = unpack(p)
    x = 2 * t / W
    z = torch.clamp(x * x, max=1.0)
    h = torch.tanh(z[:, None] * W1[None, :] + b1[None, :])
    h = torch.tanh(h @ W2.T + b2)
    h = torch.tanh(h @ W3.T + b3)
    g = h @ Wo + bo[0]
    es = -beta * z / (torch.sqrt(torch.clamp(1 - z, min=0.0)) + 1)
    return torch.where(t.abs() < W / 2, torch.exp(es + g), torch.zeros_like(t))


def objective(params: np.ndarray, W: int, sigma: float = 2.0):
    """(L, d log L / d params) in FP64 on the CPU."""
    p = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
    beta = es_beta(W, sigma)
    xg, wg = np.polynomial.legendre.leggauss(NQ)
    tq = torch.tensor(xg * W / 2)
    wq = torch.tensor(wg * W / 2)
    xi = torch.linspace(-0.5 / sigma, 0.5 / sigma, NXI, dtype=torch.float64)
    f = (torch.arange(NF, dtype=torch.float64) + 0.5) / NF
    T = torch.ceil(f[:, None] - W / 2) + torch.arange(W, dtype=torch.float64)[None, :] - f[:, None]
    psi = (window(p, tq, W, beta)[None, :] * torch.cos(2 * math.pi * xi[:, None] * tq[None, :])) @ wq
    P = window(p, T.reshape(-1), W, beta).reshape(T.shape)
    ang = 2 * math.pi * xi[:, None, None] * T[None]
    Sr = (torch.cos(ang) * P[None]).sum(-1)
    Si = (torch.sin(ang) * P[None]).sum(-1)
    er = Sr / psi[:, None] - 1
    ei = Si / psi[:, None]
    L = torch.sqrt(torch.mean(er ** 2 + ei ** 2))
    torch.log(L).backward()
    return float(L), p.grad.numpy()
