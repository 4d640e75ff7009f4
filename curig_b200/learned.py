"""Learned gridding window (host side of curig_train_window & co.).

The window is phi(t) = exp(beta (sqrt(1 - x^2) - 1) + g(x^2)), x = 2t/W,
|t| < W/2, with g a 1-32-32-32-1 tanh MLP whose FP32 parameters are trained on
the GPU by the library's own kernels (forward, backward and Adam in
curig_b200/csrc/learned.cu).  The objective is the RMS error, per axis, of
gridding one visibility with the window, transforming, and correcting by the
window's Fourier transform, against the exact DFT over the image band.  The
ES window is the starting point (g = 0) and stays the fallback: a plan with
window="learned" uses the narrowest registered width whose error reaches the
requested epsilon, and windows are registered only through this module.

Trained parameters for sigma = 2 ship in curig_b200/windows/learned_sigma2.json
(written by oracle/train_windows.py on a B200).
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import _lib

NPARAMS = int(_lib.lib.curig_window_nparams())
DEGREE = 11                      # Horner degree of the tabulated window
WINDOWS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "windows")
DEFAULT_FILE = os.path.join(WINDOWS_DIR, "learned_sigma2.json")
# 3-D error of one transform relative to the per-axis objective (three axes)
AXES_FACTOR = float(np.sqrt(3.0))


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) hidden layers, zero output layer
    (so training starts exactly at the ES window)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, dtype=np.float32)
    o = 0
    for n, fan in ((32, 1), (32, 1), (1024, 32), (32, 32), (1024, 32), (32, 32)):
        p[o:o + n] = rng.uniform(-1, 1, n) / np.sqrt(fan)
        o += n
    return p                      # Wo, bo stay zero


def loss_and_grad(W: int, params: np.ndarray, sigma: float = 2.0):
    """(per-axis RMS error, gradient of its log) evaluated by the GPU kernel."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    loss = np.zeros(1)
    grad = np.zeros(NPARAMS, dtype=np.float32)
    _lib.check(_lib.lib.curig_window_loss_grad(W, sigma, params.ctypes.data, loss.ctypes.data,
                                               grad.ctypes.data), "window_loss_grad")
    return float(loss[0]), grad


def train(W: int, iters: int = 3000, lr: float = 3e-3, sigma: float = 2.0, params=None, seed: int = 0,
          mc_seed=None):
    """Adam on the GPU; returns (params, loss history).  mc_seed: train on
    random visibility offsets drawn afresh at every step (64 per step) from that
    seed, instead of the fixed grid of offsets."""
    p = init_params(seed) if params is None else np.array(params, dtype=np.float32)
    hist = np.zeros(max(iters, 1))
    if mc_seed is None:
        _lib.check(_lib.lib.curig_train_window(W, sigma, iters, lr, p.ctypes.data, hist.ctypes.data),
                   "train_window")
    else:
        _lib.check(_lib.lib.curig_train_window_mc(W, sigma, iters, lr, int(mc_seed), p.ctypes.data,
                                                  hist.ctypes.data), "train_window_mc")
    return p, hist[:iters]


def table(W: int, params: np.ndarray, sigma: float = 2.0, degree: int = DEGREE) -> np.ndarray:
    params = np.ascontiguousarray(params, dtype=np.float32)
    coef = np.zeros((W, degree + 1))
    _lib.check(_lib.lib.curig_window_table(W, sigma, params.ctypes.data, degree, coef.ctypes.data),
               "window_table")
    return coef


def register(W: int, params: np.ndarray, eps_reached: float, sigma: float = 2.0) -> None:
    coef = np.ascontiguousarray(table(W, params, sigma), dtype=np.float64)
    _lib.check(_lib.lib.curig_set_window(W, DEGREE, coef.ctypes.data, float(eps_reached)),
               "set_window")


def clear() -> None:
    _lib.lib.curig_clear_windows()


def load_default_windows(path: str = DEFAULT_FILE) -> bool:
    """Register the shipped sigma = 2 windows; False if none are available."""
    if not os.path.exists(path):
        return False
    data = json.load(open(path))
    n = 0
    for entry in data.get("windows", []):
        params = np.array(entry["params"], dtype=np.float32)
        if params.size != NPARAMS:
            continue
        register(int(entry["W"]), params, float(entry["eps_reached"]), float(data.get("sigma", 2.0)))
        n += 1
    return n > 0
