"""Learned window: GPU forward/backward against the CPU autograd oracle,
training gain over the ES start, tabulation accuracy, and what the trained
windows gain end to end against the FP64 DFT."""
import os

import numpy as np
import pytest

from conftest import disk_inputs, l2err


def test_table_reproduces_window_on_cpu():
    """curig_window_table is host code: the Horner table matches the MLP window."""
    import torch
    from curig_b200 import learned
    from oracle import learned_ref
    W = 6
    p = learned.init_params(3)
    p[-33:-1] = np.random.default_rng(1).normal(0, 0.05, 32).astype(np.float32)   # non-trivial g
    coef = learned.table(W, p)
    t = np.linspace(-W / 2 + 1e-6, W / 2 - 1e-6, 2001)
    ref = learned_ref.window(torch.tensor(p.astype(np.float64)), torch.tensor(t), W,
                             learned_ref.es_beta(W)).numpy()
    ref = ref / ref.max() if ref.max() > 0 else ref
    u = t + W / 2
    d = np.minimum(np.floor(u).astype(int), W - 1)
    s = 2 * (u - d) - 1
    got = np.array([np.polyval(coef[di], si) for di, si in zip(d, s)])
    assert np.max(np.abs(got - ref)) < 5e-7


@pytest.mark.gpu
@pytest.mark.parametrize("W", [4, 6, 8])
def test_gpu_loss_and_gradient_match_cpu_oracle(W):
    from curig_b200 import learned
    from oracle import learned_ref
    p = learned.init_params(W)
    rng = np.random.default_rng(W)
    p[-33:] = rng.normal(0, 0.02, 33).astype(np.float32)          # output layer away from zero
    L, g = learned.loss_and_grad(W, p)
    Lr, gr = learned_ref.objective(p, W)
    assert abs(L - Lr) <= 1e-8 * Lr
    assert np.linalg.norm(g - gr) <= 1e-5 * np.linalg.norm(gr)


@pytest.mark.gpu
def test_training_reduces_error_from_es_start():
    from curig_b200 import learned
    p0 = learned.init_params(0)
    l0, _ = learned.loss_and_grad(6, p0)
    p, hist = learned.train(6, iters=400, lr=3e-3, params=p0)
    l1, _ = learned.loss_and_grad(6, p)
    assert hist[0] == pytest.approx(l0, rel=1e-9)
    assert l1 < 0.8 * l0


@pytest.mark.gpu
def test_shipped_windows_beat_es_against_dft():
    """The trained windows (curig_b200/windows) against the ES window of the
    same width, both measured end to end against the exact DFT."""
    import torch
    from curig_b200 import GridderPlan, learned
    from oracle import dft
    assert learned.load_default_windows(), "trained windows missing"
    freq, uvw, ms, wgt = disk_inputs(2500, 1, 192, 2.0, max_pix=80, wmax=300, seed=11)
    n, psx = 192, 2.0 * np.pi / 180 / 192
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, n, n, psx, psx, 1)
    errs = {}
    for W in (5, 6):
        for window in ("es", "learned"):
            eps = 10.0 ** (1 - W) if window == "es" else learned_eps(W)
            p = GridderPlan(1, n, n, psx, psx, eps, 2.0, 1, precision="fp64", window=window)
            p.setpts(torch.from_numpy(uvw).cuda(), freq)
            assert p.info()["kw"] == W
            d = torch.empty((n, n), dtype=torch.complex128, device="cuda")
            p.execute(torch.from_numpy(ms).cuda(), torch.from_numpy(wgt).cuda(), d)
            errs[(W, window)] = l2err(ref, d.cpu().numpy())
            p.close()
    learned.clear()
    for W in (5, 6):
        assert errs[(W, "learned")] < 0.75 * errs[(W, "es")], errs


def learned_eps(W):
    import json
    from curig_b200 import learned
    for e in json.load(open(learned.DEFAULT_FILE))["windows"]:
        if e["W"] == W:
            return e["eps_reached"] * 1.0000001
    raise KeyError(W)
