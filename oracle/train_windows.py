"""Train the learned windows on the GPU and record their measured accuracy.

    python oracle/train_windows.py [out.json] [--iters N]

For each support width W (sigma = 2) the MLP window is trained by the
library's own kernels (curig_train_window), tabulated, and its error measured
end to end: ms2dirty (FP64) of a seeded 256 x 256 / 3000-visibility problem
with w-stacking against the exact FP64 DFT (oracle/dft.c, used here only as the
checker).  The ES window of the same width is measured on the same problem.
The output JSON holds the trained parameters and eps_reached (the measured
learned error) per width; curig_b200.learned.load_default_windows() reads it.
The recipe lives beside the oracle, not in the package: the package never
imports the oracle.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


def measure(W, window, params=None):
    """Relative l2 error of FP64 ms2dirty (window of width W) against the DFT."""
    import torch
    from curig_b200 import GridderPlan, learned
    from oracle import dft
    rng = np.random.default_rng(7)
    nrow, n, fov, f0 = 3000, 256, 2.0, 1.0e9
    R = 110 * (299792458.0 / f0) / (fov * np.pi / 180)
    r = R * np.sqrt(rng.random(nrow))
    th = 2 * np.pi * rng.random(nrow)
    uvw = np.stack([r * np.cos(th), r * np.sin(th), rng.uniform(-300, 300, nrow)], 1)
    vis = rng.standard_normal((nrow, 1)) + 1j * rng.standard_normal((nrow, 1))
    psx = fov * np.pi / 180 / n
    eps = 10.0 ** (1 - W)                    # the reference's width rule gives W at this epsilon
    learned.clear()
    if window == "learned":
        learned.register(W, params, 0.0)     # eps_reached 0: always eligible
    p = GridderPlan(1, n, n, psx, psx, eps, 2.0, -1, precision="fp64", window=window)
    p.setpts(torch.from_numpy(uvw).cuda(), np.array([f0]))
    assert p.info()["kw"] == W, p.info()
    d = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    p.execute(torch.from_numpy(vis).cuda(), None, d)
    out = d.cpu().numpy()
    p.close()
    ref = dft.ms2dirty_dft(uvw, [f0], vis, None, n, n, psx, psx, -1)
    learned.clear()
    return float(np.sqrt(np.sum(np.abs(out - ref) ** 2) / np.sum(np.abs(ref) ** 2)))


def main():
    from curig_b200 import learned
    out = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else learned.DEFAULT_FILE
    iters = int(sys.argv[sys.argv.index("--iters") + 1]) if "--iters" in sys.argv else 4000
    res = {"sigma": 2.0, "objective": "per-axis RMS error of gridding + correction vs exact DFT, "
                                      "image band |xi| <= 1/(2 sigma)", "iters": iters, "windows": []}
    for W in (4, 5, 6, 7, 8):
        t0 = time.time()
        p0 = learned.init_params(W)
        l0, _ = learned.loss_and_grad(W, p0)
        p, hist = learned.train(W, iters=iters, lr=3e-3, params=p0)
        p, hist2 = learned.train(W, iters=iters // 2, lr=1e-3, params=p)
        l1, _ = learned.loss_and_grad(W, p)
        e_es = measure(W, "es")
        e_l = measure(W, "learned", p)
        print(f"W={W}: objective ES {l0:.3e} -> learned {l1:.3e}; measured ms2dirty error ES {e_es:.3e}, "
              f"learned {e_l:.3e} ({time.time() - t0:.1f} s)", flush=True)
        res["windows"].append({"W": W, "eps_reached": e_l, "es_measured": e_es, "objective_es": l0,
                               "objective_learned": l1, "params": [float(x) for x in p]})
    os.makedirs(os.path.dirname(out), exist_ok=True)
    json.dump(res, open(out, "w"))
    print("wrote", out)


if __name__ == "__main__":
    main()
