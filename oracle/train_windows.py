"""Train the learned windows on the GPU and record their measured accuracy.

    python oracle/train_windows.py [out.json]

For each support width W (sigma = 2) the MLP window is trained by the
library's own kernels on method-generated random visibilities
(curig_train_window_mc: 64 random cell offsets per Adam step, 1.02e6 in all),
tabulated, and its error measured end to end against the exact FP64 DFT, used
here only as the checker: ms2dirty (FP64) of a seeded 256 x 256 /
3000-visibility problem with w-stacking (oracle/dft.c), and at the 4096^2
configuration's geometry on 2,000 sampled pixels (oracle/dft_torch.py).  The ES
window of the same width is measured on the same problems.  The output JSON
holds the trained parameters and eps_reached (the larger measured learned
error) per width; curig_b200.learned.load_default_windows() reads it.  The
recipe lives beside the oracle, not in the package: the package never imports
the oracle.
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


def measure_4096(W, window, params=None):
    """Relative l2 error of FP64 ms2dirty at the 4096^2 configuration's geometry
    (fov 3 deg, Gaussian u,v, w +-1000 m, 16 channels 0.9-1.1 GHz; 2e5 rows)
    against the FP64 DFT on 2,000 sampled pixels (oracle/dft_torch.py on the GPU)."""
    import torch
    from curig_b200 import GridderPlan, learned
    from oracle import dft_torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import gaussian_uv_inputs
    npix, fov = 4096, 3.0
    freq, uvw, vis, wgt = gaussian_uv_inputs(200_000, 16, npix, fov, seed=11)
    psx = fov * np.pi / 180 / npix
    pix = np.random.default_rng(12).choice(npix * npix, 2000, replace=False)
    eps = 10.0 ** (1 - W)
    learned.clear()
    if window == "learned":
        learned.register(W, params, 0.0)
    p = GridderPlan(1, npix, npix, psx, psx, eps, 2.0, -1, precision="fp64", window=window)
    u = torch.from_numpy(uvw).cuda()
    p.setpts(u, freq)
    assert p.info()["kw"] == W, p.info()
    d = torch.empty((npix, npix), dtype=torch.complex128, device="cuda")
    v, w = torch.from_numpy(vis).cuda(), torch.from_numpy(wgt).cuda()
    p.execute(v, w, d)
    got = d.reshape(-1)[torch.from_numpy(pix).cuda()].cpu().numpy()
    p.close()
    ref = dft_torch.ms2dirty_dft(u, freq, v, w, npix, npix, psx, psx, -1, pix)
    learned.clear()
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


def main():
    """Train every width on method-generated random visibilities (64 random
    offsets per step, three learning-rate stages, 16,000 steps: 1.02e6
    visibilities), then record the measured errors at 256^2 and at the
    4096^2 geometry; eps_reached (what a plan compares with epsilon) is the
    larger of the two."""
    from curig_b200 import learned
    out = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else learned.DEFAULT_FILE
    stages = [(8000, 3e-3), (5000, 1e-3), (3000, 3e-4)]
    nvis = 64 * sum(n for n, _ in stages)
    res = {"sigma": 2.0,
           "objective": "per-axis RMS error of gridding + correction vs exact DFT, image band |xi| <= 1/(2 sigma)",
           "training": f"{nvis} method-generated random visibilities (64 uniform cell offsets per Adam step, "
                       f"stages {stages})",
           "windows": []}
    for W in (4, 5, 6, 7, 8):
        t0 = time.time()
        p = learned.init_params(W)
        l0, _ = learned.loss_and_grad(W, p)
        for k, (n, lr) in enumerate(stages):
            p, _ = learned.train(W, iters=n, lr=lr, params=p, mc_seed=1000 * W + k)
        l1, _ = learned.loss_and_grad(W, p)
        e_es, e_l = measure(W, "es"), measure(W, "learned", p)
        g_es, g_l = measure_4096(W, "es"), measure_4096(W, "learned", p)
        print(f"W={W}: objective ES {l0:.3e} -> learned {l1:.3e}; ms2dirty error 256^2 ES {e_es:.3e} learned "
              f"{e_l:.3e}; 4096^2 ES {g_es:.3e} learned {g_l:.3e} ({time.time() - t0:.1f} s)", flush=True)
        res["windows"].append({"W": W, "eps_reached": max(e_l, g_l), "eps_256": e_l, "eps_4096": g_l,
                               "es_measured": max(e_es, g_es), "es_256": e_es, "es_4096": g_es,
                               "objective_es": l0, "objective_learned": l1, "params": [float(x) for x in p]})
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    json.dump(res, open(out, "w"))
    print("wrote", out)


if __name__ == "__main__":
    main()
