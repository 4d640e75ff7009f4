#!/usr/bin/env python
"""Benchmark: visibilities/s of ms2dirty + dirty2ms on one B200 (or N, weak scaling).

Workload (the 4096^2 configuration): 1e7 rows x 16 channels (0.9-1.1 GHz)
= 1.6e8 visibilities, 4096 x 4096 image, fov 3 deg, sigma 2, epsilon 1e-5,
u,v from an isotropic Gaussian baseline density (sigma = 0.3 R, truncated at
R, R * fov / lambda_min = 0.47 * 4096 pixels), w uniform in +-1000 m, complex
normal visibilities, weights uniform in (0.5, 1]; seeded synthetic data
generated on the device (no dataset exists for this configuration).

One step = set points (w range, sizing, binning) + ms2dirty + dirty2ms over
the whole visibility set, inputs resident in HBM (`value`); `e2e` is the same
step through the C ABI one-shot calls (curig_ms2dirty / curig_dirty2ms) from
pinned host buffers, host<->device copies inside the timed region.  For N > 1
each rank grids its own 1.6e8 visibilities and the partial dirty images are
summed with one NCCL all-reduce before the degridding (weak scaling).

`--impl reference` times the reference's CPU path for this transform (its
explicit FP64 DFT, python/curagridder/test_wst.py:15-32, restated in C/OpenMP
in oracle/dft.c) on the host cores over a bounded sample, extrapolated to the
full workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

C = 299792458.0
METRIC = "vis/s ms2dirty & dirty2ms at eps=1e-5: learned-kernel vs ES, same B200"


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="curig", choices=["curig", "reference"])
    ap.add_argument("--nrow", type=int, default=10_000_000)
    ap.add_argument("--nchan", type=int, default=16)
    ap.add_argument("--npix", type=int, default=4096)
    ap.add_argument("--fov", type=float, default=3.0)
    ap.add_argument("--eps", type=float, default=1e-5)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--window", default="auto", choices=["auto", "es", "learned"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-arms", action="store_true", help="skip the comparison arms (ES, FP64, exact FP32)")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="skip timing the reference's own GPU library (oracle/_ref) beside this one")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--accumulate", type=int, default=0, help="tile accumulation: 0 automatic, 1 float atomics, 2 one-word int32 fixed point, 3 two-word (exact); FP64: 1 double atomics, else exact three-word int32")
    ap.add_argument("--bin", type=int, default=0, help="bin edge in cells (0 automatic)")
    ap.add_argument("--smem", type=int, default=0, help="shared-memory budget per tile CTA (bytes)")
    ap.add_argument("--sub", type=int, default=0, help="visibilities per tile chunk (0 automatic)")
    ap.add_argument("--sparse", type=int, default=0,
                    help="FP32 spreader: chunks below this many visibilities skip the tile (0 automatic, -1 never)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="row slabs of the one-shot calls timed as e2e (0 automatic, 1..8)")
    ap.add_argument("--error-table", action="store_true",
                    help="print errors per epsilon and precision form (FP64 DFT, FP64 GPU) and exit")
    return ap.parse_args()


def bench_config(a, world):
    """The workload description both arms print (a function of the arguments only)."""
    acc = {0: "automatic", 1: "float atomics", 2: "one-word int32 fixed point",
           3: "two-word int32 fixed point (exact)"}.get(a.accumulate, str(a.accumulate))
    return {"workload": f"ms2dirty+dirty2ms, {a.nrow} rows x {a.nchan} ch ({a.nrow * a.nchan} vis), "
                        f"{a.npix}^2, fov {a.fov} deg, eps {a.eps}, sigma 2",
            "window": a.window, "precision": a.precision, "accumulate": acc,
            "l2": "inputs (>= 1.9 GB per step) larger than L2; no flush needed",
            "parallelism": f"dp{world} (visibility shards, all-reduce of dirty)" if world > 1 else "single GPU"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def workload(torch, nrow, nchan, npix, fov, seed, device):
    """Seeded synthetic visibilities on the device."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    freq = np.linspace(0.9e9, 1.1e9, nchan) if nchan > 1 else np.array([1.0e9])
    lam_min = C / freq.max()
    R = 0.47 * npix * lam_min / (fov * np.pi / 180)
    s = 0.3 * R
    uv = torch.randn((nrow, 2), generator=g, device=device, dtype=torch.float64) * s
    for _ in range(64):                                  # truncate the Gaussian at R
        bad = (uv * uv).sum(1) > R * R
        nb = int(bad.sum())
        if nb == 0:
            break
        uv[bad] = torch.randn((nb, 2), generator=g, device=device, dtype=torch.float64) * s
    w = (torch.rand((nrow, 1), generator=g, device=device, dtype=torch.float64) * 2 - 1) * 1000.0
    uvw = torch.cat([uv, w], 1).contiguous()
    vis = torch.complex(torch.randn((nrow, nchan), generator=g, device=device),
                        torch.randn((nrow, nchan), generator=g, device=device))
    wgt = 1.0 - torch.rand((nrow, nchan), generator=g, device=device) * 0.5   # (0.5, 1]
    return freq, uvw, vis.contiguous(), wgt.contiguous()


class Clocks:
    """nvidia-smi samples during the timed region (recipe's clocks line)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        fd, self.path = tempfile.mkstemp(prefix="curig_clocks_", suffix=".csv")
        os.close(fd)
        self.p = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        except Exception:
            return None
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def measured_peak():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(uvw_h, freq, vis_h, wgt_h, npix, fov, target_s):
    """Reference CPU path (explicit FP64 DFT, oracle/dft.c port) on a bounded
    sample: nv visibilities x np pixels, extrapolated to full-image vis/s."""
    from oracle import dft
    psx = fov * np.pi / 180 / npix
    nchan = len(freq)
    rng = np.random.default_rng(0)
    nrow_s = max(1, 20000 // nchan)
    u = uvw_h[:nrow_s]
    v = vis_h[:nrow_s]
    w = wgt_h[:nrow_s]
    npx, t1 = 64, 0.0
    while t1 < 0.5 and npx < npix * npix:                  # calibrate to ~target_s seconds
        npx *= 4
        t0 = time.perf_counter()
        dft.ms2dirty_dft(u, freq, v, w, npix, npix, psx, psx, -1, pix=rng.integers(0, npix * npix, npx))
        t1 = time.perf_counter() - t0
    npx = int(min(npix * npix, max(64, npx * target_s / max(t1, 1e-3))))
    pix = rng.integers(0, npix * npix, npx)
    t0 = time.perf_counter()
    dft.ms2dirty_dft(u, freq, v, w, npix, npix, psx, psx, -1, pix=pix)
    t = time.perf_counter() - t0
    rate = nrow_s * nchan * npx / t                          # pixel * vis / s
    vis_per_s = rate / (2.0 * npix * npix)                   # ms2dirty + dirty2ms over the full image
    return {"value": vis_per_s, "unit": "vis/s", "cores": os.cpu_count(), "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"{nrow_s * nchan} vis x {npx} pixels of the {npix}^2 image, FP64 DFT "
                      f"(oracle/dft.c, OpenMP), {t:.1f} s; extrapolated to ms2dirty+dirty2ms over "
                      f"all pixels", "pixel_vis_per_s": rate, "sample_seconds": t}


def numpy_explicit_baseline(uvw_h, freq, vis_h, npix, fov, target_s):
    """The reference's own CPU path as it runs: its numpy explicit gridder and
    degridder (restated in oracle/explicit_numpy.py), one process, whole-image
    array operations per visibility, on the full npix^2 image for a few
    visibilities; vis/s of ms2dirty + dirty2ms over the full image."""
    from oracle import explicit_numpy as X
    psx = fov * np.pi / 180 / npix
    img = np.zeros((npix, npix))
    n, t = 1, 0.0
    while True:
        t0 = time.perf_counter()
        X.explicit_gridder(uvw_h[:n], freq[:1], vis_h[:n, :1], npix, npix, psx, psx)
        X.explicit_degridder(uvw_h[:n], freq[:1], img, psx, psx, -1)
        t = time.perf_counter() - t0
        if t >= target_s or n >= 64:
            break
        n = max(n + 1, int(n * min(8.0, 1.2 * target_s / max(t, 1e-3))))
    return {"value": n / t, "unit": "vis/s", "cores": 1, "kind": "port",
            "sample": f"{n} vis, ms2dirty + dirty2ms each over the full {npix}^2 image (numpy, "
                      f"one process), {t:.1f} s", "sample_seconds": t}


def _bind_reference_abi(path):
    """ms2dirty_2 / dirty2ms_2 of a libcurafft.so with plain pointer arguments
    (include/cugridder.h:13-20 of the reference)."""
    import ctypes
    lib = ctypes.CDLL(path)
    P, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    for name in ("ms2dirty_2", "dirty2ms_2"):
        f = getattr(lib, name)
        f.argtypes = [ci, ci, ci, cd, cd, P, P, P, P, cd, cd, ci]
        f.restype = ci
    return lib


def reference_gpu(torch, uvw, freq, vis, wgt, npix, fov, eps):
    """The reference's own GPU library on the same B200, beside this library's
    reference ABI: libcurafft.so built for sm_100a from the reference's sources
    (oracle/Makefile.ref, flag-only changes) into oracle/_ref/, called through
    its stock one-shot ABI (ms2dirty_2 / dirty2ms_2: FP64, host buffers, one
    frequency per call, src/astro/cugridder.cu:587-612) once per channel, as its
    Python package does (python/curagridder/curagridder.py:92 passes freq[0]).
    Each call is one 1e7-row single-channel FP64 transform with its own copies.
    The same 2 x nchan calls then go through this library's reference ABI.
    Wall time of the calls alone; the host-side channel sum is not timed.
    The outputs of the two libraries are compared over the whole image and
    all visibilities."""
    path = os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libcurafft_ref.so not built (needs the reference sources)"}
    from curig_b200 import _lib
    ref, mine = _bind_reference_abi(path), _bind_reference_abi(_lib.LIB_PATH)
    nrow, nchan = vis.shape
    fovd = float(fov)
    h_uvw = uvw.to(torch.float64).contiguous().cpu().pin_memory()
    vis_ch = [vis[:, c].to(torch.complex128).contiguous().cpu().pin_memory() for c in range(nchan)]
    wgt_ch = [wgt[:, c].to(torch.float64).contiguous().cpu().pin_memory() for c in range(nchan)]
    img = torch.complex(torch.randn((npix, npix), dtype=torch.float64),
                        torch.randn((npix, npix), dtype=torch.float64)).pin_memory()
    out = torch.empty((npix, npix), dtype=torch.complex128).pin_memory()
    vout = torch.empty(nrow, dtype=torch.complex128).pin_memory()

    def step(lib, keep_vis):
        """One step of 2 x nchan reference-ABI calls: (seconds in the calls,
        dirty image summed over channels, per-channel visibilities if kept)."""
        t = 0.0
        acc = torch.zeros((npix, npix), dtype=torch.complex128)
        kept = []
        for c in range(nchan):
            t0 = time.perf_counter()
            s1 = lib.ms2dirty_2(nrow, npix, npix, fovd, float(freq[c]), h_uvw.data_ptr(), vis_ch[c].data_ptr(),
                                wgt_ch[c].data_ptr(), out.data_ptr(), eps, 2.0, -1)
            t += time.perf_counter() - t0
            acc += out
            t0 = time.perf_counter()
            s2 = lib.dirty2ms_2(nrow, npix, npix, fovd, float(freq[c]), h_uvw.data_ptr(), vout.data_ptr(),
                                wgt_ch[c].data_ptr(), img.data_ptr(), eps, 2.0, -1)
            t += time.perf_counter() - t0
            if s1 or s2:
                raise RuntimeError(f"reference ABI status {s1} / {s2}")
            if keep_vis:
                kept.append(vout.clone())
        return t, acc, kept

    # warm-up: one channel through each library (context, module loading)
    for lib in (ref, mine):
        lib.ms2dirty_2(nrow, npix, npix, fovd, float(freq[0]), h_uvw.data_ptr(), vis_ch[0].data_ptr(),
                       wgt_ch[0].data_ptr(), out.data_ptr(), eps, 2.0, -1)
    t_ref, d_ref, v_ref = step(ref, True)
    t_mine, d_mine, v_mine = step(mine, True)
    num_v = sum(float(torch.sum(torch.abs(x - y) ** 2)) for x, y in zip(v_mine, v_ref))
    den_v = sum(float(torch.sum(torch.abs(y) ** 2)) for y in v_ref)
    M = nrow * nchan
    return {"value": M / t_ref, "unit": "vis/s", "ms_per_step": round(1e3 * t_ref, 1),
            "this_library_same_calls": {"value": M / t_mine, "ms_per_step": round(1e3 * t_mine, 1)},
            "speedup_same_calls": round(t_ref / t_mine, 2),
            "rel_diff_ms2dirty": float(torch.linalg.vector_norm(d_mine - d_ref) / torch.linalg.vector_norm(d_ref)),
            "rel_diff_dirty2ms": float(np.sqrt(num_v / den_v)),
            "calls": f"{nchan} x ms2dirty_2 + {nchan} x dirty2ms_2, {nrow} rows each, FP64, eps {eps}, "
                     f"pinned host buffers, wall time of the calls",
            "library": "reference libcurafft.so built for sm_100a from its sources (flag-only changes)"}


def es_width_for(eps):
    """Smallest ES width whose measured error (shipped window study, 256^2 FP64
    against the DFT) is <= eps, and an epsilon that makes the reference's width
    rule pick it; falls back to the rule itself."""
    try:
        from curig_b200 import learned
        data = json.load(open(learned.DEFAULT_FILE))
        ok = sorted(e["W"] for e in data["windows"] if e["es_measured"] <= eps)
        if ok:
            return ok[0], 10.0 ** (1 - ok[0]), {e["W"]: e for e in data["windows"]}
    except Exception:
        pass
    return None, eps, {}


def accuracy_probe(torch, plan_kw, uvw, freq, vis, wgt, npix, fov, nrow_s=1250, npx=192):
    """Relative l2 error of one ms2dirty on a visibility subset at the full image
    geometry against the FP64 DFT (oracle/dft.c as the checker) on sampled pixels."""
    from curig_b200.plan import GridderPlan
    from oracle import dft
    psx = fov * np.pi / 180 / npix
    u = uvw[:nrow_s].contiguous()
    v = vis[:nrow_s].contiguous()
    w = wgt[:nrow_s].contiguous()
    p = GridderPlan(1, npix, npix, psx, psx, **plan_kw)
    p.setpts(u, freq)
    d = torch.empty((npix, npix), dtype=v.dtype, device=v.device)
    p.execute(v, w, d)
    torch.cuda.synchronize()
    p.close()
    pix = np.random.default_rng(5).integers(0, npix * npix, npx)
    got = d.reshape(-1)[torch.from_numpy(pix).to(d.device)].cpu().numpy()
    ref = dft.ms2dirty_dft(u.cpu().numpy(), freq, v.cpu().numpy().astype(np.complex128),
                           w.cpu().numpy().astype(np.float64), npix, npix, psx, psx, -1, pix=pix)
    return float(np.sqrt(np.sum(np.abs(got - ref) ** 2) / np.sum(np.abs(ref) ** 2)))


def accumulation_check(torch, plan_kw, accumulate, uvw, freq, vis, wgt, npix, fov):
    """Relative l2 difference of one full-workload ms2dirty accumulated in the
    given FP32 tile mode against the exact two-word fixed-point mode."""
    from curig_b200.plan import GridderPlan
    psx = fov * np.pi / 180 / npix
    out = []
    for acc in (accumulate, 3):
        p = GridderPlan(1, npix, npix, psx, psx, accumulate=acc, **plan_kw)
        p.setpts(uvw, freq)
        d = torch.empty((npix, npix), dtype=vis.dtype, device=vis.device)
        p.execute(vis, wgt, d)
        torch.cuda.synchronize()
        p.close()
        out.append(d)
    return float(torch.linalg.vector_norm(out[0] - out[1]) / torch.linalg.vector_norm(out[1]))


def batch8_autograd(torch, dev, steps, warmup, seed, window):
    """8 independent problems, 1e6 visibilities each (1 channel at 1 GHz),
    1024^2, fov 2 deg, FP32, eps 1e-5: one step = differentiable ms2dirty of
    all 8 + backward of ||dirty - d||^2 to the visibilities and weights.
    Points are set once (outside the timed region); inputs on the device."""
    from curig_b200.autograd import BatchGridder
    B, nrow, npix, fov = 8, 1_000_000, 1024, 2.0
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 1000)
    lam = C / 1.0e9
    R = 0.47 * npix * lam / (fov * np.pi / 180)
    uvws = []
    for _ in range(B):
        r = R * torch.sqrt(torch.rand(nrow, generator=g, device=dev, dtype=torch.float64))
        th = 2 * np.pi * torch.rand(nrow, generator=g, device=dev, dtype=torch.float64)
        w = (torch.rand(nrow, generator=g, device=dev, dtype=torch.float64) * 2 - 1) * 200.0
        uvws.append(torch.stack([r * torch.cos(th), r * torch.sin(th), w], 1).contiguous())
    vis = torch.complex(torch.randn((B, nrow, 1), generator=g, device=dev),
                        torch.randn((B, nrow, 1), generator=g, device=dev))
    wgt = 1.0 - torch.rand((B, nrow, 1), generator=g, device=dev) * 0.5
    d = torch.complex(torch.randn((B, npix, npix), generator=g, device=dev),
                      torch.randn((B, npix, npix), generator=g, device=dev))
    psx = fov * np.pi / 180 / npix
    bg = BatchGridder(uvws, np.array([1.0e9]), npix, npix, psx, psx, 1e-5, precision="fp32", window=window)

    def step():
        v = vis.detach().requires_grad_()
        w = wgt.detach().requires_grad_()
        loss = ((bg.ms2dirty(v, w) - d).abs() ** 2).sum()
        loss.backward()
        return v.grad, w.grad

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    bg.close()
    return {"value": B * nrow / (ms / 1e3), "unit": "vis/s", "ms_per_step": round(ms, 3),
            "workload": "8 problems x 1e6 vis (1 ch), 1024^2, fov 2 deg, eps 1e-5, FP32; "
                        "step = ms2dirty + backward to vis and wgt (points set once)"}


def error_table(a, torch, dev):
    """Errors per epsilon and precision form on the bench workload's geometry.
    DFT columns: one ms2dirty / dirty2ms of a visibility subset against the FP64
    DFT (2000 pixels / 2000 visibilities); full-density columns: FP32 ms2dirty of
    all visibilities against the FP64 one (isolates the FP32 arithmetic)."""
    from curig_b200.plan import GridderPlan
    from oracle import dft
    freq, uvw, vis, wgt = workload(torch, a.nrow, a.nchan, a.npix, a.fov, a.seed, dev)
    psx = a.fov * np.pi / 180 / a.npix
    rng = np.random.default_rng(11)
    pix = rng.integers(0, a.npix * a.npix, 2000)
    ns = 2000 // a.nchan + 1
    u_s, v_s, w_s = uvw[:ns].contiguous(), vis[:ns].contiguous(), wgt[:ns].contiguous()
    ref = dft.ms2dirty_dft(u_s.cpu().numpy(), freq, v_s.cpu().numpy().astype(np.complex128),
                           w_s.cpu().numpy().astype(np.float64), a.npix, a.npix, psx, psx, -1, pix=pix)
    img = rng.standard_normal((a.npix, a.npix)) + 1j * rng.standard_normal((a.npix, a.npix))
    vref = dft.dirty2ms_dft(u_s.cpu().numpy(), freq, img, w_s.cpu().numpy().astype(np.float64), psx, psx, -1)

    def rel(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    def run(prec, acc, eps, u, v, w, direction, dirty_in=None):
        cdt = torch.complex64 if prec == "fp32" else torch.complex128
        rdt = torch.float32 if prec == "fp32" else torch.float64
        p = GridderPlan(1, a.npix, a.npix, psx, psx, eps, 2.0, -1, precision=prec, window="es", accumulate=acc)
        p.setpts(u, freq)
        vv, ww = v.to(cdt), w.to(rdt)
        if direction == 1:
            out = torch.empty((a.npix, a.npix), dtype=cdt, device=dev)
            p.execute_dir(1, vv, ww, out)
        else:
            out = torch.empty_like(vv)
            p.execute_dir(2, out, ww, torch.from_numpy(dirty_in).to(cdt).to(dev))
        torch.cuda.synchronize()
        p.close()
        return out

    forms = [("fp64", 0, "FP64"), ("fp32", 3, "FP32 two-word (exact tiles)"), ("fp32", 2, "FP32 one-word"),
             ("fp32", 1, "FP32 float atomics")]
    table = []
    for eps in (1e-4, 1e-5, 1e-6):
        full64 = run("fp64", 0, eps, uvw, vis, wgt, 1)
        for prec, acc, name in forms:
            d = run(prec, acc, eps, u_s, v_s, w_s, 1).reshape(-1)[torch.from_numpy(pix).to(dev)].cpu().numpy()
            vo = run(prec, acc, eps, u_s, v_s, w_s, 2, img).cpu().numpy()
            row = {"eps": eps, "form": name, "ms2dirty_vs_dft": rel(d, ref), "dirty2ms_vs_dft": rel(vo, vref)}
            if prec == "fp32":
                full = run(prec, acc, eps, uvw, vis, wgt, 1)
                row["ms2dirty_full_vs_fp64"] = float(torch.linalg.vector_norm(full.to(torch.complex128) - full64)
                                                     / torch.linalg.vector_norm(full64))
                del full
            table.append(row)
        del full64
    return {"error_table": table, "workload": f"{a.nrow} rows x {a.nchan} ch, {a.npix}^2, fov {a.fov} deg, ES window; "
            f"DFT columns: {ns} rows on 2000 pixels / all their visibilities"}


def main():
    a = args_()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return reference_arm(a, rank, world)
    import torch
    if a.error_table:
        torch.cuda.set_device(local)
        print(json.dumps(error_table(a, torch, torch.device("cuda", local))))
        return 0
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from curig_b200.plan import GridderPlan, launch_count, set_timing

    freq, uvw, vis, wgt = workload(torch, a.nrow, a.nchan, a.npix, a.fov, a.seed + rank, dev)
    M = a.nrow * a.nchan
    psx = a.fov * np.pi / 180 / a.npix
    cdt = torch.complex64 if a.precision == "fp32" else torch.complex128
    rdt = torch.float32 if a.precision == "fp32" else torch.float64
    vis = vis.to(cdt)
    wgt = wgt.to(rdt)
    window = "es"
    if a.window in ("auto", "learned"):
        from curig_b200 import learned
        have = learned.load_default_windows()
        if a.window == "learned" and not have:
            raise RuntimeError("no trained windows found")
        window = "learned" if have else "es"
    stream = torch.cuda.current_stream()
    dirty = torch.empty((a.npix, a.npix), dtype=cdt, device=dev)
    vout = torch.empty_like(vis)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # every arm accumulates like the headline (automatic mode resolved at its epsilon)
    acc_mode = a.accumulate or (2 if a.eps >= 1e-5 else 3)

    def time_arm(win, eps, steps, warmup, with_clocks=False, precision=None, accumulate=None):
        prec = precision or a.precision
        if prec == a.precision:
            v_, w_, d_, o_ = vis, wgt, dirty, vout
        else:                                            # another precision: its own copies
            c_ = torch.complex64 if prec == "fp32" else torch.complex128
            v_, w_ = vis.to(c_), wgt.to(torch.float32 if prec == "fp32" else torch.float64)
            d_, o_ = torch.empty((a.npix, a.npix), dtype=c_, device=dev), torch.empty_like(v_)
        plan = GridderPlan(1, a.npix, a.npix, psx, psx, eps, 2.0, -1, precision=prec, window=win,
                           stream=stream, bin_xy=a.bin, sub=a.sub, smem_budget=a.smem,
                           accumulate=acc_mode if accumulate is None else accumulate, sparse=a.sparse)

        def step():
            plan.setpts(uvw, freq)
            plan.execute_dir(1, v_, w_, d_)
            if world > 1:
                torch.distributed.all_reduce(d_)
            plan.execute_dir(2, o_, w_, d_)

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        set_timing(True)
        stages = []
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        n0 = launch_count()
        clk = Clocks(local) if with_clocks else None
        if clk:
            clk.__enter__()
        ev0.record(stream)
        for _ in range(steps):
            step()
            stages.append(plan.timings())
        ev1.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__()
        if world > 1:
            torch.distributed.barrier()
        launches = launch_count() - n0
        set_timing(False)
        ms = ev0.elapsed_time(ev1) / steps
        if world > 1:
            t = torch.tensor([ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        info = plan.info()
        info["error_estimate"] = plan.error_estimate()
        plan.close()
        st = {k: float(np.mean([s[k] for s in stages])) for k in stages[0]}
        return {"value": M * world / (ms / 1e3), "ms": ms, "stages": st, "info": info,
                "launches": launches // steps, "clocks": clk.summary() if clk else None}

    head = time_arm(window, a.eps, a.steps, a.warmup, with_clocks=True)
    value, ms, st, info = head["value"], head["ms"], head["stages"], head["info"]

    # ES arms beside the learned one (single process only, to keep N > 1 runs short)
    arms = {}
    if world == 1 and window == "learned" and not a.no_arms:
        w_es, eps_es, table = es_width_for(a.eps)
        ks = max(2, a.steps // 2)
        if w_es is not None:
            r = time_arm("es", eps_es, ks, 2)
            arms["es_equal_error"] = {"value": r["value"], "ms_per_step": round(r["ms"], 3), "kw": r["info"]["kw"],
                                      "measured_error_256": table[w_es]["es_measured"],
                                      "rule": "smallest ES width whose measured error <= eps"}
        r = time_arm("es", a.eps, ks, 2)
        kw = r["info"]["kw"]
        arms["es_reference_rule"] = {"value": r["value"], "ms_per_step": round(r["ms"], 3), "kw": kw,
                                     "measured_error_256": table.get(kw, {}).get("es_measured"),
                                     "rule": "kw = ceil(-log10(eps/10)) (conv_interp_invoker.cu:84)"}
        if table:
            arms["learned_measured_error_256"] = table[info["kw"]]["eps_reached"]
    if world == 1 and not a.no_arms:
        # the exact (compensated) FP32 tile form at the headline epsilon and window
        if a.precision == "fp32" and acc_mode != 3:
            r = time_arm(window, a.eps, max(2, a.steps // 2), 2, accumulate=3)
            arms["fp32_two_word_exact"] = {"value": r["value"], "ms_per_step": round(r["ms"], 3),
                                           "kw": r["info"]["kw"], "window": window,
                                           "accumulate": "two-word int32 fixed point (exact)"}
        # the reference's arithmetic: FP64, ES window at the reference's width rule
        r = time_arm("es", a.eps, max(2, a.steps // 2), 2, precision="fp64", accumulate=0)
        arms["fp64_es_reference_rule"] = {"value": r["value"], "ms_per_step": round(r["ms"], 3),
                                          "kw": r["info"]["kw"], "window": "es",
                                          "accumulate": "three-word int32 fixed point (exact)"}
        torch.cuda.empty_cache()

    # batch of 8 independent problems through the autograd pair (single process)
    batch8 = None
    if world == 1 and not a.no_arms:
        batch8 = batch8_autograd(torch, dev, max(3, a.steps), a.warmup, a.seed, window)

    # accuracy at the full image geometry (visibility subset vs the FP64 DFT)
    acc = None
    if rank == 0 and not a.no_cpu:
        try:
            base = dict(sigma=2.0, sign=-1, precision=a.precision, accumulate=acc_mode, sub=a.sub)
            acc = {"headline": accuracy_probe(torch, dict(base, epsilon=a.eps, window=window), uvw, freq, vis,
                                              wgt, a.npix, a.fov)}
            if a.precision == "fp32" and acc_mode != 3:
                acc["accumulation_vs_exact"] = accumulation_check(
                    torch, dict(sigma=2.0, sign=-1, precision=a.precision, epsilon=a.eps, window=window, sub=a.sub,
                                bin_xy=a.bin), acc_mode, uvw, freq, vis, wgt, a.npix, a.fov)
            if "es_equal_error" in arms:
                acc["es_equal_error"] = accuracy_probe(torch, dict(base, epsilon=10.0 ** (1 - arms["es_equal_error"]["kw"]),
                                                                   window="es"), uvw, freq, vis, wgt, a.npix, a.fov)
            if "es_reference_rule" in arms:
                acc["es_reference_rule"] = accuracy_probe(torch, dict(base, epsilon=a.eps, window="es"), uvw,
                                                          freq, vis, wgt, a.npix, a.fov)
        except Exception as exc:  # pragma: no cover
            acc = {"error": str(exc)}

    # roofline of the dominant kernel (algorithmic bytes per launch, live event times)
    c = 8 if a.precision == "fp32" else 16
    r = c // 2
    G = info["nf1"] * info["nf2"] * info["nf3"]
    alg = {"spread": 24 * a.nrow + M * (c + r) + G * c,
           "interp": G * c + 24 * a.nrow + M * (r + c)}
    dom = "spread" if st["spread"] >= st["interp"] else "interp"
    peak, peak_kind = measured_peak()
    achieved = alg[dom] / (st[dom] / 1e3) / 1e9
    traffic = None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        key = f"{dom}_{a.precision}_kw{info['kw']}"
        wl = prof.get("workload", {})
        same = all(wl.get(k) == v for k, v in (("nrow", a.nrow), ("nchan", a.nchan), ("npix", a.npix),
                                               ("fov", a.fov), ("eps", a.eps)))
        if key in prof and same:
            traffic = prof[key]["bytes_per_launch"]
    except Exception:
        pass
    kname = {"spread": "k_spread_f32" if a.precision == "fp32" else "k_spread_t", "interp": "k_interp_t"}
    roof = {"bound": "hbm", "kernel": kname[dom], "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "algorithmic_bytes": alg[dom], "kernel_ms": round(st[dom], 3)}
    # The spreader's binding limit is shared-memory integer atomics (FP32 tiles: two
    # per tap, one per component); measured on this part: 27.6 int32 atomics per
    # clock per SM without bank conflicts.  Taps per second against that peak at
    # the SM clock sampled during the timed region.
    clk_mhz = (head["clocks"] or {}).get("sm_mhz")
    if a.precision == "fp32" and clk_mhz:
        taps = M * info["kw"] ** 3 / (st["spread"] / 1e3)
        tap_peak = 27.6 / 2 * torch.cuda.get_device_properties(dev).multi_processor_count * clk_mhz * 1e6
        roof["shared_atomic_bound"] = {"kernel": kname["spread"], "achieved_taps_per_s": taps,
                                       "peak_taps_per_s": tap_peak, "frac": round(taps / tap_peak, 4),
                                       "peak_basis": "27.6 int32 shared atomics / clock / SM (measured), "
                                                     "2 per tap, sampled SM clock"}

    # e2e through the C ABI with pinned host buffers
    e2e = None
    if not a.no_e2e:
        import ctypes
        from curig_b200 import _lib
        h_uvw = uvw.cpu().pin_memory()
        h_vis = vis.cpu().pin_memory()
        h_wgt = wgt.cpu().pin_memory()
        h_dirty = torch.empty((a.npix, a.npix), dtype=cdt).pin_memory()
        h_vout = torch.empty_like(h_vis).pin_memory()
        fr = np.ascontiguousarray(freq, dtype=np.float64)
        opts = _lib.make_opts(1 if a.precision == "fp32" else 0, 1 if window == "learned" else 0,
                              a.bin, a.sub, a.smem, stream.cuda_stream, a.accumulate, slabs=a.slabs)

        def e2e_step():
            s1 = _lib.lib.curig_ms2dirty(a.nrow, a.nchan, a.npix, a.npix, psx, psx, fr.ctypes.data,
                                         h_uvw.data_ptr(), h_vis.data_ptr(), h_wgt.data_ptr(),
                                         h_dirty.data_ptr(), a.eps, 2.0, -1, ctypes.byref(opts))
            s2 = _lib.lib.curig_dirty2ms(a.nrow, a.nchan, a.npix, a.npix, psx, psx, fr.ctypes.data,
                                         h_uvw.data_ptr(), h_vout.data_ptr(), h_wgt.data_ptr(),
                                         h_dirty.data_ptr(), a.eps, 2.0, -1, ctypes.byref(opts))
            _lib.check(s1, "curig_ms2dirty")
            _lib.check(s2, "curig_dirty2ms")

        for _ in range(min(a.warmup, 2)):
            e2e_step()
        ke = max(1, min(a.steps, 3))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(ke):
            e2e_step()
        ev1.record(stream)
        torch.cuda.synchronize()
        ems = ev0.elapsed_time(ev1) / ke
        if world > 1:                                    # whole job: slowest rank
            t = torch.tensor([ems], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ems = float(t.item())
        bi = 2 * h_uvw.numel() * 8 + h_vis.numel() * h_vis.element_size() + \
            2 * h_wgt.numel() * h_wgt.element_size() + h_dirty.numel() * h_dirty.element_size()
        bo = h_dirty.numel() * h_dirty.element_size() + h_vout.numel() * h_vout.element_size()
        e2e = {"value": M * world / (ems / 1e3), "unit": "vis/s", "h2d_bytes_per_step": int(bi),
               "d2h_bytes_per_step": int(bo), "ms_per_step": round(ems, 3), "steps": ke,
               "api": "curig_ms2dirty + curig_dirty2ms (C ABI, pinned host buffers)",
               "slabs": a.slabs or "automatic"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        n = max(1, 20000 // a.nchan)
        cpu = cpu_baseline(uvw[:n].cpu().numpy(), freq, vis[:n].cpu().numpy().astype(np.complex128),
                           wgt[:n].cpu().numpy().astype(np.float64), a.npix, a.fov, a.cpu_seconds)
        cpu["numpy_explicit"] = numpy_explicit_baseline(uvw[:64].cpu().numpy(), freq,
                                                        vis[:64].cpu().numpy().astype(np.complex128),
                                                        a.npix, a.fov, min(a.cpu_seconds, 8.0))

    refgpu = None
    if rank == 0 and world == 1 and not a.no_refgpu:
        try:
            refgpu = reference_gpu(torch, uvw, freq, vis, wgt, a.npix, a.fov, a.eps)
        except Exception as exc:  # pragma: no cover
            refgpu = {"error": str(exc)}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "vis/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if a.precision == "fp32" else "f64",
            "data": "synthetic (seeded Gaussian uv density, uniform w, complex-normal vis; generated on device)",
            "config": bench_config(a, world),
            "plan": {"window": window, "kw": info["kw"], "nf": [info["nf1"], info["nf2"], info["nf3"]],
                     "bin_xy": info["bin_xy"], "error_estimate": info["error_estimate"],
                     "accumulate": ({1: "float atomics", 2: "one-word int32 fixed point",
                                     3: "two-word int32 fixed point (exact)"}[acc_mode] if a.precision == "fp32" else
                                    "double atomics" if acc_mode == 1 else "three-word int32 fixed point (exact)")},
            "reference_gpu": refgpu,
            "e2e": e2e, "gpu_launches": int(head["launches"]), "clocks": head["clocks"],
            "roofline": roof, "cpu_baseline": cpu, "arms": arms, "batch8_autograd": batch8,
            "accuracy_vs_dft": acc,
            "stages_ms": {k: round(v, 3) for k, v in st.items()},
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def reference_arm(a, rank, world):
    """The reference's CPU path for this transform on the host cores: its
    explicit FP64 DFT (python/curagridder/test_wst.py:15-32,
    explicit_test.py:32-54), as the C/OpenMP port oracle/dft.c on all host
    threads.  One step = one bounded sample of the workload (ms_per_step is the
    sample's measured duration); value = the vis/s that rate gives for
    ms2dirty + dirty2ms over the full workload (extrapolated_ms_per_step)."""
    if rank != 0:
        return
    rng = np.random.default_rng(a.seed)
    nchan = a.nchan
    freq = np.linspace(0.9e9, 1.1e9, nchan) if nchan > 1 else np.array([1.0e9])
    R = 0.47 * a.npix * (C / freq.max()) / (a.fov * np.pi / 180)
    nrow = max(1, 20000 // nchan)
    uv = rng.standard_normal((nrow, 2)) * 0.3 * R
    uv[np.sum(uv * uv, 1) > R * R] *= 0.5
    uvw = np.concatenate([uv, rng.uniform(-1000, 1000, (nrow, 1))], 1)
    vis = rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))
    wgt = 1.0 - 0.5 * rng.random((nrow, nchan))
    per = max(2.0, min(a.cpu_seconds, 150.0 / max(1, a.steps + a.warmup)))
    for _ in range(a.warmup):
        cpu_baseline(uvw, freq, vis, wgt, a.npix, a.fov, per / 4)
    vals = [cpu_baseline(uvw, freq, vis, wgt, a.npix, a.fov, per) for _ in range(a.steps)]
    v = float(np.median([x["value"] for x in vals]))
    sample_ms = float(np.mean([x["sample_seconds"] for x in vals])) * 1e3
    cb = dict(vals[-1])
    cb["value"] = v
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "vis/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(sample_ms, 1),
           "extrapolated_ms_per_step": 1e3 * (a.nrow * a.nchan) / v,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded Gaussian uv density, uniform w, complex-normal vis)",
           "config": bench_config(a, world),
           "path": "explicit FP64 DFT on host cores (the reference's CPU path; C/OpenMP port)",
           "step": "one bounded sample of the workload, timed; value extrapolated to the full workload",
           "cpu_baseline": cb,
           "e2e": {"value": v, "unit": "vis/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
