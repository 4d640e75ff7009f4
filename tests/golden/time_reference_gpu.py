"""Time the reference library's own GPU path beside this library, same B200.

The reference's libcurafft.so is built for sm_100a from its own sources by
oracle/Makefile.ref into oracle/_ref/ (flag-only changes).  Its one-shot ABI
(ms2dirty_2 / dirty2ms_2, FP64, host buffers, one frequency per call,
src/astro/cugridder.cu:587-612) is called once per channel, as its Python
package does (python/curagridder/curagridder.py:92 passes freq[0]), and the
channel results are summed (ms2dirty) or stacked (dirty2ms).  The same calls go
through this library's reference ABI, then its multi-channel one-shot calls in
FP64 and FP32.  All runs read the same pinned host buffers, and every timed call
includes its own host<->device copies, as the ABI does.  The difference between
the two libraries' full-size outputs is reported as well.

Workload: the bench's (seeded Gaussian uv density, w uniform in +-1000 m,
complex-normal visibilities, weights in (0.5, 1]), 4096^2, fov 3 deg, eps 1e-5,
sigma 2, sign -1; the row count is an argument (default 1e7, 16 channels).
The grid there is 8192 x 8192 x 18: the reference's flat grid index
(src/fourier/conv.cu:213, int) stays below 2^31 while nf3 < 32.

    python tests/golden/time_reference_gpu.py [nrow] > gpurun_out/ref_gpu.json
"""
from __future__ import annotations

import ctypes
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def _bind(path):
    """The reference ABI of a libcurafft.so with plain pointer arguments."""
    lib = ctypes.CDLL(path)
    P, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    for name in ("ms2dirty_2", "dirty2ms_2"):
        f = getattr(lib, name)
        f.argtypes = [ci, ci, ci, cd, cd, P, P, P, P, cd, cd, ci]
        f.restype = ci
    return lib


def main():
    import torch
    import bench
    from curig_b200 import _lib

    nrow = int(sys.argv[1]) if len(sys.argv) > 1 else 10_000_000
    nchan, npix, fov, eps, sigma, sign = 16, 4096, 3.0, 1e-5, 2.0, -1
    dev = torch.device("cuda:0")
    freq, uvw_d, vis_d, wgt_d = bench.workload(torch, nrow, nchan, npix, fov, 0, dev)
    psx = fov * np.pi / 180 / npix

    def pinned(t):
        return t.contiguous().cpu().pin_memory()

    uvw = pinned(uvw_d)                                               # [nrow][3] f64
    vis_ch = [pinned(vis_d[:, c].to(torch.complex128)) for c in range(nchan)]   # per channel
    wgt_ch = [pinned(wgt_d[:, c].to(torch.float64)) for c in range(nchan)]
    fr = np.ascontiguousarray(freq, dtype=np.float64)
    img64 = torch.empty((npix, npix), dtype=torch.complex128).pin_memory()
    acc = np.zeros((npix, npix), dtype=np.complex128)
    out_ch = [torch.empty(nrow, dtype=torch.complex128).pin_memory() for _ in range(nchan)]
    ref = _bind(os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so"))
    mine_abi = _bind(_lib.lib._name)
    mine = _lib.lib

    def per_channel(lib, kind):
        """One step of reference-ABI calls, one per channel: ms2dirty summed over
        channels, or dirty2ms of the image per channel.  Returns the result and
        the summed wall time of the calls alone (the host-side sum / stack of
        the channel results is not timed)."""
        tc = 0.0
        if kind == 1:
            acc[:] = 0
            for c in range(nchan):
                t0 = time.perf_counter()
                st = lib.ms2dirty_2(nrow, npix, npix, fov, fr[c], uvw.data_ptr(), vis_ch[c].data_ptr(),
                                    wgt_ch[c].data_ptr(), img64.data_ptr(), eps, sigma, sign)
                tc += time.perf_counter() - t0
                assert st == 0, st
                acc[:] += img64.numpy()
            return acc.copy(), tc
        for c in range(nchan):
            t0 = time.perf_counter()
            st = lib.dirty2ms_2(nrow, npix, npix, fov, fr[c], uvw.data_ptr(), out_ch[c].data_ptr(),
                                wgt_ch[c].data_ptr(), img_in.data_ptr(), eps, sigma, sign)
            tc += time.perf_counter() - t0
            assert st == 0, st
        return np.stack([o.numpy() for o in out_ch], axis=1), tc

    def timed(fn, *a):
        fn(*a)                                       # warm-up step (allocator, cuFFT plans of every channel)
        torch.cuda.synchronize()
        return fn(*a)

    def timed_step(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    M = nrow * nchan
    res = {"workload": f"{nrow} rows x {nchan} ch ({M} vis), {npix}^2, fov {fov} deg, eps {eps}, sigma 2",
           "timing": "wall clock of the synchronous host-buffer calls alone (copies included), after one warm-up step"}
    # reference GPU, FP64, per channel
    d_ref, t = timed(per_channel, ref, 1)
    img_in = pinned(torch.from_numpy(d_ref / np.abs(d_ref).max()))
    v_ref, t2 = timed(per_channel, ref, 2)
    res["reference_gpu_fp64_per_channel"] = {"ms2dirty_s": t, "dirty2ms_s": t2, "vis_per_s": M / (t + t2)}
    # this library, the same reference-ABI calls
    d_my, t = timed(per_channel, mine_abi, 1)
    v_my, t2 = timed(per_channel, mine_abi, 2)
    res["curig_b200_fp64_per_channel"] = {"ms2dirty_s": t, "dirty2ms_s": t2, "vis_per_s": M / (t + t2)}
    res["l2_diff_vs_reference"] = {
        "ms2dirty": float(np.linalg.norm(d_my - d_ref) / np.linalg.norm(d_ref)),
        "dirty2ms": float(np.linalg.norm(v_my - v_ref) / np.linalg.norm(v_ref))}
    del vis_ch, wgt_ch, out_ch
    # this library, multi-channel one-shot calls (all channels in one transform)
    for prec, cdt, rdt in (("fp64", torch.complex128, torch.float64), ("fp32", torch.complex64, torch.float32)):
        v, w = pinned(vis_d.to(cdt)), pinned(wgt_d.to(rdt))          # [nrow][nchan]
        opts = _lib.make_opts(precision=1 if prec == "fp32" else 0)
        dimg = torch.empty((npix, npix), dtype=cdt).pin_memory()
        vout = torch.empty_like(v).pin_memory()
        din = pinned(img_in.to(cdt))

        def step():
            st = mine.curig_ms2dirty(nrow, nchan, npix, npix, psx, psx, fr.ctypes.data, uvw.data_ptr(),
                                     v.data_ptr(), w.data_ptr(), dimg.data_ptr(), eps, sigma, sign,
                                     ctypes.byref(opts))
            assert st == 0, st
            st = mine.curig_dirty2ms(nrow, nchan, npix, npix, psx, psx, fr.ctypes.data, uvw.data_ptr(),
                                     vout.data_ptr(), w.data_ptr(), din.data_ptr(), eps, sigma, sign,
                                     ctypes.byref(opts))
            assert st == 0, st

        t = timed_step(step)
        res[f"curig_b200_{prec}_multichannel"] = {"step_s": t, "vis_per_s": M / t}
        if prec == "fp64":
            res["l2_diff_vs_reference"]["ms2dirty_multichannel"] = float(
                np.linalg.norm(dimg.numpy() - d_ref) / np.linalg.norm(d_ref))
            res["l2_diff_vs_reference"]["dirty2ms_multichannel"] = float(
                np.linalg.norm(vout.numpy() - v_ref) / np.linalg.norm(v_ref))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
