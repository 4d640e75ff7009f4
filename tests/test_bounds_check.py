"""Memory safety of the GPU kernels, checked by the bounds-checked build.

compute-sanitizer is not available everywhere, so the library has a second
build, curig_b200/libcurafft_check.so (curig_b200/csrc/build.py --check,
-DCURIG_BOUNDS_CHECK), in which the binning, spreading, interpolation and
correction kernels check every buffer index they compute (tile words, grid
cells, sorted positions, input indices, transposed-image offsets); an index
outside its buffer raises an error flag instead of being used, and the call
returns status 1 ("an index left its buffer").  A worker process loads that
build (CURIG_LIB) and runs the one-shot calls over the code paths: FP32 with
one-word, exact two-word and float tiles, tiles only and sparse chunks only,
row slabs, the w-free mode with an explicit grid, narrow and wide windows,
the learned window, FP64 through the reference ABI and multi-channel with
double atomics.  Every call must return 0, and the results must equal those
of the regular build run here."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CHECK_LIB = os.path.join(ROOT, "curig_b200", "libcurafft_check.so")

# name: precision (1 FP32, 0 FP64), channels, epsilon, window (0 ES, 1 learned), accumulate,
# sparse threshold, slabs, w_term, explicit grid, reference ABI
CASES = {
    "f32_one_word_learned": dict(prec=1, nchan=16, eps=1e-5, window=1),
    "f32_two_word": dict(prec=1, nchan=16, eps=1e-6, accumulate=3),
    "f32_float_atomics": dict(prec=1, nchan=16, eps=1e-5, accumulate=1),
    "f32_tiles_only": dict(prec=1, nchan=16, eps=1e-5, sparse=-1),
    "f32_sparse_only": dict(prec=1, nchan=16, eps=1e-5, sparse=1 << 30),
    "f32_slabs3": dict(prec=1, nchan=16, eps=1e-5, slabs=3),
    "f32_wfree_grid": dict(prec=1, nchan=4, eps=1e-5, w_term=1, grid=600),
    "f32_narrow": dict(prec=1, nchan=4, eps=2e-2),
    "f64_multichannel": dict(prec=0, nchan=8, eps=1e-9),
    "f64_double_atomics": dict(prec=0, nchan=8, eps=1e-7, accumulate=1),
    "f64_wide": dict(prec=0, nchan=2, eps=1e-13),
    "f64_reference_abi": dict(prec=0, nchan=1, eps=1e-6, abi=True),
}
NROW, N, FOV = 20000, 256, 2.0


def run_cases(L):
    """Every case's ms2dirty image and dirty2ms visibilities, and the calls'
    statuses, through the library that L has loaded."""
    sys.path.insert(0, HERE)
    from conftest import disk_inputs
    psx = FOV * np.pi / 180 / N
    out = {}
    for name, c in CASES.items():
        prec, nchan = c["prec"], c["nchan"]
        freq, uvw, ms, wgt = disk_inputs(NROW, nchan, N, FOV, f0=0.9e9, fmax=1.1e9, max_pix=110.0, wmax=300.0,
                                         seed=11)
        uvw = np.ascontiguousarray(uvw)
        ct, rt = (np.complex64, np.float32) if prec else (np.complex128, np.float64)
        vis = np.ascontiguousarray(ms.astype(ct))
        w = np.ascontiguousarray(wgt.astype(rt))
        img = (np.random.default_rng(12).standard_normal((N, N)) + 0j).astype(ct)
        dirty = np.zeros((N, N), dtype=ct)
        vout = np.zeros_like(vis)
        if c.get("abi"):
            s1 = L.ms2dirty_2(NROW, N, N, FOV, freq[0], uvw, vis[:, 0].copy(), w[:, 0].copy(), dirty,
                              c["eps"], 2.0, -1)
            v1 = np.zeros(NROW, dtype=np.complex128)
            s2 = L.dirty2ms_2(NROW, N, N, FOV, freq[0], uvw, v1, w[:, 0].copy(), img, c["eps"], 2.0, -1)
            vout[:, 0] = v1
        else:
            g = c.get("grid", 0)
            o = L.make_opts(precision=prec, window=c.get("window", 0), accumulate=c.get("accumulate", 0),
                            sparse=c.get("sparse", 0), slabs=c.get("slabs", 0), w_term=c.get("w_term", 0),
                            grid_x=g, grid_y=g)
            fr = np.ascontiguousarray(freq, dtype=np.float64)
            s1 = L.lib.curig_ms2dirty(NROW, nchan, N, N, psx, psx, fr.ctypes.data, uvw.ctypes.data,
                                      vis.ctypes.data, w.ctypes.data, dirty.ctypes.data, c["eps"], 2.0, -1,
                                      ctypes.byref(o))
            s2 = L.lib.curig_dirty2ms(NROW, nchan, N, N, psx, psx, fr.ctypes.data, uvw.ctypes.data,
                                      vout.ctypes.data, w.ctypes.data, img.ctypes.data, c["eps"], 2.0, -1,
                                      ctypes.byref(o))
        out[name + "__status"] = np.array([s1, s2])
        out[name + "__dirty"] = dirty
        out[name + "__vis"] = vout
    return out


def _worker(path):
    sys.path[:0] = [ROOT, HERE]
    import curig_b200._lib as L
    import curig_b200.learned as learned
    assert os.path.samefile(L.LIB_PATH, CHECK_LIB), L.LIB_PATH
    learned.load_default_windows()
    res = run_cases(L)
    errs = {k: L.lib.curig_last_error().decode() for k in res if k.endswith("__status") and np.any(res[k])}
    if errs:
        print("failed calls:", errs, file=sys.stderr)
    np.savez(path, **res)


@pytest.mark.gpu
def test_bounds_checked_build_flags_nothing_and_agrees(tmp_path):
    assert os.path.exists(CHECK_LIB), "build it with: python curig_b200/csrc/build.py --check"
    path = str(tmp_path / "checked.npz")
    env = dict(os.environ, CURIG_LIB=CHECK_LIB)
    r = subprocess.run([sys.executable, os.path.abspath(__file__), path], env=env, capture_output=True,
                       text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-4000:]
    chk = dict(np.load(path))
    import curig_b200._lib as L
    import curig_b200.learned as learned
    learned.load_default_windows()
    ref = run_cases(L)
    for name in CASES:
        assert list(chk[name + "__status"]) == [0, 0], (name, chk[name + "__status"], r.stderr[-2000:])
        assert list(ref[name + "__status"]) == [0, 0], (name, ref[name + "__status"])
        tol = 1e-12 if CASES[name]["prec"] == 0 else 1e-5
        for part in ("__dirty", "__vis"):
            a, b = chk[name + part], ref[name + part]
            rel = np.linalg.norm(a - b) / np.linalg.norm(b)
            assert rel < tol, (name + part, rel)


if __name__ == "__main__":
    _worker(sys.argv[1])
