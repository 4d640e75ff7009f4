"""The C++ plan API (gridder_setting -> plan->fk -> gridder_execution ->
gridder_destroy, include/cugridder.h) driven by a C++ caller written like the
reference's test mains (test/w_s_gridder_test.cu:105-222,274,
test/w_s_degridder_test.cu:195-229): both directions, with and without
kv.weight, against the FP64 DFT oracle.  The driver is compiled here with g++
against include/cugridder.h and libcurafft.so."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, disk_inputs, l2err
from oracle import dft

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIBDIR = os.path.join(ROOT, "curig_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "plan_api_driver.cpp")


def _compile(out_dir):
    exe = os.path.join(out_dir, "plan_api_driver")
    cmd = ["g++", "-O2", "-std=c++17", SRC, "-o", exe, "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(CUDA_HOME, "include"), LIBDIR + "/libcurafft.so",
           "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-Wl,-rpath," + LIBDIR,
           "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_plan_api_driver_compiles(tmp_path):
    """Source compatibility: a C++ caller of the reference's structs builds and links."""
    assert os.path.exists(_compile(str(tmp_path)))


@pytest.mark.gpu
@pytest.mark.parametrize("nrow,n,fov,eps", [(3000, 128, 2.0, 1e-6), (500, 96, 5.0, 1e-9)])
def test_plan_api_both_directions_against_dft(tmp_path, nrow, n, fov, eps):
    freq, uvw, ms, wgt = disk_inputs(nrow, 1, n, fov, max_pix=0.45 * n, seed=nrow)
    nx, ny = n, n + 16
    rng = np.random.default_rng(9)
    dirty = rng.standard_normal((nx, ny)) + 1j * rng.standard_normal((nx, ny))
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([nrow, nx, ny], dtype=np.int32).tofile(f)
        np.array([fov, freq[0], eps, 2.0]).tofile(f)
        for a in (uvw[:, 0], uvw[:, 1], uvw[:, 2]):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        np.ascontiguousarray(ms[:, 0], dtype=np.complex128).tofile(f)
        np.ascontiguousarray(wgt[:, 0], dtype=np.float64).tofile(f)
        np.ascontiguousarray(dirty, dtype=np.complex128).tofile(f)
    exe = _compile(str(tmp_path))
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr)
    res = np.fromfile(out, dtype=np.complex128)
    npix = nx * ny
    d_w, d_nw = res[:npix].reshape(nx, ny), res[npix:2 * npix].reshape(nx, ny)
    v_w, v_nw = res[2 * npix:2 * npix + nrow], res[2 * npix + nrow:]
    xps, yps = fov * np.pi / 180 / nx, fov * np.pi / 180 / ny
    # direction 1 (vis -> image): sign -1 as in the reference's test main
    assert l2err(dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, xps, yps, -1), d_w) < 10 * eps
    assert l2err(dft.ms2dirty_dft(uvw, freq, ms, None, nx, ny, xps, yps, -1), d_nw) < 10 * eps
    # direction 0 (image -> vis)
    assert l2err(dft.dirty2ms_dft(uvw, freq, dirty, wgt, xps, yps, -1)[:, 0], v_w) < 10 * eps
    assert l2err(dft.dirty2ms_dft(uvw, freq, dirty, None, xps, yps, -1)[:, 0], v_nw) < 10 * eps
