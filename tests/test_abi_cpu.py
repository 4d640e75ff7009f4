"""CPU tests of the C ABI: the library loads, exports every function the
public headers declare, its host-side sizing rules agree bit-for-bit with the
oracle's restatement of the reference, and argument errors come back as
status codes (no GPU is touched)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import params as P


def _declared_functions():
    names = set()
    for h in ("curig.h",):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", src, flags=re.M):
            if m.group(1) not in ("if", "sizeof"):
                names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_header_symbols():
    import curig_b200._lib as L
    names = _declared_functions()
    assert {"ms2dirty_1", "ms2dirty_2", "dirty2ms_1", "dirty2ms_2"} <= set(names)
    missing = [n for n in names if not hasattr(L.lib, n)]
    assert not missing, missing


def test_cpp_plan_api_exported():
    import subprocess
    out = subprocess.run(["nm", "-DC", "--defined-only", os.path.join(ROOT, "curig_b200", "libcurafft.so")],
                         capture_output=True, text=True).stdout
    for fn in ("gridder_setting(", "gridder_execution(", "gridder_destroy("):
        assert fn in out


@pytest.mark.parametrize("nx,ny,fov,wmax,eps,sigma", [
    (256, 256, 2.0, 4190.0, 1e-6, 2.0), (4096, 4096, 3.0, 23000.0, 1e-5, 2.0),
    (30, 128, 10.0, 3.1, 5e-7, 2.0), (16, 64, 20.0, 3.1, 5e-12, 2.0), (128, 250, 1.0, 3.1, 2e-1, 2.0),
    (512, 512, 60.0, 100.0, 1e-12, 2.0), (64, 48, 5.0, 50.0, 1e-6, 1.25), (100, 100, 2.0, 0.0, 1e-4, 2.0)])
def test_native_grid_params_match_oracle(nx, ny, fov, wmax, eps, sigma):
    import curig_b200._lib as L
    psx, psy = P.pixel_sizes(fov, nx, ny)
    wmin = -0.7 * wmax
    io = (ctypes.c_int * 4)()
    do = (ctypes.c_double * 6)()
    assert L.lib.curig_grid_params(nx, ny, psx, psy, wmin, wmax, eps, sigma, io, do) == 0
    ref = P.gridder_params(nx, ny, None, None, None, eps, sigma, 1, psx, psy, w_range=(wmin, wmax))
    assert list(io) == [ref.nf1, ref.nf2, ref.nf3, ref.opts.kw]
    assert list(do) == [ref.opts.beta, ref.gamma, ref.h, ref.i_center, ref.i_half, ref.o_center]


@pytest.mark.parametrize("nf,eps", [(512, 1e-6), (60, 5e-12), (8192, 1e-5), (128, 2e-1)])
def test_native_psi_hat_matches_oracle(nf, eps):
    import curig_b200._lib as L
    out = (ctypes.c_double * (nf // 2 + 1))()
    assert L.lib.curig_psi_hat(nf, eps, 2.0, out) == 0
    opts = P.setup_conv_opts(eps, 2.0)
    ref = P.psi_hat_grid(nf, opts) * np.exp(-opts.beta)
    got = np.array(out[:])
    assert np.max(np.abs(got - ref) / np.abs(ref)) < 1e-10


def test_argument_errors_return_codes():
    import curig_b200._lib as L
    lib = L.lib
    assert lib.curig_ms2dirty(10, 1, 16, 16, 1e-3, 1e-3, None, None, None, None, None, 1e-6, 2.0, 1, None) == 3
    assert lib.curig_ms2dirty(-1, 1, 16, 16, 1e-3, 1e-3, None, None, None, None, None, 1e-6, 2.0, 1, None) == 3
    io = (ctypes.c_int * 4)()
    assert lib.curig_grid_params(16, 16, 1e-3, 1e-3, -1.0, 1.0, 1e-6, 0.9, io, None) == 2   # sigma <= 1
    assert lib.curig_grid_params(16, 16, 1e-3, 1e-3, float("nan"), 1.0, 1e-6, 2.0, io, None) == 7
    assert lib.curig_grid_params(16, 16, 0.2, 0.2, -1.0, 1.0, 1e-6, 2.0, io, None) == 3     # beyond horizon
    h = ctypes.c_void_p()
    assert lib.curig_makeplan(3, 16, 16, 1e-3, 1e-3, 1e-6, 2.0, 1, None, ctypes.byref(h)) == 3
    coef = np.zeros(5 * 4)
    assert lib.curig_set_window(1, 3, coef.ctypes.data, 1e-5) == 3


def test_empty_visibility_set_gives_zero_image():
    import curig_b200._lib as L
    dirty = np.ones((8, 8), dtype=np.complex128)
    freq = np.array([1e9])
    st = L.lib.curig_ms2dirty(0, 1, 8, 8, 1e-3, 1e-3, freq.ctypes.data, None, None, None,
                              dirty.ctypes.data, 1e-6, 2.0, 1, None)
    assert st == 0 and not dirty.any()


def test_reference_binding_rejects_wrong_dtypes():
    import curig_b200 as C
    uvw = np.zeros((4, 3), dtype=np.float32)
    ms = np.zeros((4, 1), dtype=np.complex128)
    with pytest.raises(ctypes.ArgumentError):
        C.ms2dirty(uvw, np.array([1e9]), ms, None, 8, 8, 1e-3, 1e-3, 0, 0, 1e-6, True)
