"""The allocation-free entry point (curig_window_loss_grad_static) against the
allocating one (curig_window_loss_grad), through the C ABI, on two calls in a
row.  It serves callers that cannot allocate device memory where they need the
window objective (memory reserved by another framework's pool, or pipelines
that forbid allocation after initialisation).  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static(lib, W, p):
    loss = np.zeros(1)
    grad = np.zeros(p.size, dtype=np.float32)
    st = lib.curig_window_loss_grad_static(W, 2.0, p.ctypes.data, loss.ctypes.data, grad.ctypes.data)
    return st, float(loss[0]), grad


def test_static_scratch_entry_matches_allocating_entry():
    from curig_b200 import _lib, learned
    lib = _lib.lib
    for call, (W, seed) in enumerate([(6, 1), (4, 2)]):        # two calls in a row, different inputs
        p = learned.init_params(seed)
        p[-33:] = np.random.default_rng(seed).normal(0, 0.02, 33).astype(np.float32)
        L_ref, g_ref = learned.loss_and_grad(W, p)
        st, L, g = _static(lib, W, p)
        assert st == 0, (call, lib.curig_last_error())
        assert abs(L - L_ref) <= 1e-8 * L_ref
        assert np.linalg.norm(g - g_ref) <= 1e-5 * np.linalg.norm(g_ref)


def _pool_reserved():
    """Bytes the device's default stream-ordered pool holds (cudaMallocAsync's source)."""
    import torch
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent)
    assert err == rt.cudaError_t.cudaSuccess
    return int(v)


def test_static_scratch_entry_allocates_no_device_memory():
    """After one warm-up call (which loads the module and its static array),
    repeated calls change neither the device's free memory (a cudaMalloc takes
    at least a 2 MiB page) nor the default pool's reservation (cudaMallocAsync)."""
    import torch
    from curig_b200 import _lib, learned
    lib = _lib.lib
    p = learned.init_params(3)
    assert _static(lib, 6, p)[0] == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    pool0 = _pool_reserved()
    for W in (6, 5, 8):
        assert _static(lib, W, p)[0] == 0, lib.curig_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert _pool_reserved() == pool0
    assert free1 >= free0 - (1 << 20), (free0, free1)


def test_static_scratch_entry_rejects_oversize():
    from curig_b200 import _lib, learned
    p = learned.init_params(0)
    st, _, _ = _static(_lib.lib, 13, p)
    assert st == 3
