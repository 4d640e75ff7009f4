"""Autograd pair (ms2dirty <-> dirty2ms adjoints, gradients w.r.t. visibilities
and weights) and the batch of independent problems.

CPU: the vector-Jacobian products of the autograd Functions checked by
torch.autograd.gradcheck against a dense stand-in operator (same weighting
convention as the library).  GPU: finite differences (FP64, step 1e-3) of a
least-squares loss through the CUDA path, adjointness, and a batch of 8."""
import numpy as np
import pytest
import torch

from conftest import disk_inputs


class DenseOp:
    """A (nx*ny x M) complex matrix with the library's weighting: apply =
    A (wgt * vis), adjoint = wgt * A^H dirty."""

    def __init__(self, nrow, nchan, nx, ny, seed=0):
        g = torch.Generator().manual_seed(seed)
        self.A = torch.complex(torch.randn(nx * ny, nrow * nchan, generator=g, dtype=torch.float64),
                               torch.randn(nx * ny, nrow * nchan, generator=g, dtype=torch.float64))
        self.nrow, self.nchan, self.nx, self.ny = nrow, nchan, nx, ny

    def apply(self, vis, wgt=None):
        u = vis if wgt is None else vis * wgt
        return (self.A @ u.reshape(-1)).reshape(self.nx, self.ny)

    def adjoint(self, dirty, wgt=None):
        v = (self.A.conj().T @ dirty.reshape(-1)).reshape(self.nrow, self.nchan)
        return v if wgt is None else v * wgt


def test_vjp_formulas_gradcheck():
    from curig_b200.autograd import _Dirty2MS, _MS2Dirty
    op = DenseOp(5, 2, 3, 4)
    g = torch.Generator().manual_seed(1)
    vis = torch.complex(torch.randn(5, 2, generator=g, dtype=torch.float64),
                        torch.randn(5, 2, generator=g, dtype=torch.float64)).requires_grad_()
    wgt = (torch.rand(5, 2, generator=g, dtype=torch.float64) + 0.5).requires_grad_()
    dirty = torch.complex(torch.randn(3, 4, generator=g, dtype=torch.float64),
                          torch.randn(3, 4, generator=g, dtype=torch.float64)).requires_grad_()
    assert torch.autograd.gradcheck(lambda v, w: _MS2Dirty.apply(v, w, op), (vis, wgt))
    assert torch.autograd.gradcheck(lambda d, w: _Dirty2MS.apply(d, w, op), (dirty, wgt))
    assert torch.autograd.gradcheck(lambda v: _MS2Dirty.apply(v, None, op), (vis,))
    assert torch.autograd.gradcheck(lambda d: _Dirty2MS.apply(d, None, op), (dirty,))


# ------------------------------------------------------------------ GPU
def _operator(nrow, nchan, npix, precision, eps, seed=0, fov=2.0):
    from curig_b200.autograd import GridderOperator
    freq, uvw, ms, wgt = disk_inputs(nrow, nchan, npix, fov, max_pix=0.45 * npix, seed=seed)
    psx = fov * np.pi / 180 / npix
    op = GridderOperator(torch.from_numpy(uvw).cuda(), freq, npix, npix, psx, psx, eps, precision=precision)
    cdt = torch.complex64 if precision == "fp32" else torch.complex128
    rdt = torch.float32 if precision == "fp32" else torch.float64
    return op, torch.from_numpy(ms).to(cdt).cuda(), torch.from_numpy(wgt).to(rdt).cuda()


def _rand_like(t, seed):
    g = torch.Generator(device=t.device).manual_seed(seed)
    if t.is_complex():
        r = torch.float64 if t.dtype == torch.complex128 else torch.float32
        return torch.complex(torch.randn(t.shape, generator=g, device=t.device, dtype=r),
                             torch.randn(t.shape, generator=g, device=t.device, dtype=r))
    return torch.randn(t.shape, generator=g, device=t.device, dtype=t.dtype)


@pytest.mark.gpu
def test_ms2dirty_gradients_match_finite_differences():
    op, vis, wgt = _operator(300, 2, 48, "fp64", 1e-10)
    d = _rand_like(torch.empty((48, 48), dtype=torch.complex128, device="cuda"), 3)

    def loss(v, w):
        return ((op.ms2dirty(v, w) - d).abs() ** 2).sum()

    v = vis.clone().requires_grad_()
    w = wgt.clone().requires_grad_()
    loss(v, w).backward()
    dv, dw, h = _rand_like(vis, 4), _rand_like(wgt, 5), 1e-3
    with torch.no_grad():
        fd_v = (loss(vis + h * dv, wgt) - loss(vis - h * dv, wgt)) / (2 * h)
        fd_w = (loss(vis, wgt + h * dw) - loss(vis, wgt - h * dw)) / (2 * h)
    an_v = (v.grad.conj() * dv).real.sum()
    an_w = (w.grad * dw).sum()
    assert abs(float(fd_v - an_v)) <= 1e-7 * abs(float(an_v))
    assert abs(float(fd_w - an_w)) <= 1e-7 * abs(float(an_w))
    op.close()


@pytest.mark.gpu
def test_dirty2ms_gradients_match_finite_differences():
    op, vis, wgt = _operator(300, 2, 48, "fp64", 1e-10, seed=1)
    dirty = _rand_like(torch.empty((48, 48), dtype=torch.complex128, device="cuda"), 6)
    target = _rand_like(vis, 7)

    def loss(x, w):
        return ((op.dirty2ms(x, w) - target).abs() ** 2).sum()

    x = dirty.clone().requires_grad_()
    w = wgt.clone().requires_grad_()
    loss(x, w).backward()
    dx, dw, h = _rand_like(dirty, 8), _rand_like(wgt, 9), 1e-3
    with torch.no_grad():
        fd_x = (loss(dirty + h * dx, wgt) - loss(dirty - h * dx, wgt)) / (2 * h)
        fd_w = (loss(dirty, wgt + h * dw) - loss(dirty, wgt - h * dw)) / (2 * h)
    assert abs(float(fd_x - (x.grad.conj() * dx).real.sum())) <= 1e-7 * abs(float(fd_x))
    assert abs(float(fd_w - (w.grad * dw).sum())) <= 1e-7 * abs(float(fd_w))
    op.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_operator_adjointness(precision, tol):
    """<A_w x, y> = <x, A_w^H y> through the differentiable entry points."""
    op, vis, wgt = _operator(2000, 3, 64, precision, 1e-10 if precision == "fp64" else 1e-5, seed=2)
    y = _rand_like(torch.empty((64, 64), dtype=vis.dtype, device="cuda"), 10)
    with torch.no_grad():
        lhs = torch.vdot(op.ms2dirty(vis, wgt).reshape(-1), y.reshape(-1))
        rhs = torch.vdot(vis.reshape(-1), op.dirty2ms(y, wgt).reshape(-1))
    assert abs(complex(lhs - rhs)) <= tol * abs(complex(lhs))
    op.close()


@pytest.mark.gpu
def test_gradient_is_one_adjoint_call():
    """grad_vis of ||A_w v - d||^2 equals 2 A_w^H (A_w v - d) from the plan."""
    op, vis, wgt = _operator(500, 2, 32, "fp64", 1e-10, seed=3)
    d = _rand_like(torch.empty((32, 32), dtype=torch.complex128, device="cuda"), 11)
    v = vis.clone().requires_grad_()
    ((op.ms2dirty(v, wgt) - d).abs() ** 2).sum().backward()
    with torch.no_grad():
        ref = 2 * op.adjoint(op.apply(vis, wgt) - d, wgt)
    assert torch.allclose(v.grad, ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max()))
    op.close()


@pytest.mark.gpu
def test_batch_of_8_matches_individual_problems():
    """8 independent problems (own uvw, shared geometry): the batched loss's
    gradients equal the per-problem ones (FP32 and FP64), and a finite-difference
    check of the whole batch in FP64."""
    from curig_b200.autograd import BatchGridder
    B, nrow, npix = 8, 3000, 96
    psx = 2.0 * np.pi / 180 / npix
    for precision in ("fp32", "fp64"):
        data = [disk_inputs(nrow, 1, npix, 2.0, max_pix=0.45 * npix, seed=20 + b) for b in range(B)]
        cdt = torch.complex64 if precision == "fp32" else torch.complex128
        rdt = torch.float32 if precision == "fp32" else torch.float64
        uvws = [torch.from_numpy(x[1]).cuda() for x in data]
        vis = torch.stack([torch.from_numpy(x[2]).to(cdt) for x in data]).cuda()
        wgt = torch.stack([torch.from_numpy(x[3]).to(rdt) for x in data]).cuda()
        eps = 1e-5 if precision == "fp32" else 1e-10
        bg = BatchGridder(uvws, data[0][0], npix, npix, psx, psx, eps, precision=precision)
        d = _rand_like(torch.empty((B, npix, npix), dtype=cdt, device="cuda"), 12)

        def loss(v, w):
            return ((bg.ms2dirty(v, w) - d).abs() ** 2).sum()

        v = vis.clone().requires_grad_()
        w = wgt.clone().requires_grad_()
        loss(v, w).backward()
        for b in range(B):
            vb = vis[b].clone().requires_grad_()
            wb = wgt[b].clone().requires_grad_()
            ((bg.ops[b].ms2dirty(vb, wb) - d[b]).abs() ** 2).sum().backward()
            # tiles flush into the grid with float atomics: equal up to summation order
            tol = 1e-5 if precision == "fp32" else 1e-12
            assert float((vb.grad - v.grad[b]).abs().max()) <= tol * float(vb.grad.abs().max())
            assert float((wb.grad - w.grad[b]).abs().max()) <= tol * float(wb.grad.abs().max())
        if precision == "fp64":
            dv, dw, h = _rand_like(vis, 13), _rand_like(wgt, 14), 1e-3
            with torch.no_grad():
                fd_v = (loss(vis + h * dv, wgt) - loss(vis - h * dv, wgt)) / (2 * h)
                fd_w = (loss(vis, wgt + h * dw) - loss(vis, wgt - h * dw)) / (2 * h)
            assert abs(float(fd_v - (v.grad.conj() * dv).real.sum())) <= 1e-7 * abs(float(fd_v))
            assert abs(float(fd_w - (w.grad * dw).sum())) <= 1e-7 * abs(float(fd_w))
        bg.close()
