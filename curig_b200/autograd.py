"""Differentiable ms2dirty / dirty2ms (torch.autograd) and a batch of
independent problems.

ms2dirty is linear in the weighted visibilities: dirty = A (wgt * vis), with A
the w-stacking NUFFT of the plan (1/n(l,m) included), and dirty2ms applies the
weights too, vis = wgt * A^H dirty (ra_exec.cu:56-104 and utils.cu:189 of the
reference: the weight multiplies in both directions), so dirty2ms is the exact
adjoint of ms2dirty.  With torch's conjugate-Wirtinger convention the
vector-Jacobian products are:

    ms2dirty:  grad_vis   = wgt * A^H g               (= dirty2ms(g, wgt))
               grad_wgt   = Re(conj(vis) * A^H g)
    dirty2ms:  grad_dirty = A (wgt * g)               (= ms2dirty(g, wgt))
               grad_wgt   = Re(g * conj(A^H dirty))

Every product runs through the plan's CUDA kernels; nothing here computes on
the host.  The reference has no autograd layer.
"""
from __future__ import annotations

import numpy as np
import torch

from .plan import GridderPlan


class GridderOperator:
    """ms2dirty / dirty2ms on fixed points (uvw on the device, set once).

    uvw: CUDA float64 [nrow, 3]; freq: host array [nchan]; the other arguments
    are those of GridderPlan.  Visibilities are [nrow, nchan], the dirty image
    [nxdirty, nydirty], both complex (complex64 for precision="fp32")."""

    def __init__(self, uvw, freq, nxdirty, nydirty, pixsize_x, pixsize_y, epsilon, sigma=2.0, sign=-1,
                 precision="fp32", window="es", accumulate=0, stream=None):
        self.nx, self.ny = int(nxdirty), int(nydirty)
        self.cdt = torch.complex64 if precision == "fp32" else torch.complex128
        self.rdt = torch.float32 if precision == "fp32" else torch.float64
        self.device = uvw.device
        # the plan's stream: given, or the caller's current stream
        self.stream = stream if stream is not None else torch.cuda.current_stream(uvw.device)
        self.plan = GridderPlan(1, nxdirty, nydirty, pixsize_x, pixsize_y, epsilon, sigma, sign,
                                precision=precision, window=window, stream=self.stream, accumulate=accumulate)
        with self._ordered():
            self.plan.setpts(uvw, np.atleast_1d(np.asarray(freq, dtype=np.float64)))
        self.nrow, self.nchan = self.plan.nrow, self.plan.nchan

    class _Order:
        """Orders the plan's stream after the caller's current stream on entry
        and the caller's after the plan's on exit (no-op when they are one)."""

        def __init__(self, op):
            self.op = op

        def __enter__(self):
            self.cur = torch.cuda.current_stream(self.op.device)
            if self.cur != self.op.stream:
                self.op.stream.wait_stream(self.cur)

        def __exit__(self, *exc):
            if self.cur != self.op.stream:
                self.cur.wait_stream(self.op.stream)
            return False

    def _ordered(self):
        return GridderOperator._Order(self)

    # raw products (no autograd) --------------------------------------------------
    def _check(self, t, dtype, shape, what):
        if t.dtype != dtype or t.device != self.device or tuple(t.shape) != shape:
            raise TypeError(f"{what} must be {dtype} {shape} on {self.device}, got {t.dtype} "
                            f"{tuple(t.shape)} on {t.device}")
        return t.contiguous()

    def apply(self, vis, wgt=None):
        """A (wgt * vis) -> dirty [nx, ny]."""
        vis = self._check(vis, self.cdt, (self.nrow, self.nchan), "vis")
        if wgt is not None:
            wgt = self._check(wgt, self.rdt, (self.nrow, self.nchan), "wgt")
        out = torch.empty((self.nx, self.ny), dtype=self.cdt, device=self.device)
        with self._ordered():
            self.plan.execute_dir(1, vis, wgt, out)
        return out

    def adjoint(self, dirty, wgt=None):
        """wgt * A^H dirty -> vis [nrow, nchan]."""
        dirty = self._check(dirty, self.cdt, (self.nx, self.ny), "dirty")
        if wgt is not None:
            wgt = self._check(wgt, self.rdt, (self.nrow, self.nchan), "wgt")
        out = torch.empty((self.nrow, self.nchan), dtype=self.cdt, device=self.device)
        with self._ordered():
            self.plan.execute_dir(2, out, wgt, dirty)
        return out

    # differentiable products -----------------------------------------------------
    def ms2dirty(self, vis, wgt=None):
        return _MS2Dirty.apply(vis, wgt, self)

    def dirty2ms(self, dirty, wgt=None):
        return _Dirty2MS.apply(dirty, wgt, self)

    def close(self):
        self.plan.close()


class _MS2Dirty(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vis, wgt, op):
        ctx.op = op
        ctx.save_for_backward(vis, wgt)
        return op.apply(vis.detach(), None if wgt is None else wgt.detach())

    @staticmethod
    def backward(ctx, g):
        vis, wgt = ctx.saved_tensors
        op = ctx.op
        need_v, need_w = ctx.needs_input_grad[0], ctx.needs_input_grad[1] and wgt is not None
        gv = gw = None
        if need_w:
            t = op.adjoint(g.contiguous(), None)                 # A^H g
            gw = (vis.detach().conj() * t).real.to(wgt.dtype)
            if need_v:
                gv = t * wgt.detach()
        elif need_v:
            gv = op.adjoint(g.contiguous(), None if wgt is None else wgt.detach())
        return gv, gw, None


class _Dirty2MS(torch.autograd.Function):
    @staticmethod
    def forward(ctx, dirty, wgt, op):
        ctx.op = op
        if wgt is not None and wgt.requires_grad:
            t = op.adjoint(dirty.detach(), None)                 # A^H dirty
            ctx.save_for_backward(wgt, t)
            return t * wgt.detach()
        ctx.save_for_backward(wgt, None)
        return op.adjoint(dirty.detach(), None if wgt is None else wgt.detach())

    @staticmethod
    def backward(ctx, g):
        wgt, t = ctx.saved_tensors
        op = ctx.op
        gd = gw = None
        if ctx.needs_input_grad[0]:
            gd = op.apply(g.contiguous(), None if wgt is None else wgt.detach())
        if ctx.needs_input_grad[1] and wgt is not None:
            gw = (g * t.conj()).real.to(wgt.dtype)
        return gd, gw, None


class BatchGridder:
    """Independent problems, one plan each (own points, same image geometry).
    Inputs are stacked: vis / wgt [B, nrow, nchan], dirty [B, nx, ny]; problems
    share nrow and nchan.  Each problem runs on its own CUDA stream, launched
    one after another and joined to the caller's stream at the end (forward and
    backward), so the small transforms of the batch overlap on the GPU."""

    def __init__(self, uvws, freq, nxdirty, nydirty, pixsize_x, pixsize_y, epsilon, **kw):
        cur = torch.cuda.current_stream()
        self.streams = [torch.cuda.Stream() for _ in uvws]
        self.ops = []
        for u, st in zip(uvws, self.streams):
            st.wait_stream(cur)                          # uvw written on the caller's stream
            with torch.cuda.stream(st):
                self.ops.append(GridderOperator(u, freq, nxdirty, nydirty, pixsize_x, pixsize_y, epsilon,
                                                stream=st, **kw))
        for st in self.streams:
            cur.wait_stream(st)

    def __len__(self):
        return len(self.ops)

    def ms2dirty(self, vis, wgt=None):
        return _BatchMS2Dirty.apply(vis, wgt, self)

    def dirty2ms(self, dirty, wgt=None):
        return _BatchDirty2MS.apply(dirty, wgt, self)

    def _each(self, fn):
        """fn(b, op) for every problem on its stream; then join to the caller's stream."""
        cur = torch.cuda.current_stream()
        for b, (op, st) in enumerate(zip(self.ops, self.streams)):
            st.wait_stream(cur)
            with torch.cuda.stream(st):
                fn(b, op)
        for st in self.streams:
            cur.wait_stream(st)

    def close(self):
        for op in self.ops:
            op.close()


class _BatchMS2Dirty(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vis, wgt, bg):
        ctx.bg = bg
        ctx.save_for_backward(vis, wgt)
        op0 = bg.ops[0]
        out = torch.empty((len(bg), op0.nx, op0.ny), dtype=op0.cdt, device=vis.device)
        vis_d = vis.detach()
        wgt_d = None if wgt is None else wgt.detach()

        def run(b, op):
            op.plan.execute_dir(1, op._check(vis_d[b], op.cdt, (op.nrow, op.nchan), "vis"),
                                None if wgt_d is None else op._check(wgt_d[b], op.rdt, (op.nrow, op.nchan), "wgt"),
                                out[b])
        bg._each(run)
        return out

    @staticmethod
    def backward(ctx, g):
        vis, wgt = ctx.saved_tensors
        bg = ctx.bg
        g = g.contiguous()
        need_v, need_w = ctx.needs_input_grad[0], ctx.needs_input_grad[1] and wgt is not None
        gv = torch.empty_like(vis) if need_v else None
        gw = torch.empty_like(wgt) if need_w else None
        vis_d = vis.detach()
        wgt_d = None if wgt is None else wgt.detach()

        def run(b, op):
            if need_w:
                t = op.adjoint(g[b], None)                    # A^H g
                gw[b].copy_((vis_d[b].conj() * t).real)
                if need_v:
                    gv[b].copy_(t * wgt_d[b])
            elif need_v:
                gv[b].copy_(op.adjoint(g[b], None if wgt_d is None else wgt_d[b]))
        bg._each(run)
        return gv, gw, None


class _BatchDirty2MS(torch.autograd.Function):
    @staticmethod
    def forward(ctx, dirty, wgt, bg):
        ctx.bg = bg
        op0 = bg.ops[0]
        keep_t = wgt is not None and wgt.requires_grad
        out = torch.empty((len(bg), op0.nrow, op0.nchan), dtype=op0.cdt, device=dirty.device)
        ts = torch.empty_like(out) if keep_t else None
        dirty_d = dirty.detach()
        wgt_d = None if wgt is None else wgt.detach()

        def run(b, op):
            if keep_t:
                t = op.adjoint(dirty_d[b], None)              # A^H dirty
                ts[b].copy_(t)
                out[b].copy_(t * wgt_d[b])
            else:
                out[b].copy_(op.adjoint(dirty_d[b], None if wgt_d is None else wgt_d[b]))
        bg._each(run)
        ctx.save_for_backward(wgt, ts)
        return out

    @staticmethod
    def backward(ctx, g):
        wgt, ts = ctx.saved_tensors
        bg = ctx.bg
        g = g.contiguous()
        need_d, need_w = ctx.needs_input_grad[0], ctx.needs_input_grad[1] and wgt is not None
        op0 = bg.ops[0]
        gd = torch.empty((len(bg), op0.nx, op0.ny), dtype=op0.cdt, device=g.device) if need_d else None
        gw = (g * ts.conj()).real.to(wgt.dtype) if need_w else None
        wgt_d = None if wgt is None else wgt.detach()

        def run(b, op):
            op.plan.execute_dir(1, g[b], None if wgt_d is None else wgt_d[b], gd[b])
        if need_d:
            bg._each(run)
        return gd, gw, None
