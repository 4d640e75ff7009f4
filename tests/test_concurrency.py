"""Concurrent use: plans on different CUDA streams, and several host threads in
the one-shot ABI at once (each thread on its own per-thread default stream).
Results must equal those of the same calls made one after another."""
import threading

import numpy as np
import pytest

from conftest import disk_inputs, l2err


@pytest.mark.gpu
def test_plans_on_two_streams_run_concurrently():
    import torch
    from curig_b200 import GridderPlan
    nx = ny = 128
    psx = 2.0 * np.pi / 180 / nx
    data = [disk_inputs(20000, 2, nx, 2.0, max_pix=50, wmax=300, seed=30 + k) for k in range(2)]
    streams = [torch.cuda.Stream() for _ in data]
    outs, plans, keep = [], [], []
    for (freq, uvw, ms, wgt), st in zip(data, streams):
        with torch.cuda.stream(st):
            p = GridderPlan(1, nx, ny, psx, psx, 1e-9, stream=st)
            p.setpts(torch.from_numpy(uvw).cuda(), freq)
            v = torch.from_numpy(ms).cuda()
            w = torch.from_numpy(wgt).cuda()
            d = torch.empty((nx, ny), dtype=torch.complex128, device="cuda")
        plans.append(p)
        keep.append((v, w))
        outs.append(d)
    for _ in range(3):                                  # both streams busy at once
        for p, (v, w), d, st in zip(plans, keep, outs, streams):
            with torch.cuda.stream(st):
                p.execute_dir(1, v, w, d)
    torch.cuda.synchronize()
    got = [d.cpu().numpy() for d in outs]
    for p, (v, w), d, st in zip(plans, keep, outs, streams):   # one at a time
        with torch.cuda.stream(st):
            p.execute_dir(1, v, w, d)
        torch.cuda.synchronize()
    for g, d in zip(got, outs):
        assert l2err(d.cpu().numpy(), g) < 1e-12
    for p in plans:
        p.close()


@pytest.mark.gpu
def test_one_shot_calls_from_several_threads():
    import curig_b200 as C
    nx = ny = 96
    psx = 2.0 * np.pi / 180 / nx
    cases = [disk_inputs(8000, 1, nx, 2.0, max_pix=40, wmax=300, seed=40 + k) for k in range(4)]

    def call(k):
        freq, uvw, ms, wgt = cases[k]
        return C.ms2dirty(uvw, freq, ms, wgt, nx, ny, psx, psx, 0, 0, 1e-9, True)

    seq = [call(k) for k in range(4)]
    par = [None] * 4

    def worker(k):
        for _ in range(3):
            par[k] = call(k)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for a, b in zip(seq, par):
        assert l2err(a, b) < 1e-12


@pytest.mark.gpu
def test_release_memory_between_calls():
    """The pool keeps freed memory for the next call; releasing it between
    calls returns it to the driver and the next call allocates it again."""
    import torch
    import curig_b200 as C
    nx = ny = 96
    psx = 2.0 * np.pi / 180 / nx
    freq, uvw, ms, wgt = disk_inputs(8000, 1, nx, 2.0, max_pix=40, wmax=300, seed=50)
    a = C.ms2dirty(uvw, freq, ms, wgt, nx, ny, psx, psx, 0, 0, 1e-9, True)
    torch.cuda.synchronize()
    C.release_memory()
    b = C.ms2dirty(uvw, freq, ms, wgt, nx, ny, psx, psx, 0, 0, 1e-9, True)
    assert l2err(a, b) < 1e-12
