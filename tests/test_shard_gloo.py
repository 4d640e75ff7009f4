"""Row sharding over ranks (world size 2, gloo on the CPU): partial ms2dirty
images summed by one all-reduce (or a reduce to a root) equal the single-process
result, and dirty2ms after a broadcast equals the local rows of the full one.
The per-rank operator is the FP64 DFT of the oracle (test infrastructure), so
only the sharding / collective logic is under test here."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import disk_inputs


class DftOp:
    """CPU stand-in with the library's conventions (weights in both directions)."""

    def __init__(self, uvw, freq, nx, ny, psx, psy):
        self.uvw, self.freq, self.nx, self.ny, self.psx, self.psy = uvw, freq, nx, ny, psx, psy

    def apply(self, vis, wgt=None):
        from oracle import dft
        w = np.ones(vis.shape) if wgt is None else wgt.numpy()
        d = dft.ms2dirty_dft(self.uvw, self.freq, vis.numpy(), w, self.nx, self.ny, self.psx, self.psy, -1)
        return torch.from_numpy(np.ascontiguousarray(d).reshape(self.nx, self.ny))

    def adjoint(self, dirty, wgt=None):
        from oracle import dft
        w = np.ones((self.uvw.shape[0], len(self.freq))) if wgt is None else wgt.numpy()
        v = dft.dirty2ms_dft(self.uvw, self.freq, dirty.numpy(), w, self.psx, self.psy, -1)
        return torch.from_numpy(np.ascontiguousarray(v).reshape(self.uvw.shape[0], len(self.freq)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from curig_b200.shard import ShardedGridder, row_range
        nx = ny = 24
        freq, uvw, ms, wgt = disk_inputs(101, 3, nx, 2.0, max_pix=10, seed=5)
        psx = 2.0 * np.pi / 180 / nx
        r0, r1 = row_range(uvw.shape[0], rank, world)
        op = DftOp(uvw[r0:r1], freq, nx, ny, psx, psx)
        sg = ShardedGridder(None, freq, nx, ny, psx, psx, 1e-12, local_op=op)
        full = sg.ms2dirty(torch.from_numpy(ms[r0:r1]), torch.from_numpy(wgt[r0:r1]))
        red = sg.ms2dirty(torch.from_numpy(ms[r0:r1]), torch.from_numpy(wgt[r0:r1]), root=0)
        img = torch.from_numpy(np.random.default_rng(9).standard_normal((nx, ny)) + 0j)
        if rank != 0:
            img = torch.zeros_like(img)                # only the root holds the image
        vis = sg.dirty2ms(img, torch.from_numpy(wgt[r0:r1]), root=0)
        out[rank] = (full.numpy(), red.numpy() if rank == 0 else None, vis.numpy(), (r0, r1))
    finally:
        dist.destroy_process_group()


def test_row_range_partitions_exactly():
    from curig_b200.shard import row_range
    for nrow in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            spans = [row_range(nrow, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nrow
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        row_range(10, 2, 2)


def test_sharded_ms2dirty_dirty2ms_world2():
    from oracle import dft
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    nx = ny = 24
    freq, uvw, ms, wgt = disk_inputs(101, 3, nx, 2.0, max_pix=10, seed=5)
    psx = 2.0 * np.pi / 180 / nx
    ref = dft.ms2dirty_dft(uvw, freq, ms, wgt, nx, ny, psx, psx, -1).reshape(nx, ny)
    for r in range(world):
        assert np.allclose(res[r][0], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    assert np.allclose(res[0][1], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    img = np.random.default_rng(9).standard_normal((nx, ny)) + 0j
    vref = dft.dirty2ms_dft(uvw, freq, img, wgt, psx, psx, -1).reshape(uvw.shape[0], len(freq))
    got = np.concatenate([res[r][2] for r in range(world)], 0)
    assert [res[r][3] for r in range(world)] == [(0, 51), (51, 101)]
    assert np.allclose(got, vref, rtol=1e-12, atol=1e-12 * np.abs(vref).max())
