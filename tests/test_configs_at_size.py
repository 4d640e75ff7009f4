"""Parity at the full configuration sizes, through the C ABI.

The 4096^2 configuration (fov 3 deg, sigma 2, Gaussian (u, v) density of
sigma 0.3 R, w uniform in +-1000 m, 16 channels 0.9-1.1 GHz), 2e6 rows x 16
channels, for epsilon 1e-4 / 1e-5 / 1e-6 and every precision form (FP64; FP32
with exact two-word tiles; FP32 with one-word tiles):

* against the FP64 DFT (oracle/dft_torch.py, pinned to oracle/dft.c) on 2,000
  sampled pixels and 2,000 sampled visibilities, at the reference's width rule;
* against the reference library's own outputs at the same inputs
  (tests/golden/reflib_cfg2_*.npz, recorded by make_ref_cfg2.py from the
  reference's libcurafft.so on a B200): the per-channel reference ABI
  like for like (1e-9), the multi-channel call, and the FP32 forms;
* FP32 against FP64 on the whole image (the precision form's cost);
* the bench density (1e7 rows x 16 channels) with one-word tiles, where the
  fixed-point box bound is exercised by 4096-visibility chunks of the
  Gaussian core;
* the learned window's width choice at 4096^2 against epsilon;

and the batch-of-8 configuration (8 x 1e6 visibilities, 1024^2): adjointness
at full size and finite differences along a random direction (FP64, step
1e-3).  Reference pattern: python/curagridder/test_wst.py:36-83."""
import ctypes
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, gaussian_image, gaussian_uv_inputs, input_checksum

pytestmark = pytest.mark.gpu

NPIX, FOV, NCHAN, NROW = 4096, 3.0, 16, 2_000_000
PSX = FOV * np.pi / 180 / NPIX
EPS = (1e-4, 1e-5, 1e-6)
FORMS = {"fp64": (0, 0), "fp32_two_word": (1, 3), "fp32_one_word": (1, 2)}   # precision, accumulate


def _samples(nrow):
    rng = np.random.default_rng(5)
    pix = np.sort(rng.choice(NPIX * NPIX, 2000, replace=False)).astype(np.int64)
    vidx = np.sort(rng.choice(nrow * NCHAN, 2000, replace=False)).astype(np.int64)
    return pix, vidx


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _cast(prec, uvw, vis, wgt, img):
    if prec:
        return (uvw, np.ascontiguousarray(vis.astype(np.complex64)), np.ascontiguousarray(wgt.astype(np.float32)),
                np.ascontiguousarray(img.astype(np.complex64)))
    return uvw, vis, wgt, img


def _oneshot(L, kind, prec, acc, freq, uvw, vis, wgt, img, eps, window=0):
    """curig_ms2dirty (kind 1) / curig_dirty2ms (kind 2) from host buffers."""
    nrow, nchan = vis.shape
    opts = L.make_opts(precision=prec, accumulate=acc, window=window)
    fr = np.ascontiguousarray(freq, dtype=np.float64)
    if kind == 1:
        out = np.zeros((NPIX, NPIX), dtype=np.complex64 if prec else np.complex128)
        st = L.lib.curig_ms2dirty(nrow, nchan, NPIX, NPIX, PSX, PSX, fr.ctypes.data, uvw.ctypes.data,
                                  vis.ctypes.data, wgt.ctypes.data, out.ctypes.data, eps, 2.0, -1,
                                  ctypes.byref(opts))
    else:
        out = np.zeros((nrow, nchan), dtype=np.complex64 if prec else np.complex128)
        st = L.lib.curig_dirty2ms(nrow, nchan, NPIX, NPIX, PSX, PSX, fr.ctypes.data, uvw.ctypes.data,
                                  out.ctypes.data, wgt.ctypes.data, img.ctypes.data, eps, 2.0, -1,
                                  ctypes.byref(opts))
    assert st == 0, L.lib.curig_last_error()
    return out


@pytest.fixture(scope="module")
def cfg2():
    """Inputs and the FP64 DFT truth at the sampled pixels / visibilities."""
    import torch
    from oracle import dft_torch
    freq, uvw, vis, wgt = gaussian_uv_inputs(NROW, NCHAN, NPIX, FOV, seed=0)
    img = gaussian_image(NPIX, seed=1)
    pix, vidx = _samples(NROW)
    u = torch.from_numpy(uvw).cuda()
    truth_d = dft_torch.ms2dirty_dft(u, freq, torch.from_numpy(vis).cuda(), torch.from_numpy(wgt).cuda(),
                                     NPIX, NPIX, PSX, PSX, -1, pix)
    truth_v = dft_torch.dirty2ms_dft(u, freq, torch.from_numpy(img).cuda(), torch.from_numpy(wgt).cuda(),
                                     PSX, PSX, -1, vidx)
    del u
    torch.cuda.empty_cache()
    return dict(freq=freq, uvw=uvw, vis=vis, wgt=wgt, img=img, pix=pix, vidx=vidx, truth_d=truth_d,
                truth_v=truth_v)


@pytest.fixture(scope="module")
def L():
    import curig_b200._lib as lib
    return lib


@pytest.mark.parametrize("form", list(FORMS))
@pytest.mark.parametrize("eps", EPS)
def test_cfg2_against_dft(cfg2, L, eps, form):
    prec, acc = FORMS[form]
    uvw, vis, wgt, img = _cast(prec, cfg2["uvw"], cfg2["vis"], cfg2["wgt"], cfg2["img"])
    d = _oneshot(L, 1, prec, acc, cfg2["freq"], uvw, vis, wgt, img, eps)
    v = _oneshot(L, 2, prec, acc, cfg2["freq"], uvw, vis, wgt, img, eps)
    ed = _rel(d.reshape(-1)[cfg2["pix"]], cfg2["truth_d"])
    ev = _rel(v.reshape(-1)[cfg2["vidx"]], cfg2["truth_v"])
    est = _estimate(cfg2, prec, acc, eps)
    print(f"\n[cfg2 {NROW}x{NCHAN}] eps {eps:g} {form}: ms2dirty vs DFT {ed:.3e}, dirty2ms vs DFT {ev:.3e}, "
          f"stated {est:.3e}")
    # the reference's width rule reaches about 1.1-1.4 eps here; FP32 adds ~3e-7 (one word ~1.5e-6)
    assert ed <= 3 * eps and ev <= 3 * eps
    # the error each plan states for its results (curig_plan_error) holds within a factor of 2
    assert est / 2 <= max(ed, ev) <= 2 * est


def _estimate(cfg2, prec, acc, eps):
    """curig_plan_error of a device plan with the same options (ms2dirty)."""
    import torch
    from curig_b200.plan import GridderPlan
    p = GridderPlan(1, NPIX, NPIX, PSX, PSX, eps, 2.0, -1, precision="fp32" if prec else "fp64", window="es",
                    accumulate=acc)
    p.setpts(torch.from_numpy(cfg2["uvw"]).cuda(), cfg2["freq"])
    est = p.error_estimate()["total"]
    p.close()
    return est


def _reflib_cfg2():
    return sorted(glob.glob(os.path.join(GOLDEN, "reflib_cfg2_*.npz")))


@pytest.mark.parametrize("path", _reflib_cfg2(), ids=os.path.basename)
def test_cfg2_against_reference_library(cfg2, L, path):
    g = np.load(path)
    assert int(g["nrow"]) == NROW and int(g["nchan"]) == NCHAN
    assert float(g["checksum"]) == input_checksum(cfg2["uvw"], cfg2["vis"], cfg2["wgt"]), "inputs changed"
    assert float(g["image_checksum"]) == input_checksum(cfg2["img"])
    pix, vidx = g["pix"], g["vidx"]
    assert np.array_equal(pix, cfg2["pix"]) and np.array_equal(vidx, cfg2["vidx"])
    freq, uvw, vis, wgt, img = cfg2["freq"], cfg2["uvw"], cfg2["vis"], cfg2["wgt"], cfg2["img"]
    vrow, vch = vidx // NCHAN, vidx % NCHAN
    for k, eps in enumerate(g["epsilons"]):
        assert not np.any(g[f"status_{k}"]), "the reference library reported an error"
        ref_d, ref_v = g[f"ms2dirty_{k}"], g[f"dirty2ms_{k}"]
        # like for like: the reference ABI once per channel (FP64, host buffers)
        acc = np.zeros((NPIX, NPIX), dtype=np.complex128)
        out = np.zeros((NPIX, NPIX), dtype=np.complex128)
        got_v = np.zeros(vidx.size, dtype=np.complex128)
        for c in range(NCHAN):
            vc, wc = np.ascontiguousarray(vis[:, c]), np.ascontiguousarray(wgt[:, c])
            assert L.ms2dirty_2(NROW, NPIX, NPIX, FOV, float(freq[c]), uvw, vc, wc, out, eps, 2.0, -1) == 0
            acc += out
            vo = np.zeros(NROW, dtype=np.complex128)
            assert L.dirty2ms_2(NROW, NPIX, NPIX, FOV, float(freq[c]), uvw, vo, wc, img, eps, 2.0, -1) == 0
            sel = vch == c
            got_v[sel] = vo[vrow[sel]]
        e1d, e1v = _rel(acc.reshape(-1)[pix], ref_d), _rel(got_v, ref_v)
        nrm = abs(np.linalg.norm(acc) / float(g[f"ms2dirty_norm_{k}"]) - 1)
        # multi-channel calls (all channels in one transform) and the FP32 forms
        md = {f: _oneshot(L, 1, *FORMS[f], freq, *_cast(FORMS[f][0], uvw, vis, wgt, img), eps).reshape(-1)[pix]
              for f in FORMS}
        mv = {f: _oneshot(L, 2, *FORMS[f], freq, *_cast(FORMS[f][0], uvw, vis, wgt, img), eps).reshape(-1)[vidx]
              for f in FORMS}
        ed = {f: _rel(md[f], ref_d) for f in FORMS}
        ev = {f: _rel(mv[f], ref_v) for f in FORMS}
        print(f"\n[reflib cfg2] eps {eps:g}: per-channel ABI {e1d:.2e} / {e1v:.2e} (norm {nrm:.1e}); "
              + ", ".join(f"{f} {ed[f]:.2e} / {ev[f]:.2e}" for f in FORMS))
        assert e1d <= 1e-9 and e1v <= 1e-9 and nrm <= 1e-9
        # one transform over all channels is another discretisation within eps of the truth
        assert ed["fp64"] <= 0.1 * eps and ev["fp64"] <= 0.1 * eps
        assert ed["fp32_two_word"] <= 1e-6 and ev["fp32_two_word"] <= 1e-6
        assert ed["fp32_one_word"] <= 4e-6 and ev["fp32_one_word"] <= 1e-6


@pytest.mark.parametrize("eps", EPS)
def test_cfg2_fp32_against_fp64_whole_image(cfg2, L, eps):
    """The precision form's own error, at full density: FP32 ms2dirty of all
    3.2e7 visibilities against the FP64 result, relative L2 over the image."""
    freq = cfg2["freq"]
    d64 = _oneshot(L, 1, 0, 0, freq, cfg2["uvw"], cfg2["vis"], cfg2["wgt"], cfg2["img"], eps)
    errs = {}
    for f in ("fp32_two_word", "fp32_one_word"):
        prec, acc = FORMS[f]
        d = _oneshot(L, 1, prec, acc, freq, *_cast(prec, cfg2["uvw"], cfg2["vis"], cfg2["wgt"], cfg2["img"]), eps)
        errs[f] = _rel(d.astype(np.complex128), d64)
    print(f"\n[cfg3] eps {eps:g}: FP32 vs FP64 whole image: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert errs["fp32_two_word"] <= 1e-6
    assert errs["fp32_one_word"] <= 4e-6


def test_bench_density_one_word_tiles(L):
    """1e7 rows x 16 channels (the bench's density), FP32 one-word tiles at
    eps 1e-5: within 3 eps of the DFT on 2,000 pixels and within 4e-6 of the
    exact two-word tiles over the whole image."""
    import torch
    from oracle import dft_torch
    nrow = 10_000_000
    freq, uvw, vis, wgt = gaussian_uv_inputs(nrow, NCHAN, NPIX, FOV, seed=2)
    pix = np.random.default_rng(6).choice(NPIX * NPIX, 2000, replace=False)
    truth = dft_torch.ms2dirty_dft(torch.from_numpy(uvw).cuda(), freq, torch.from_numpy(vis).cuda(),
                                   torch.from_numpy(wgt).cuda(), NPIX, NPIX, PSX, PSX, -1, pix)
    torch.cuda.empty_cache()
    u, v, w, _ = _cast(1, uvw, vis, wgt, np.zeros((1, 1)))
    del vis, wgt
    one = _oneshot(L, 1, 1, 2, freq, u, v, w, None, 1e-5)
    two = _oneshot(L, 1, 1, 3, freq, u, v, w, None, 1e-5)
    e_dft = _rel(one.reshape(-1)[pix], truth)
    e_two = _rel(one, two)
    print(f"\n[bench density 1e7x16] one-word vs DFT {e_dft:.3e}, one-word vs two-word {e_two:.3e}")
    assert e_dft <= 3e-5 and e_two <= 4e-6


def test_learned_window_width_meets_eps_at_4096(cfg2, L):
    """The learned window picks its width from an error calibrated on a small
    problem; at 4096^2 the width it picks must still meet epsilon against the DFT."""
    from curig_b200 import learned
    assert learned.load_default_windows()
    try:
        eps = 1e-5
        uvw, vis, wgt, img = _cast(1, cfg2["uvw"], cfg2["vis"], cfg2["wgt"], cfg2["img"])
        d = _oneshot(L, 1, 1, 0, cfg2["freq"], uvw, vis, wgt, img, eps, window=1)
        v = _oneshot(L, 2, 1, 0, cfg2["freq"], uvw, vis, wgt, img, eps, window=1)
        ed = _rel(d.reshape(-1)[cfg2["pix"]], cfg2["truth_d"])
        ev = _rel(v.reshape(-1)[cfg2["vidx"]], cfg2["truth_v"])
        print(f"\n[learned window at 4096^2] ms2dirty {ed:.3e}, dirty2ms {ev:.3e}")
        assert ed <= eps and ev <= eps
    finally:
        learned.clear()


# ------------------------------------------------------------------ batch of 8 x 1e6, 1024^2
def _cfg5(precision, seed=0):
    import torch
    from conftest import disk_inputs
    B, nrow, npix, fov = 8, 1_000_000, 1024, 2.0
    data = [disk_inputs(nrow, 1, npix, fov, max_pix=0.47 * npix, seed=seed + b) for b in range(B)]
    cdt = torch.complex64 if precision == "fp32" else torch.complex128
    rdt = torch.float32 if precision == "fp32" else torch.float64
    uvws = [torch.from_numpy(x[1]).cuda() for x in data]
    vis = torch.stack([torch.from_numpy(x[2]).to(cdt) for x in data]).cuda()
    wgt = torch.stack([torch.from_numpy(x[3]).to(rdt) for x in data]).cuda()
    return data[0][0], uvws, vis, wgt, npix, fov * np.pi / 180 / npix


def test_cfg5_batch_adjointness_full_size():
    """<A x, y> = <x, A^H y> for all 8 problems of 1e6 visibilities at 1024^2
    (FP32, eps 1e-5), relative to the Cauchy-Schwarz bound |A x| |y| (the
    inner product itself cancels to about |A x| |y| / sqrt(N)): within the
    FP32 arithmetic."""
    import torch
    from curig_b200.autograd import BatchGridder
    freq, uvws, vis, wgt, npix, psx = _cfg5("fp32")
    bg = BatchGridder(uvws, freq, npix, npix, psx, psx, 1e-5, precision="fp32")
    g = torch.Generator(device="cuda").manual_seed(3)
    y = torch.complex(torch.randn((8, npix, npix), generator=g, device="cuda"),
                      torch.randn((8, npix, npix), generator=g, device="cuda"))
    with torch.no_grad():
        ax = bg.ms2dirty(vis, wgt)
        ahy = bg.dirty2ms(y, wgt)
    for b in range(8):
        lhs = torch.vdot(ax[b].reshape(-1).to(torch.complex128), y[b].reshape(-1).to(torch.complex128))
        rhs = torch.vdot(vis[b].reshape(-1).to(torch.complex128), ahy[b].reshape(-1).to(torch.complex128))
        bound = float(torch.linalg.vector_norm(ax[b]) * torch.linalg.vector_norm(y[b]))
        rel = float(abs(lhs - rhs)) / bound
        assert rel <= 1e-6, (b, rel)
    bg.close()


def test_cfg5_finite_differences_full_size():
    """Gradients of ||ms2dirty(v, w) - d||^2 with respect to the visibilities and
    the weights of all 8 problems (FP64 plans, eps 1e-10) against central finite
    differences with step 1e-3 along a random direction."""
    import torch
    from curig_b200.autograd import BatchGridder
    freq, uvws, vis, wgt, npix, psx = _cfg5("fp64", seed=40)
    bg = BatchGridder(uvws, freq, npix, npix, psx, psx, 1e-10, precision="fp64")
    g = torch.Generator(device="cuda").manual_seed(4)

    def rnd(shape, cplx):
        r = torch.randn(shape, generator=g, device="cuda", dtype=torch.float64)
        return torch.complex(r, torch.randn(shape, generator=g, device="cuda", dtype=torch.float64)) if cplx else r

    d = rnd((8, npix, npix), True)

    def loss(v, w):
        return ((bg.ms2dirty(v, w) - d).abs() ** 2).sum()

    v = vis.clone().requires_grad_()
    w = wgt.clone().requires_grad_()
    loss(v, w).backward()
    dv, dw, h = rnd(vis.shape, True), rnd(wgt.shape, False), 1e-3
    with torch.no_grad():
        fd_v = (loss(vis + h * dv, wgt) - loss(vis - h * dv, wgt)) / (2 * h)
        fd_w = (loss(vis, wgt + h * dw) - loss(vis, wgt - h * dw)) / (2 * h)
    an_v = (v.grad.conj() * dv).real.sum()
    an_w = (w.grad * dw).sum()
    print(f"\n[cfg5 FD] vis {float(abs(fd_v - an_v) / abs(fd_v)):.2e}, wgt {float(abs(fd_w - an_w) / abs(fd_w)):.2e}")
    assert abs(float(fd_v - an_v)) <= 1e-7 * abs(float(fd_v))
    assert abs(float(fd_w - an_w)) <= 1e-7 * abs(float(fd_w))
    bg.close()
