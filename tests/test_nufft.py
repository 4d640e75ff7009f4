"""Generic NUFFT (types 1 and 2, one and two dimensions) against the direct
nonuniform DFT (numpy, FP64), with points inside and beyond [-pi, pi)."""
import numpy as np
import pytest


def _direct(x, y, n_modes, iflag):
    """Matrix E[j, k] = exp(i iflag k.x_j) over the modes k = index - n/2."""
    k1 = np.arange(n_modes[0]) - n_modes[0] // 2
    ph = np.outer(x, k1)
    if len(n_modes) == 2:
        k2 = np.arange(n_modes[1]) - n_modes[1] // 2
        ph = ph[:, :, None] + np.outer(y, k2)[:, None, :]
    return np.exp(1j * iflag * ph).reshape(len(x), -1)


def test_nufft_symbols_exported():
    from curig_b200 import _lib
    for name in ("curig_nufft_makeplan", "curig_nufft_setpts", "curig_nufft_execute", "curig_nufft_destroy"):
        assert hasattr(_lib.lib, name)


CASES = [((64,), 1), ((64,), -1), ((40, 36), 1), ((40, 36), -1), ((33, 17), 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("n_modes,iflag", CASES)
@pytest.mark.parametrize("precision,eps,tol", [("fp64", 1e-10, 1e-9), ("fp32", 1e-5, 3e-5)])
def test_nufft_types_1_and_2_match_direct(n_modes, iflag, precision, eps, tol):
    import torch
    from curig_b200.nufft import Nufft
    rng = np.random.default_rng(sum(n_modes) + iflag)
    m = 700
    x = rng.uniform(-np.pi, np.pi, m)
    x[:50] *= 2.5                                   # periodic beyond [-pi, pi)
    y = rng.uniform(-np.pi, np.pi, m)
    c = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    fk = rng.standard_normal(n_modes) + 1j * rng.standard_normal(n_modes)
    E = _direct(x, y, n_modes, iflag)
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda() if len(n_modes) == 2 else None
    p1 = Nufft(1, n_modes, eps, iflag, precision=precision)
    p1.setpts(dx, dy)
    out = torch.empty(n_modes, dtype=cdt, device="cuda")
    p1.execute(torch.from_numpy(c).to(cdt).cuda(), out)
    ref1 = (c @ E).reshape(n_modes)
    got1 = out.cpu().numpy()
    assert np.linalg.norm(got1 - ref1) <= tol * np.linalg.norm(ref1)
    p2 = Nufft(2, n_modes, eps, iflag, precision=precision)
    p2.setpts(dx, dy)
    cout = torch.empty(m, dtype=cdt, device="cuda")
    p2.execute(cout, torch.from_numpy(fk).to(cdt).cuda())
    ref2 = E @ fk.reshape(-1)
    got2 = cout.cpu().numpy()
    assert np.linalg.norm(got2 - ref2) <= tol * np.linalg.norm(ref2)
    p1.close()
    p2.close()


@pytest.mark.gpu
def test_nufft_rejects_bad_arguments():
    from curig_b200._lib import CurigError
    from curig_b200.nufft import Nufft
    with pytest.raises(CurigError):
        Nufft(3, (16, 16), 1e-6)                   # type 3 is one-dimensional
    with pytest.raises(CurigError):
        Nufft(1, (16, 16), 1e-6, iflag=2)


# ------------------------------------------------------------------ type 3
def _direct3(x, s, c, iflag):
    return np.exp(1j * iflag * np.outer(s, x)) @ c


def _type3(x, s, c, iflag, eps, precision="fp64"):
    import torch
    from curig_b200.nufft import Nufft3
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    p = Nufft3(eps, iflag, precision=precision)
    p.setpts(torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda(),
             torch.from_numpy(np.ascontiguousarray(s, dtype=np.float64)).cuda())
    out = torch.empty(len(s), dtype=cdt, device="cuda")
    p.execute(torch.from_numpy(np.ascontiguousarray(c)).to(cdt).cuda(), out)
    info = p.info()
    p.close()
    return out.cpu().numpy(), info


@pytest.mark.gpu
def test_type3_reference_case_points_to_frequencies():
    """test/nufft_1d_3_1_test.cu:32-62,210-241 of the reference: M = 100 points
    u_i = 2 + i pi / M, strengths (uniform(-1,1) * 1000, i), N = 100 frequencies
    k_i = -i / N, epsilon 1e-6, iflag +1, against the direct sum."""
    M, N, eps = 100, 100, 1e-6
    rng = np.random.default_rng(31)
    u = 2.0 + np.arange(M) * np.pi / M
    c = rng.uniform(-1, 1, M) * 1000 + 1j * np.arange(M)
    k = -np.arange(N) / N
    got, info = _type3(u, k, c, +1, eps)
    ref = _direct3(u, k, c, +1)
    assert info["nf"] >= 2 * 7 and info["nf"] % 2 == 0
    assert np.linalg.norm(got - ref) <= 10 * eps * np.linalg.norm(ref)


@pytest.mark.gpu
def test_type3_reference_case_single_frequency_to_points():
    """test/nufft_1d_3_2_test.cu:31-95,110-160 of the reference: values at one
    frequency (k = 0) transformed to M = 25 points u_i = 2 + i with iflag -1,
    epsilon 1e-12 -- the same type 3 with points and frequencies exchanged."""
    M, eps = 25, 1e-12
    k = np.array([0.0])
    fk = np.array([0.7 - 0.3j])
    u = 2.0 + np.arange(M, dtype=np.float64)
    got, _ = _type3(k, u, fk, -1, eps)
    ref = _direct3(k, u, fk, -1)
    assert np.linalg.norm(got - ref) <= 1e-9 * np.linalg.norm(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("iflag", (1, -1))
@pytest.mark.parametrize("precision,eps,tol", [("fp64", 1e-9, 1e-8), ("fp64", 1e-4, 1e-3), ("fp32", 1e-5, 5e-5)])
def test_type3_random_wide_ranges(iflag, precision, eps, tol):
    rng = np.random.default_rng(7 + iflag)
    m, n = 3000, 2000
    x = rng.uniform(-30.0, 50.0, m)
    s = rng.uniform(-80.0, 20.0, n)
    c = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    got, info = _type3(x, s, c, iflag, eps, precision)
    ref = _direct3(x, s, c, iflag)
    assert abs(info["i_center"] - (x.max() + x.min()) / 2) < 1e-12 * 50
    assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref)


# ------------------------------------------------------------------ 3-D types 1 and 2
def _direct3d(x, y, z, n_modes, iflag):
    ks = [np.arange(n) - n // 2 for n in n_modes]
    ph = (np.outer(x, ks[0])[:, :, None, None] + np.outer(y, ks[1])[:, None, :, None]
          + np.outer(z, ks[2])[:, None, None, :])
    return np.exp(1j * iflag * ph).reshape(len(x), -1)


@pytest.mark.gpu
@pytest.mark.parametrize("n_modes,iflag", [((12, 10, 8), 1), ((12, 10, 8), -1), ((16, 6, 21), 1)])
@pytest.mark.parametrize("precision,eps,tol", [("fp64", 1e-10, 1e-9), ("fp32", 1e-5, 3e-5)])
def test_nufft_3d_types_1_and_2_match_direct(n_modes, iflag, precision, eps, tol):
    """The reference's cunufft_setting in three dimensions (src/fourier/cuft.cu:293-305)."""
    import torch
    from curig_b200.nufft import Nufft
    rng = np.random.default_rng(sum(n_modes) + 7 * iflag)
    m = 600
    x, y, z = (rng.uniform(-np.pi, np.pi, m) for _ in range(3))
    z[:40] *= 2.2                                   # periodic beyond [-pi, pi) on the third axis too
    c = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    fk = rng.standard_normal(n_modes) + 1j * rng.standard_normal(n_modes)
    E = _direct3d(x, y, z, n_modes, iflag)
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    dx, dy, dz = (torch.from_numpy(a).cuda() for a in (x, y, z))
    p1 = Nufft(1, n_modes, eps, iflag, precision=precision)
    p1.setpts(dx, dy, dz)
    out = torch.empty(n_modes, dtype=cdt, device="cuda")
    p1.execute(torch.from_numpy(c).to(cdt).cuda(), out)
    ref1 = (c @ E).reshape(n_modes)
    assert np.linalg.norm(out.cpu().numpy() - ref1) <= tol * np.linalg.norm(ref1)
    p2 = Nufft(2, n_modes, eps, iflag, precision=precision)
    p2.setpts(dx, dy, dz)
    cout = torch.empty(m, dtype=cdt, device="cuda")
    p2.execute(cout, torch.from_numpy(fk).to(cdt).cuda())
    ref2 = E @ fk.reshape(-1)
    assert np.linalg.norm(cout.cpu().numpy() - ref2) <= tol * np.linalg.norm(ref2)
    p1.close()
    p2.close()
