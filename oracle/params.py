"""Oracle: CPU restatement of CuRIG's parameter rules for ms2dirty / dirty2ms.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``curig_b200``) imports this
module; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg use it, and only as the checker.

Every rule below restates the reference's arithmetic (same operation order,
FP64) so that the sizes chosen here (kernel width, beta, grid sizes, number of
w-planes, gamma, h) are bit-identical to the reference's:

* kernel width / ES beta / ES c ......... src/fourier/conv_interp_invoker.cu:46-116
* fine grid size (get_num_cells) ......... src/fourier/conv_interp_invoker.cu:29-44
* 2-3-5-smooth even sizes ................ src/utils.cu:251-276 (next235beven),
                                           contrib/common.cpp:15-33 (next235even)
* w-plane count, h, gamma (type-3) ....... contrib/common.cpp:161-195 (set_nhg_type3)
* pixel sizes, n-1 corner, w centre ...... src/astro/cugridder.cu:29-101
* effective coordinates .................. src/astro/precomp.cu:48-79
* kernel Fourier transform (quadrature) .. src/fourier/deconv.cu:13-197

The Gauss-Legendre rule is written from its definition (Newton iteration on the
three-term Legendre recurrence); the reference vendors the Glaser-Liu-Rokhlin
code (contrib/legendre_rule_fast.c:15-93) for the same nodes and weights.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SPEEDOFLIGHT = 299792458.0          # include/utils.h:103
PI = math.pi                        # include/utils.h:97 (M_PI)
M_1_2PI = 0.159154943091895336      # include/utils.h:94
EPSILON = 1.1e-16                   # include/utils.h:99
MAX_KERNEL_WIDTH = 28               # include/curafft_plan.h:14
INT_MAX = 2147483647                # g++ folds (int)1e11 in contrib/common.h:14 to INT_MAX


def next235beven(n: int, b: int = 1) -> int:
    """Smallest even n' >= n whose prime factors are 2, 3, 5 and n' % b == 0
    (src/utils.cu:251-276)."""
    if n <= 2:
        return 2
    if n % 2 == 1:
        n += 1
    nplus = n - 2
    numdiv = 2
    while numdiv > 1 or nplus % b != 0:
        nplus += 2
        numdiv = nplus
        for f in (2, 3, 5):
            while numdiv % f == 0:
                numdiv //= f
    return nplus


def next235even(n: int) -> int:
    """contrib/common.cpp:15-33 (same rule with b = 1)."""
    return next235beven(n, 1)


@dataclass
class ConvOpts:
    kw: int
    beta: float
    c: float
    halfwidth: float
    upsampfac: float
    ier: int = 0


def setup_conv_opts(eps: float, upsampfac: float, kerevalmeth: int = 0) -> ConvOpts:
    """Kernel width and ES parameters (src/fourier/conv_interp_invoker.cu:63-116)."""
    ier = 0
    if upsampfac != 2.0:
        if kerevalmeth == 1:
            raise ValueError("nonstandard upsampling factor with kerevalmeth=1")
        if upsampfac <= 1.0:
            raise ValueError("upsampling factor too small")
    if eps < EPSILON:
        eps = EPSILON
        ier = 1
    kw = math.ceil(-math.log10(eps / 10.0))
    if upsampfac != 2.0:
        kw = math.ceil(-math.log(eps) / (PI * math.sqrt(1.0 - 1.0 / upsampfac)))
    kw = max(2, kw)
    if kw > MAX_KERNEL_WIDTH:
        kw = MAX_KERNEL_WIDTH
    betaoverns = 2.30
    if kw == 2:
        betaoverns = 2.20
    if kw == 3:
        betaoverns = 2.26
    if kw == 4:
        betaoverns = 2.38
    if upsampfac != 2.0:
        gamma = 0.97
        betaoverns = gamma * PI * (1 - 1 / (2 * upsampfac))
    return ConvOpts(kw=kw, beta=betaoverns * kw, c=4.0 / (kw * kw),
                    halfwidth=kw / 2.0, upsampfac=upsampfac, ier=ier)


def get_num_cells(ms: int, opts: ConvOpts) -> int:
    """src/fourier/conv_interp_invoker.cu:29-44."""
    nf = int(opts.upsampfac * ms)
    if nf < 2 * opts.kw:
        nf = 2 * opts.kw
    if nf < 1e11:
        nf = next235beven(nf, 1)
    return nf


def set_nhg_type3(S: float, X: float, opts: ConvOpts):
    """(nf, h, gamma) for the w axis (contrib/common.cpp:161-195)."""
    nss = opts.kw + 1
    Xsafe, Ssafe = X, S
    if X == 0.0:
        if S == 0.0:
            Xsafe, Ssafe = 1.0, 1.0
        else:
            Xsafe = max(Xsafe, 1 / S)
    else:
        Ssafe = max(Ssafe, 1 / X)
    nfd = 2.0 * opts.upsampfac * Ssafe * Xsafe / PI + nss
    if not math.isfinite(nfd):
        nfd = 0.0
    nf = int(nfd)
    if nf < 2 * opts.kw:
        nf = 2 * opts.kw
    if nf < INT_MAX:
        nf = next235even(nf)
    h = 2 * PI / nf
    gam = nf / (2.0 * opts.upsampfac * Ssafe)
    return nf, h, gam


def pixel_sizes(fov_deg: float, nxdirty: int, nydirty: int):
    """(pixelsize_x, pixelsize_y) in radians (src/astro/cugridder.cu:48-49);
    x pairs with nxdirty (N2), y with nydirty (N1)."""
    return fov_deg / 180.0 * PI / nxdirty, fov_deg / 180.0 * PI / nydirty


def gauss_legendre(n: int):
    """n-point Gauss-Legendre nodes (ascending) and weights on [-1, 1].

    Newton iteration on P_n from the three-term recurrence, started at the
    Tricomi approximation; weights 2 / ((1 - x^2) P_n'(x)^2), then scaled to sum
    to 2 (the reference normalises the same way, legendre_rule_fast.c:80-90)."""
    x = np.empty(n)
    w = np.empty(n)
    for i in range(n):
        xi = math.cos(PI * (i + 0.75) / (n + 0.5))
        for _ in range(100):
            p0, p1 = 1.0, xi
            for k in range(2, n + 1):
                p0, p1 = p1, ((2 * k - 1) * xi * p1 - (k - 1) * p0) / k
            if n == 1:
                p0, p1 = 1.0, xi
            dp = n * (xi * p1 - p0) / (xi * xi - 1.0)
            dx = p1 / dp
            xi -= dx
            if abs(dx) < 1e-16:
                break
        p0, p1 = 1.0, xi
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * xi * p1 - (k - 1) * p0) / k
        dp = n * (xi * p1 - p0) / (xi * xi - 1.0)
        x[n - 1 - i] = xi
        w[n - 1 - i] = 2.0 / ((1.0 - xi * xi) * dp * dp)
    w *= 2.0 / w.sum()
    return x, w


def es_kernel(x, opts: ConvOpts):
    """exp(beta*sqrt(1 - c x^2)) on |x| < kw/2, else 0 (src/fourier/conv.cu:17-25;
    no '-1' normalisation)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    m = np.abs(x) < opts.halfwidth
    out[m] = np.exp(opts.beta * np.sqrt(1.0 - opts.c * x[m] * x[m]))
    return out


def quadrature_terms(opts: ConvOpts, window=None):
    """Half-rule nodes x_n (grid units, x >= 0) and weights g_n = alpha*w_n*phi(x_n)
    with p = int(2 + 3*alpha) positive nodes out of a 2p-point rule
    (src/fourier/deconv.cu:60-102, 151-197)."""
    alpha = opts.kw / 2.0
    p = int(2 + 3.0 * alpha)
    z, w = gauss_legendre(2 * p)
    z, w = z[p:], w[p:]                       # the p positive nodes
    xs = z * alpha
    phi = es_kernel(xs, opts) if window is None else window(xs)
    return xs, alpha * w * phi


def psi_hat_grid(nf: int, opts: ConvOpts, window=None):
    """Kernel FT on the fine grid, indices 0..nf/2, including the (-1)^k factor
    from the half-grid shift of the spreading coordinate
    (src/fourier/deconv.cu:13-24 with N = nf/2 + 1)."""
    xs, g = quadrature_terms(opts, window)
    N = nf // 2 + 1
    k = np.arange(N, dtype=np.float64)
    arg = np.outer(k, (xs - N + 1) / (N - 1) * PI)
    return 2.0 * (np.cos(arg) @ g)


def psi_hat_w(kprime, opts: ConvOpts, window=None):
    """Kernel FT along w at the scaled output coordinate k' (deconv.cu:45-57)."""
    xs, g = quadrature_terms(opts, window)
    kp = np.asarray(kprime, dtype=np.float64)
    return 2.0 * (np.cos(np.multiply.outer(kp, xs)) @ g)


@dataclass
class GridderParams:
    nxdirty: int
    nydirty: int
    nf1: int          # fine-grid size along the fastest axis (pairs with v, nydirty)
    nf2: int          # fine-grid size along the slower axis (pairs with u, nxdirty)
    nf3: int          # number of w-planes
    opts: ConvOpts
    pixsize_x: float
    pixsize_y: float
    i_center: float   # centre of the effective w range
    i_half: float
    o_center: float   # centre of the n-1 range
    o_half: float
    gamma: float
    h: float
    sign: int


def effective_w_range(uvw, freqs, sign: int):
    """min/max of w * f/c * sign * 2pi over all rows and channels, in the
    reference's operation order (precomp.cu:61-69)."""
    w = np.asarray(uvw, dtype=np.float64)[:, 2]
    wmin, wmax = float(w.min()), float(w.max())
    lo, hi = math.inf, -math.inf
    for f in np.atleast_1d(freqs):
        a = float(f) / SPEEDOFLIGHT * sign
        for ww in (wmin, wmax):
            v = (ww * a) * (2 * PI)
            lo, hi = min(lo, v), max(hi, v)
    return lo, hi


def gridder_params(nxdirty: int, nydirty: int, fov_deg=None, uvw=None, freqs=None,
                   eps: float = 1e-6, sigma: float = 2.0, sign: int = 1,
                   pixsize_x=None, pixsize_y=None, w_range=None) -> GridderParams:
    """All sizes and scalars of one ms2dirty / dirty2ms call
    (src/astro/cugridder.cu:105-260)."""
    opts = setup_conv_opts(eps, sigma)
    if pixsize_x is None:
        pixsize_x, pixsize_y = pixel_sizes(fov_deg, nxdirty, nydirty)
    N1, N2 = nydirty, nxdirty
    l_min = 0 - 0.5 * pixsize_x * N2
    m_min = 0 - 0.5 * pixsize_y * N1
    n_lm = math.sqrt(1.0 - l_min ** 2 - m_min ** 2)
    if w_range is None:
        w_range = effective_w_range(uvw, freqs, sign)
    i_min, i_max = w_range
    i_center = (i_max + i_min) / 2.0
    i_half = (i_max - i_min) / 2.0
    o_min = n_lm - 1
    o_center = o_min / 2.0
    o_half = abs(o_min / 2.0)
    nf3, h, gam = set_nhg_type3(o_half, i_half, opts)
    nf1 = get_num_cells(N1, opts)
    nf2 = get_num_cells(N2, opts)
    return GridderParams(nxdirty=nxdirty, nydirty=nydirty, nf1=nf1, nf2=nf2, nf3=nf3,
                         opts=opts, pixsize_x=pixsize_x, pixsize_y=pixsize_y,
                         i_center=i_center, i_half=i_half, o_center=o_center,
                         o_half=o_half, gamma=gam, h=h, sign=sign)
