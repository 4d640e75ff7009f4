// Host-side parameter rules of the gridder.  The arithmetic follows the
// reference operation by operation so that kernel width, ES beta, fine-grid
// sizes, w-plane count, gamma and h come out bit-identical:
//   kernel width / beta ......... src/fourier/conv_interp_invoker.cu:46-116
//   fine grid size .............. src/fourier/conv_interp_invoker.cu:29-44
//   2-3-5-smooth even sizes ..... src/utils.cu:251-276, contrib/common.cpp:15-33
//   w planes, h, gamma .......... contrib/common.cpp:161-195
//   pixel sizes, w / n-1 centres  src/astro/cugridder.cu:29-101
//   kernel FT by quadrature ..... src/fourier/deconv.cu:13-197
#include "curig_internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>

namespace curig {

int setup_kernel(double eps, double sigma, KernelParams &kp) {
    kp = KernelParams();
    if (!(sigma > 1.0)) return ERR_SIGMA;          // upsampfac <= 1 is rejected
    if (!(eps > 0.0) || !std::isfinite(eps)) return ERR_ARG;
    int ier = 0;
    if (eps < 1.1e-16) { eps = 1.1e-16; ier = 1; }
    int kw = (int)std::ceil(-std::log10(eps / 10.0));
    if (sigma != 2.0) kw = (int)std::ceil(-std::log(eps) / (PI_D * std::sqrt(1.0 - 1.0 / sigma)));
    kw = std::max(2, kw);
    if (kw > MAX_KW) kw = MAX_KW;
    double bon = 2.30;
    if (kw == 2) bon = 2.20;
    if (kw == 3) bon = 2.26;
    if (kw == 4) bon = 2.38;
    if (sigma != 2.0) bon = 0.97 * PI_D * (1 - 1 / (2 * sigma));
    kp.kw = kw;
    kp.beta = bon * (double)kw;
    kp.c = 4.0 / (double)(kw * kw);
    kp.upsampfac = sigma;
    kp.ier = ier;
    return OK;
}

int next235beven(int n, int b) {
    if (n <= 2) return 2;
    if (n % 2 == 1) n += 1;
    int nplus = n - 2, numdiv = 2;
    while (numdiv > 1 || nplus % b != 0) {
        nplus += 2;
        numdiv = nplus;
        while (numdiv % 2 == 0) numdiv /= 2;
        while (numdiv % 3 == 0) numdiv /= 3;
        while (numdiv % 5 == 0) numdiv /= 5;
    }
    return nplus;
}

int get_num_cells(int ms, const KernelParams &kp) {
    int nf = (int)(kp.upsampfac * ms);
    if (nf < 2 * kp.kw) nf = 2 * kp.kw;
    if (nf < 1e11) nf = next235beven(nf, 1);
    return nf;
}

void set_nhg_type3(double S, double X, const KernelParams &kp, int &nf, double &h, double &gam) {
    int nss = kp.kw + 1;
    double Xsafe = X, Ssafe = S;
    if (X == 0.0) {
        if (S == 0.0) { Xsafe = 1.0; Ssafe = 1.0; }
        else Xsafe = std::max(Xsafe, 1 / S);
    } else {
        Ssafe = std::max(Ssafe, 1 / X);
    }
    double nfd = 2.0 * kp.upsampfac * Ssafe * Xsafe / PI_D + nss;
    if (!std::isfinite(nfd)) nfd = 0.0;
    nf = (int)nfd;
    if (nf < 2 * kp.kw) nf = 2 * kp.kw;
    if (nf < INT_MAX) nf = next235beven(nf, 1);
    h = 2 * PI_D / nf;
    gam = (double)nf / (2.0 * kp.upsampfac * Ssafe);
}

// Gauss-Legendre rule on [-1,1], nodes ascending: Newton iteration on P_n
// evaluated by the three-term recurrence, Tricomi starting values; weights
// 2/((1-x^2) P_n'(x)^2) scaled to sum to 2.
void gauss_legendre(int n, double *x, double *w) {
    for (int i = 0; i < n; ++i) {
        double xi = std::cos(PI_D * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = xi;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2 * k - 1) * xi * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (xi * p1 - p0) / (xi * xi - 1.0);
            double dx = p1 / dp;
            xi -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        double p0 = 1.0, p1 = xi;
        for (int k = 2; k <= n; ++k) {
            double p2 = ((2 * k - 1) * xi * p1 - (k - 1) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (xi * p1 - p0) / (xi * xi - 1.0);
        x[n - 1 - i] = xi;
        w[n - 1 - i] = 2.0 / ((1.0 - xi * xi) * dp * dp);
    }
    double s = 0;
    for (int i = 0; i < n; ++i) s += w[i];
    for (int i = 0; i < n; ++i) w[i] = 2.0 * w[i] / s;
}

// Window value at t (cells).  ES is normalised by e^-beta (exp(beta*(s-1)));
// every consumer (spreader, interpolator, correction) uses the same form, so
// the product equals the reference's un-normalised kernel up to rounding.
double window_value(const KernelParams &kp, const Window &win, double t) {
    double h = 0.5 * kp.kw;
    if (!(std::fabs(t) < h)) return 0.0;
    if (win.kind == 0) return std::exp(kp.beta * (std::sqrt(1.0 - kp.c * t * t) - 1.0));
    double u = t + h;                       // in [0, kw)
    int d = (int)std::floor(u);
    if (d < 0) d = 0;
    if (d >= kp.kw) d = kp.kw - 1;
    double s = 2.0 * (u - d) - 1.0;         // [-1, 1)
    const double *c = &win.coef[(size_t)d * (win.degree + 1)];
    double v = c[0];
    for (int i = 1; i <= win.degree; ++i) v = v * s + c[i];
    return v;
}

// p = int(2 + 3 kw/2) positive nodes of a 2p-point rule, scaled by kw/2;
// g = (kw/2) * weight * window (deconv.cu:72-86).
int quadrature_terms(const KernelParams &kp, const Window &win, double *xs, double *g) {
    double alpha = kp.kw / 2.0;
    int p = (int)(2 + 3.0 * alpha);
    if (win.kind != 0) p = std::min(2 * p, MAX_QUAD);   // tabulated windows: finer rule
    double z[2 * MAX_QUAD], w[2 * MAX_QUAD];
    gauss_legendre(2 * p, z, w);
    for (int n = 0; n < p; ++n) {
        xs[n] = z[p + n] * alpha;
        g[n] = alpha * w[p + n] * window_value(kp, win, xs[n]);
    }
    return p;
}

// psi1/psi2 on indices 0..nf/2 including the (-1)^k of the half-grid shift
// (deconv.cu:13-24 with N = nf/2 + 1).
void psi_hat_grid(int nf, const KernelParams &kp, const Window &win, std::vector<double> &out) {
    double xs[MAX_QUAD], g[MAX_QUAD];
    int p = quadrature_terms(kp, win, xs, g);
    int N = nf / 2 + 1;
    out.assign(N, 0.0);
    for (int k = 0; k < N; ++k) {
        double s = 0.0;
        for (int i = 0; i < p; ++i) s += g[i] * std::cos((xs[i] - N + 1) / (double)(N - 1) * PI_D * k);
        out[k] = 2 * s;
    }
}

int grid_params(int nx, int ny, double psx, double psy, double wmin, double wmax, double eps,
                double sigma, int sign, GridParams &gp, int kw_override, const GridRequest &req) {
    gp = GridParams();
    if (nx <= 0 || ny <= 0) return ERR_ARG;
    if (!std::isfinite(wmin) || !std::isfinite(wmax) || !std::isfinite(psx) || !std::isfinite(psy))
        return ERR_NONFINITE;
    // explicit oversampled grid (Nifty's nx, ny): both even and at least the
    // image; the oversampling factor of the kernel rule is the smaller ratio
    const bool given = req.grid_x > 0 || req.grid_y > 0;
    if (given) {
        if (req.grid_x < nx || req.grid_y < ny || req.grid_x % 2 || req.grid_y % 2) return ERR_ARG;
        sigma = std::min((double)req.grid_x / nx, (double)req.grid_y / ny);
    }
    int st = setup_kernel(eps, sigma, gp.kp);
    if (st != OK) return st;
    if (kw_override > 0) gp.kp.kw = kw_override;   // tabulated window of another width
    gp.nx = nx;
    gp.ny = ny;
    gp.pixsize_x = psx;
    gp.pixsize_y = psy;
    gp.sign = sign;
    gp.no_w = req.no_w;
    int N1 = ny, N2 = nx;
    if (req.no_w) {
        // w ignored (Nifty's do_wstacking = False): one plane, no n - 1 term,
        // no w phase, no division by n
        gp.nf3 = 1;
        gp.gamma = 1.0;
        gp.h = 0.0;
        gp.nf1 = given ? req.grid_y : get_num_cells(N1, gp.kp);
        gp.nf2 = given ? req.grid_x : get_num_cells(N2, gp.kp);
        if (gp.nf1 < std::max(ny, 2 * gp.kp.kw) || gp.nf2 < std::max(nx, 2 * gp.kp.kw)) return ERR_ARG;
        return OK;
    }
    double l_min = 0 - 0.5 * psx * N2;
    double m_min = 0 - 0.5 * psy * N1;
    double arg = 1.0 - std::pow(l_min, 2) - std::pow(m_min, 2);
    if (!(arg > 0.0)) return ERR_ARG;                // field of view beyond the horizon
    double n_lm = std::sqrt(arg);
    gp.i_center = (wmax + wmin) / 2.0;
    gp.i_half = (wmax - wmin) / 2.0;
    double o_min = n_lm - 1;
    gp.o_center = o_min / 2.0;
    gp.o_half = std::fabs(o_min / 2.0);
    set_nhg_type3(gp.o_half, gp.i_half, gp.kp, gp.nf3, gp.h, gp.gamma);
    gp.nf1 = given ? req.grid_y : get_num_cells(N1, gp.kp);
    gp.nf2 = given ? req.grid_x : get_num_cells(N2, gp.kp);
    if (gp.nf1 < std::max(ny, 2 * gp.kp.kw) || gp.nf2 < std::max(nx, 2 * gp.kp.kw)) return ERR_ARG;
    return OK;
}

// Piecewise polynomial form of the ES window: on each unit interval d of
// [-kw/2, kw/2] a degree-`degree` polynomial in s in [-1,1] interpolating the
// window at Chebyshev points; stored highest power first for Horner.
void es_horner_window(const KernelParams &kp, int degree, Window &win) {
    Window es;
    win.kind = 1;
    win.kw = kp.kw;
    win.degree = degree;
    win.coef.assign((size_t)kp.kw * (degree + 1), 0.0);
    const int n = degree + 1;
    std::vector<double> sn(n), fv(n), a(n), m(n);
    for (int d = 0; d < kp.kw; ++d) {
        for (int j = 0; j < n; ++j) {
            sn[j] = std::cos(PI_D * (j + 0.5) / n);
            double t = (sn[j] + 1.0) * 0.5 + d - 0.5 * kp.kw;
            fv[j] = window_value(kp, es, t);
        }
        // Chebyshev coefficients a_k, then convert sum a_k T_k(s) to monomials.
        for (int k = 0; k < n; ++k) {
            double s = 0;
            for (int j = 0; j < n; ++j) s += fv[j] * std::cos(PI_D * k * (j + 0.5) / n);
            a[k] = s * (k == 0 ? 1.0 : 2.0) / n;
        }
        std::vector<double> tkm1(n, 0.0), tk(n, 0.0), tkp1(n, 0.0);
        std::fill(m.begin(), m.end(), 0.0);
        tkm1[0] = 1.0;                                  // T_0
        if (n > 1) tk[1] = 1.0;                         // T_1
        for (int i = 0; i < n; ++i) m[i] += a[0] * tkm1[i];
        if (n > 1) for (int i = 0; i < n; ++i) m[i] += a[1] * tk[i];
        for (int k = 2; k < n; ++k) {
            std::fill(tkp1.begin(), tkp1.end(), 0.0);
            for (int i = 0; i < n - 1; ++i) tkp1[i + 1] += 2.0 * tk[i];
            for (int i = 0; i < n; ++i) tkp1[i] -= tkm1[i];
            for (int i = 0; i < n; ++i) m[i] += a[k] * tkp1[i];
            tkm1.swap(tk);
            tk.swap(tkp1);
        }
        double *c = &win.coef[(size_t)d * n];
        for (int i = 0; i < n; ++i) c[i] = m[degree - i];
    }
}

}  // namespace curig
