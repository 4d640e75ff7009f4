#define _GNU_SOURCE
/*
 * Oracle: FP64 explicit (direct) Fourier transforms for ms2dirty / dirty2ms.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker, never the product.  Built into
 * oracle/_build/liboracle_dft.so by oracle/build.py and loaded only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 *
 * Restates the reference's own truth computations:
 *   gridder   python/curagridder/test_wst.py:15-32  (explicit_gridder, before .real)
 *             src/astro/precomp.cu:242-275          (explicit_gridder kernel)
 *   degridder python/curagridder/explicit_test.py:32-54 (explicit_degridder)
 *
 * Conventions (those of the reference library, src/astro/ra_exec.cu:22-37):
 *   dirty is [nx][ny] row-major; pixel (ix, iy) sits at
 *   l = (ix - nx/2) * pixsize_x, m = (iy - ny/2) * pixsize_y (integer halves);
 *   n - 1 = -(l^2+m^2) / (sqrt(1 - l^2 - m^2) + 1)   (test_wst.py:22-24);
 *   phase = f/c * (l*u + m*v + sign*w*(n-1));
 *   ms2dirty:  dirty = sum_j wgt_j vis_j exp(+2 pi i phase) / n
 *   dirty2ms:  vis_j = wgt_j * sum_pix dirty/n * exp(-2 pi i phase)
 * vis / wgt are [nrow][nchan]; wgt may be NULL.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stddef.h>

#define SPEEDOFLIGHT 299792458.0

static void pix_lmn(int64_t p, int nx, int ny, double psx, double psy,
                    double *l, double *m, double *nm1, double *n)
{
    int64_t ix = p / ny, iy = p % ny;
    double x = (double)(ix - nx / 2) * psx;
    double y = (double)(iy - ny / 2) * psy;
    double e = x * x + y * y;
    *l = x;
    *m = y;
    *nm1 = -e / (sqrt(1.0 - e) + 1.0);
    *n = *nm1 + 1.0;
}

/* dirty[p] for the npix pixels listed in pix (or all nx*ny pixels if pix == NULL). */
void oracle_ms2dirty_dft(int64_t nrow, int nchan, int nx, int ny, double psx, double psy,
                         const double *freq, const double *uvw,
                         const double complex *vis, const double *wgt, int sign,
                         int64_t npix, const int64_t *pix, double complex *out)
{
    if (pix == NULL) npix = (int64_t)nx * ny;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < npix; ++t) {
        int64_t p = pix ? pix[t] : t;
        double l, m, nm1, n;
        pix_lmn(p, nx, ny, psx, psy, &l, &m, &nm1, &n);
        double sr = 0.0, si = 0.0;
        for (int64_t r = 0; r < nrow; ++r) {
            double u = uvw[3 * r], v = uvw[3 * r + 1], w = uvw[3 * r + 2];
            double base = l * u + m * v + sign * w * nm1;
            for (int c = 0; c < nchan; ++c) {
                double ph = 2.0 * M_PI * (freq[c] / SPEEDOFLIGHT * base);
                double s, co;
                sincos(ph, &s, &co);
                double complex z = vis[r * nchan + c];
                double wt = wgt ? wgt[r * nchan + c] : 1.0;
                double zr = creal(z) * wt, zi = cimag(z) * wt;
                sr += zr * co - zi * s;
                si += zr * s + zi * co;
            }
        }
        out[t] = (sr + I * si) / n;
    }
}

/* vis[j] for the nvis (row, chan) pairs listed in idx (flat r*nchan+c), or all. */
void oracle_dirty2ms_dft(int64_t nrow, int nchan, int nx, int ny, double psx, double psy,
                         const double *freq, const double *uvw,
                         const double complex *dirty, const double *wgt, int sign,
                         int64_t nvis, const int64_t *idx, double complex *out)
{
    if (idx == NULL) nvis = nrow * nchan;
    const int64_t npix = (int64_t)nx * ny;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t t = 0; t < nvis; ++t) {
        int64_t j = idx ? idx[t] : t;
        int64_t r = j / nchan;
        int c = (int)(j % nchan);
        double u = uvw[3 * r], v = uvw[3 * r + 1], w = uvw[3 * r + 2];
        double foc = freq[c] / SPEEDOFLIGHT;
        double sr = 0.0, si = 0.0;
        for (int64_t p = 0; p < npix; ++p) {
            double l, m, nm1, n;
            pix_lmn(p, nx, ny, psx, psy, &l, &m, &nm1, &n);
            double ph = -2.0 * M_PI * (foc * (l * u + m * v + sign * w * nm1));
            double s, co;
            sincos(ph, &s, &co);
            double complex d = dirty[p];
            double dr = creal(d) / n, di = cimag(d) / n;
            sr += dr * co - di * s;
            si += dr * s + di * co;
        }
        double wt = wgt ? wgt[j] : 1.0;
        out[t] = (sr + I * si) * wt;
    }
}
