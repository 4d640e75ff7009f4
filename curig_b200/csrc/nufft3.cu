// Generic NUFFT of type 3 in one dimension (nonuniform points to nonuniform
// frequencies):  f_k = sum_j c_j e^{i iflag s_k x_j},  j < m, k < n.
//
// The reference's form (src/fourier/cuft.cu:19-124, 249-424, driven by
// test/nufft_1d_3_1_test.cu and nufft_1d_3_2_test.cu): centres i_c, o_c and
// half widths X, S of the points and frequencies; grid size nf, cell h and
// scale gamma from set_nhg_type3 (contrib/common.cpp:161-195); the strengths
// pre-phased c'_j = c_j e^{i iflag o_c x_j} (pre_stage_1); points rescaled to
// x'_j = (x_j - i_c) / gamma and frequencies to theta_k = (s_k - o_c) gamma h
// (pre_stage_2); c' spread onto the nf-point periodic grid with the ES window;
// the grid's Fourier series evaluated at theta_k; the result divided by the
// window's transform at theta_k (Gauss-Legendre quadrature, as psi3 of the
// gridder) and multiplied by e^{i iflag (s_k - o_c) i_c}.
//
// Where the reference evaluates the grid's series by a direct sum over all nf
// grid points for every frequency (in its test driver), this evaluation is
// this library's own type-2 NUFFT of the grid at the points theta_k (grid
// point m is mode m - nf/2): O(nf log nf + n kw) instead of O(n nf).  Kernels
// wider than 12 (epsilon below about 1e-11) keep the direct sum.
#include "plan.h"

#include "../../include/curig.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

namespace curig {

struct Nufft3 {
    int iflag = 1, precision = 0;
    double eps = 1e-6, sigma = 2.0;
    cudaStream_t st = nullptr;
    long long m = 0, n = 0;
    int nf = 0;
    KernelParams kp;
    double i_c = 0, o_c = 0, X = 0, S = 0, gamma = 1, h = 0;
    double *d_xp = nullptr, *d_theta = nullptr;        // rescaled points / frequencies
    double2 *d_pre = nullptr, *d_post = nullptr;       // e^{i iflag o_c x_j}; e^{i iflag t_k i_c} / psi(theta_k)
    double *d_quad = nullptr;
    unsigned long long *d_keys = nullptr;
    int *d_err = nullptr;
    void *d_grid = nullptr, *d_F = nullptr;            // nf-point grid; its series at theta_k
    curig_nufft inner = nullptr;                       // type 2 on the grid
};

__global__ void k_t3_points(long long m, const double *__restrict__ x, double ic, double gamma, double oc,
                            int iflag, double *__restrict__ xp, double2 *__restrict__ pre) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < m;
         j += (long long)gridDim.x * blockDim.x) {
        const double xj = x[j];
        xp[j] = (xj - ic) / gamma;                     // pre_stage_2 (cuft.cu:53-72)
        double sn, cs;
        sincos(oc * xj * iflag, &sn, &cs);             // pre_stage_1 (cuft.cu:19-39)
        pre[j] = make_double2(cs, sn);
    }
}

// theta_k and the per-frequency factor e^{i iflag (s_k - o_c) i_c} / psi(theta_k),
// psi(theta) = 2 sum_q g_q cos(theta x_q) (the window's transform at theta
// radians per cell).
__global__ void k_t3_targets(long long n, const double *__restrict__ s, double oc, double gamma, double h, double ic,
                             int iflag, int nq, const double *__restrict__ qx, const double *__restrict__ qg,
                             double *__restrict__ theta, double2 *__restrict__ post) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const double t = s[k] - oc;
        const double th = t * gamma * h;               // pre_stage_2 of the frequencies
        theta[k] = th;
        double psi = 0.0;
        for (int q = 0; q < nq; ++q) psi += qg[q] * cos(th * qx[q]);
        psi *= 2.0;
        double sn, cs;
        sincos(t * ic * iflag, &sn, &cs);
        post[k] = make_double2(cs / psi, sn / psi);
    }
}

// One thread per point: kw taps of the ES window onto the periodic grid
// (grid point m at angle (m - nf/2) * 2 pi / nf), global atomics.
template <typename T>
__global__ void k_t3_spread(long long m, const double *__restrict__ xp, const double2 *__restrict__ pre,
                            const typename cplx_t<T>::type *__restrict__ c, int nf, int kw, double beta, double cc,
                            typename cplx_t<T>::type *__restrict__ grid) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < m;
         j += (long long)gridDim.x * blockDim.x) {
        const double g = (xp[j] * INV_2PI + 0.5) * nf;
        const double st = ceil(g - 0.5 * kw);
        const double2 p = pre[j];
        const double cr = (double)c[j].x * p.x - (double)c[j].y * p.y;
        const double ci = (double)c[j].x * p.y + (double)c[j].y * p.x;
        long long i0 = (long long)st;
        i0 %= nf;
        if (i0 < 0) i0 += nf;
        for (int d = 0; d < kw; ++d) {
            const double t = st + d - g;
            const double a = 1.0 - cc * t * t;
            const double w = a > 0.0 ? exp(beta * (sqrt(a) - 1.0)) : 0.0;
            long long idx = i0 + d;
            if (idx >= nf) idx -= nf;
            atomicAdd(&grid[idx].x, (T)(cr * w));
            atomicAdd(&grid[idx].y, (T)(ci * w));
        }
    }
}

// The grid's series by direct summation (tolerances that need kernels wider
// than the type-2 NUFFT's tile kernels take): thread per frequency, the phase
// e^{i iflag theta (m - nf/2)} advanced by one rotation per grid point and
// taken afresh from sincos every 64 points.
template <typename T>
__global__ void k_t3_direct(long long n, const double *__restrict__ theta, int iflag, int nf,
                            const typename cplx_t<T>::type *__restrict__ grid, typename cplx_t<T>::type *__restrict__ F) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const double th = theta[k] * iflag;
        double sr, cr;
        sincos(th, &sr, &cr);
        double ar = 0.0, ai = 0.0, er = 0.0, ei = 0.0;
        for (int m = 0; m < nf; ++m) {
            if ((m & 63) == 0) sincos(th * (double)(m - nf / 2), &ei, &er);
            const double gr = grid[m].x, gi = grid[m].y;
            ar += gr * er - gi * ei;
            ai += gr * ei + gi * er;
            const double nr = er * cr - ei * sr;
            ei = er * sr + ei * cr;
            er = nr;
        }
        F[k].x = (T)ar;
        F[k].y = (T)ai;
    }
}

template <typename T>
__global__ void k_t3_finish(long long n, const double2 *__restrict__ post, const typename cplx_t<T>::type *__restrict__ F,
                            typename cplx_t<T>::type *__restrict__ f) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const double2 q = post[k];
        const double fr = F[k].x, fi = F[k].y;
        f[k].x = (T)(fr * q.x - fi * q.y);
        f[k].y = (T)(fr * q.y + fi * q.x);
    }
}

static int grid_blocks(long long n) { return (int)std::max(1LL, std::min((n + 255) / 256, 148LL * 32)); }

static void nufft3_free_points(Nufft3 *p) {
    for (void **b : {(void **)&p->d_xp, (void **)&p->d_theta, (void **)&p->d_pre, (void **)&p->d_post,
                     (void **)&p->d_quad, (void **)&p->d_keys, (void **)&p->d_err, &p->d_grid, &p->d_F})
        if (*b) {
            cudaFreeAsync(*b, p->st);
            *b = nullptr;
        }
    if (p->inner) {
        curig_nufft_destroy(p->inner);
        p->inner = nullptr;
    }
}

Nufft3 *nufft3_create(int iflag, double eps, double sigma, int precision, cudaStream_t st) {
    Nufft3 *p = new Nufft3();
    p->iflag = iflag >= 0 ? 1 : -1;
    p->eps = eps;
    p->sigma = sigma;
    p->precision = precision;
    p->st = st;
    return p;
}

void nufft3_destroy(Nufft3 *p) {
    if (!p) return;
    nufft3_free_points(p);
    cudaStreamSynchronize(p->st);
    delete p;
}

static double key_value(unsigned long long k) {
    unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
    double d;
    std::memcpy(&d, &b, 8);
    return d;
}

// min / max of n device doubles (launch_wrange), synchronising.
static int range_of(Nufft3 *p, const double *d, long long n, double &lo, double &hi) {
    unsigned long long hk[2] = {ULLONG_MAX, 0ULL};
    int herr = 0;
    if (cudaMemcpyAsync(p->d_keys, hk, sizeof(hk), cudaMemcpyHostToDevice, p->st) != cudaSuccess ||
        cudaMemsetAsync(p->d_err, 0, sizeof(int), p->st) != cudaSuccess)
        return ERR_CUDA;
    launch_wrange(d, 1, n, p->d_keys, p->d_err, p->st);
    if (cudaMemcpyAsync(hk, p->d_keys, sizeof(hk), cudaMemcpyDeviceToHost, p->st) != cudaSuccess ||
        cudaMemcpyAsync(&herr, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, p->st) != cudaSuccess ||
        cudaStreamSynchronize(p->st) != cudaSuccess)
        return ERR_CUDA;
    if (herr & EF_NONFINITE) return ERR_NONFINITE;
    lo = key_value(hk[0]);
    hi = key_value(hk[1]);
    return OK;
}

int nufft3_setpts(Nufft3 *p, long long m, const double *d_x, long long n, const double *d_s,
                  const ::curig_opts *opts) {
    if (!p || m <= 0 || n <= 0 || !d_x || !d_s || m >= INT_MAX || n >= INT_MAX) return ERR_ARG;
    nufft3_free_points(p);
    int s = setup_kernel(p->eps, p->sigma, p->kp);
    if (s != OK) return s;
    p->m = m;
    p->n = n;
    const size_t esz = p->precision ? 8 : 16;
    if (alloc_async((void **)&p->d_keys, 2 * sizeof(unsigned long long), p->st) != cudaSuccess ||
        alloc_async((void **)&p->d_err, sizeof(int), p->st) != cudaSuccess)
        return ERR_NOMEM;
    double xlo, xhi, slo, shi;
    if ((s = range_of(p, d_x, m, xlo, xhi)) || (s = range_of(p, d_s, n, slo, shi))) return s;
    p->i_c = (xhi + xlo) / 2.0;                          // cuft.cu:330-333
    p->X = (xhi - xlo) / 2.0;
    p->o_c = (shi + slo) / 2.0;
    p->S = (shi - slo) / 2.0;
    set_nhg_type3(p->S, p->X, p->kp, p->nf, p->h, p->gamma);
    if (p->nf <= 0 || p->nf >= (1 << 30)) return ERR_UNSUPPORTED;
    double qx[MAX_QUAD], qg[MAX_QUAD];
    const int nq = quadrature_terms(p->kp, Window(), qx, qg);
    if (alloc_async((void **)&p->d_xp, m * sizeof(double), p->st) != cudaSuccess ||
        alloc_async((void **)&p->d_pre, m * sizeof(double2), p->st) != cudaSuccess ||
        alloc_async((void **)&p->d_theta, n * sizeof(double), p->st) != cudaSuccess ||
        alloc_async((void **)&p->d_post, n * sizeof(double2), p->st) != cudaSuccess ||
        alloc_async((void **)&p->d_quad, 2 * MAX_QUAD * sizeof(double), p->st) != cudaSuccess ||
        alloc_async(&p->d_grid, (size_t)p->nf * esz, p->st) != cudaSuccess ||
        alloc_async(&p->d_F, n * esz, p->st) != cudaSuccess)
        return ERR_NOMEM;
    if (cudaMemcpyAsync(p->d_quad, qx, nq * sizeof(double), cudaMemcpyHostToDevice, p->st) != cudaSuccess ||
        cudaMemcpyAsync(p->d_quad + MAX_QUAD, qg, nq * sizeof(double), cudaMemcpyHostToDevice, p->st) != cudaSuccess)
        return ERR_CUDA;
    count_launch(2);
    k_t3_points<<<grid_blocks(m), 256, 0, p->st>>>(m, d_x, p->i_c, p->gamma, p->o_c, p->iflag, p->d_xp, p->d_pre);
    k_t3_targets<<<grid_blocks(n), 256, 0, p->st>>>(n, d_s, p->o_c, p->gamma, p->h, p->i_c, p->iflag, nq, p->d_quad,
                                                    p->d_quad + MAX_QUAD, p->d_theta, p->d_post);
    // the grid's Fourier series at theta_k: a type-2 NUFFT with nf modes (its
    // tile kernels take widths up to 12; beyond, direct summation)
    if (p->kp.kw > TAB_KW) return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA;
    curig_opts o;
    curig_default_opts(&o);
    if (opts) o = *opts;
    o.stream = p->st;
    o.precision = p->precision;
    if ((s = curig_nufft_makeplan(2, 1, p->nf, 1, p->eps, p->iflag, p->sigma, &o, &p->inner)) != OK) return s;
    if ((s = curig_nufft_setpts(p->inner, n, p->d_theta, nullptr)) != OK) return s;
    return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA;
}

int nufft3_execute(Nufft3 *p, const void *d_c, void *d_f) {
    if (!p || !p->d_grid || !d_c || !d_f) return ERR_ARG;
    const size_t esz = p->precision ? 8 : 16;
    if (cudaMemsetAsync(p->d_grid, 0, (size_t)p->nf * esz, p->st) != cudaSuccess) return ERR_CUDA;
    count_launch(2);
    if (p->precision) {
        k_t3_spread<float><<<grid_blocks(p->m), 256, 0, p->st>>>(p->m, p->d_xp, p->d_pre,
                                                                static_cast<const float2 *>(d_c), p->nf, p->kp.kw,
                                                                p->kp.beta, p->kp.c, static_cast<float2 *>(p->d_grid));
    } else {
        k_t3_spread<double><<<grid_blocks(p->m), 256, 0, p->st>>>(p->m, p->d_xp, p->d_pre,
                                                                 static_cast<const double2 *>(d_c), p->nf, p->kp.kw,
                                                                 p->kp.beta, p->kp.c, static_cast<double2 *>(p->d_grid));
    }
    if (p->inner) {
        int s = curig_nufft_execute(p->inner, p->d_F, p->d_grid);
        if (s != OK) return s;
    } else {
        count_launch();
        if (p->precision)
            k_t3_direct<float><<<grid_blocks(p->n), 256, 0, p->st>>>(p->n, p->d_theta, p->iflag, p->nf,
                                                                    static_cast<const float2 *>(p->d_grid),
                                                                    static_cast<float2 *>(p->d_F));
        else
            k_t3_direct<double><<<grid_blocks(p->n), 256, 0, p->st>>>(p->n, p->d_theta, p->iflag, p->nf,
                                                                     static_cast<const double2 *>(p->d_grid),
                                                                     static_cast<double2 *>(p->d_F));
    }
    if (p->precision)
        k_t3_finish<float><<<grid_blocks(p->n), 256, 0, p->st>>>(p->n, p->d_post, static_cast<const float2 *>(p->d_F),
                                                                static_cast<float2 *>(d_f));
    else
        k_t3_finish<double><<<grid_blocks(p->n), 256, 0, p->st>>>(p->n, p->d_post, static_cast<const double2 *>(p->d_F),
                                                                 static_cast<double2 *>(d_f));
    return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA;
}

void nufft3_info(const Nufft3 *p, int *nf, double *dinfo) {
    if (nf) *nf = p->nf;
    if (dinfo) {
        dinfo[0] = p->i_c; dinfo[1] = p->X; dinfo[2] = p->o_c; dinfo[3] = p->S; dinfo[4] = p->gamma; dinfo[5] = p->h;
    }
}

}  // namespace curig
