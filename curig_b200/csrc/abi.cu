// Exported entry points of libcurafft.so: the reference's C ABI
// (src/astro/cugridder.cu:330-612), the multi-channel / FP32 one-shot calls,
// the device-pointer plan API and the C++ gridder_* mirror.
#include "plan.h"

#include "../../include/curig.h"
#include "../../include/cugridder.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

using namespace curig;

static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

static Options to_options(const curig_opts *o) {
    Options opt;
    if (o) {
        opt.precision = o->precision;
        opt.window = o->window;
        opt.bin_xy = o->bin_xy;
        opt.sub = o->sub;
        opt.smem_budget = o->smem_budget > 0 ? (size_t)o->smem_budget : 0;
        opt.stream = (cudaStream_t)o->stream;
        opt.smode = o->accumulate;
        opt.w_term = o->w_term;
        opt.grid_x = o->grid_x;
        opt.grid_y = o->grid_y;
        opt.bin_z = o->bin_z;
        opt.sparse = o->sparse;
    }
    return opt;
}

extern "C" void curig_default_opts(curig_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
}

extern "C" const char *curig_last_error(void) { return g_last_error.c_str(); }

extern "C" int curig_release_memory(void) {
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
        cudaMemPoolTrimTo(pool, 0) != cudaSuccess)
        return fail(ERR_CUDA, "memory pool trim failed");
    fft_cache_trim();
    return OK;
}

// One call with host buffers: allocate, copy in, plan, execute, copy out, free
// (the reference's ms2dirty_exec / dirty2ms_exec life cycle, cugridder.cu:330-582),
// pipelined over row slabs.  A copy stream uploads uvw first (set points needs
// it, and the w range it yields sizes the planes that the image's correction
// fills), then for dirty2ms the image, then each slab's visibilities /
// weights with an event per slab; the plan's stream spreads slab k as soon as
// it is on the device (ms2dirty), or interpolates slab k and a download stream
// returns its rows while slab k+1 is interpolated (dirty2ms).  With pinned
// host buffers the transfers in both directions overlap the kernels.
static int oneshot(int type, long long nrow, int nchan, int nx, int ny, double psx, double psy,
                   const double *freq, const double *uvw, void *vis, const void *wgt, void *dirty,
                   double eps, double sigma, int sign, const curig_opts *opts) {
    if (nrow < 0 || nchan <= 0 || nx <= 0 || ny <= 0 || !freq || !dirty || (nrow > 0 && (!uvw || !vis)))
        return fail(ERR_ARG, "invalid argument");
    if (opts && (opts->slabs < 0 || opts->slabs > MAX_SLABS)) return fail(ERR_ARG, "slabs outside 0 .. 8");
    if (nrow == 0) {                      // no visibilities: empty sum / nothing to degrid
        if (type == 1) std::memset(dirty, 0, (size_t)nx * ny * 2 * (opts && opts->precision ? 4 : 8));
        return OK;
    }
    Options opt = to_options(opts);
    cudaStream_t st = opt.stream ? opt.stream : cudaStreamPerThread;
    opt.stream = st;
    const size_t rs = opt.precision ? 4 : 8, cs = 2 * rs;
    const size_t M = (size_t)nrow * nchan, npix = (size_t)nx * ny;
    const size_t row_bytes = (size_t)nchan * (cs + (wgt ? rs : 0));
    // automatic: 3 slabs from 1 GiB of visibilities + weights, 2 from 384 MiB.
    // Slabs overlap the transfers with the tile kernels but split every bin
    // (more chunks and tile loads).  ms2dirty + dirty2ms at 4096^2 with 1e7
    // rows, 1 / 2 / 3 slabs: FP32 16 channels (1.9 GB) 137.0 / 119.5 / 113.5 ms,
    // FP32 4 channels (480 MB) 64.0 / 61.7 / 64.9 ms, FP64 1 channel (240 MB,
    // the reference ABI's call) 93.5 / 106.5 / 116.5 ms.
    const size_t up_bytes = (size_t)nrow * row_bytes;
    int nslab = opts && opts->slabs > 0 ? opts->slabs
                                        : up_bytes >= ((size_t)1 << 30) ? 3 : up_bytes >= ((size_t)384 << 20) ? 2 : 1;
    if (nslab > nrow) nslab = (int)nrow;
    opt.slabs = nslab;
    double *d_uvw = nullptr;
    void *d_vis = nullptr, *d_wgt = nullptr, *d_dirty = nullptr;
    Plan *p = nullptr;
    int s = OK;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && s == OK) {
            s = e == cudaErrorMemoryAllocation ? ERR_NOMEM : ERR_CUDA;
            g_last_error = cudaGetErrorString(e);
        }
        return s == OK;
    };
    cudaStream_t cp = nullptr, dn = nullptr, bn = nullptr;   // uploads, downloads, dirty2ms binning
    cudaEvent_t ev_alloc = nullptr, ev_uvw = nullptr, ev_img = nullptr, ev_geom = nullptr, ev_bin = nullptr;
    cudaEvent_t ev_ready[MAX_SLABS] = {}, ev_done[MAX_SLABS] = {};
    bool ok = chk(cudaStreamCreateWithFlags(&cp, cudaStreamNonBlocking)) &&
              chk(cudaStreamCreateWithFlags(&dn, cudaStreamNonBlocking)) &&
              chk(cudaStreamCreateWithFlags(&bn, cudaStreamNonBlocking)) &&
              chk(cudaEventCreateWithFlags(&ev_geom, cudaEventDisableTiming)) &&
              chk(cudaEventCreateWithFlags(&ev_bin, cudaEventDisableTiming)) &&
              chk(cudaEventCreateWithFlags(&ev_alloc, cudaEventDisableTiming)) &&
              chk(cudaEventCreateWithFlags(&ev_uvw, cudaEventDisableTiming)) &&
              chk(cudaEventCreateWithFlags(&ev_img, cudaEventDisableTiming));
    for (int k = 0; ok && k < nslab; ++k)
        ok = chk(cudaEventCreateWithFlags(&ev_ready[k], cudaEventDisableTiming)) &&
             chk(cudaEventCreateWithFlags(&ev_done[k], cudaEventDisableTiming));
    ok = ok && chk(alloc_async((void **)&d_uvw, 3 * nrow * sizeof(double), st)) &&
         chk(alloc_async(&d_vis, M * cs, st)) && (!wgt || chk(alloc_async(&d_wgt, M * rs, st))) &&
         chk(alloc_async(&d_dirty, npix * cs, st)) && chk(cudaEventRecord(ev_alloc, st)) &&
         chk(cudaStreamWaitEvent(cp, ev_alloc, 0)) &&
         chk(cudaMemcpyAsync(d_uvw, uvw, 3 * nrow * sizeof(double), cudaMemcpyHostToDevice, cp)) &&
         chk(cudaEventRecord(ev_uvw, cp)) &&
         (type != 2 || chk(cudaMemcpyAsync(d_dirty, dirty, npix * cs, cudaMemcpyHostToDevice, cp))) &&
         chk(cudaEventRecord(ev_img, cp));
    for (int k = 0; ok && k < nslab; ++k) {          // slab k: rows [r0, r1)
        const long long r0 = slab_first_row(nrow, nslab, k), r1 = slab_first_row(nrow, nslab, k + 1);
        const size_t e0 = (size_t)r0 * nchan, ne = (size_t)(r1 - r0) * nchan;
        ok = (type != 1 || chk(cudaMemcpyAsync(static_cast<char *>(d_vis) + e0 * cs,
                                               static_cast<const char *>(vis) + e0 * cs, ne * cs,
                                               cudaMemcpyHostToDevice, cp))) &&
             (!wgt || chk(cudaMemcpyAsync(static_cast<char *>(d_wgt) + e0 * rs,
                                          static_cast<const char *>(wgt) + e0 * rs, ne * rs,
                                          cudaMemcpyHostToDevice, cp))) &&
             chk(cudaEventRecord(ev_ready[k], cp));
    }
    if (ok) {
        s = plan_create(type, nx, ny, psx, psy, eps, sigma, sign, opt, &p);
        if (s == OK && !chk(cudaStreamWaitEvent(st, ev_uvw, 0))) s = ERR_CUDA;
        if (s == OK) s = plan_setpts_geometry(p, nrow, nchan, d_uvw, d_uvw + 1, d_uvw + 2, 3, freq);
        if (s == OK && type == 1) {
            s = plan_setpts_bin(p, st);
        } else if (s == OK) {
            // dirty2ms: the grid preparation (plan's stream) runs while a second
            // stream bins the visibilities; neither depends on the other
            if (!chk(cudaEventRecord(ev_geom, st)) || !chk(cudaStreamWaitEvent(bn, ev_geom, 0)))
                s = ERR_CUDA;
            if (s == OK) s = plan_d2m_prologue(p, d_dirty, ev_img);
            if (s == OK) s = plan_setpts_bin(p, bn);
            if (s == OK && (!chk(cudaEventRecord(ev_bin, bn)) || !chk(cudaStreamWaitEvent(st, ev_bin, 0))))
                s = ERR_CUDA;
        }
        if (s == OK && !chk(cudaStreamWaitEvent(st, ev_img, 0))) s = ERR_CUDA;
        if (s == OK)
            s = plan_execute_slabs(p, type, d_vis, d_wgt, d_dirty, ev_ready, type == 2 ? ev_done : nullptr, nslab,
                                   type == 2);
        if (s == OK) {
            if (type == 1) {
                chk(cudaMemcpyAsync(dirty, d_dirty, npix * cs, cudaMemcpyDeviceToHost, st));
            } else {
                for (int k = 0; s == OK && k < nslab; ++k) {
                    const long long r0 = slab_first_row(nrow, nslab, k), r1 = slab_first_row(nrow, nslab, k + 1);
                    const size_t e0 = (size_t)r0 * nchan, ne = (size_t)(r1 - r0) * nchan;
                    if (chk(cudaStreamWaitEvent(dn, ev_done[k], 0)))
                        chk(cudaMemcpyAsync(static_cast<char *>(vis) + e0 * cs,
                                            static_cast<const char *>(d_vis) + e0 * cs, ne * cs,
                                            cudaMemcpyDeviceToHost, dn));
                }
            }
        }
        if (s == OK) s = plan_device_status(p);   // flags raised by kernels (synchronises)
        if (p && s != OK && !p->last_error.empty()) g_last_error = p->last_error;
    }
    // nothing is freed while a transfer may still run
    for (cudaStream_t x : {cp, dn, bn})
        if (x) cudaStreamSynchronize(x);
    if (p) plan_destroy(p);
    for (cudaStream_t x : {cp, dn, bn})
        if (x) cudaStreamDestroy(x);
    for (cudaEvent_t e : {ev_alloc, ev_uvw, ev_img, ev_geom, ev_bin})
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < MAX_SLABS; ++k) {
        if (ev_ready[k]) cudaEventDestroy(ev_ready[k]);
        if (ev_done[k]) cudaEventDestroy(ev_done[k]);
    }
    if (d_uvw) cudaFreeAsync(d_uvw, st);
    if (d_vis) cudaFreeAsync(d_vis, st);
    if (d_wgt) cudaFreeAsync(d_wgt, st);
    if (d_dirty) cudaFreeAsync(d_dirty, st);
    chk(cudaStreamSynchronize(st));
    return s;
}

static void ref_pixsizes(double fov, int nx, int ny, double &psx, double &psy) {
    const double PI = PI_D;                       // (PCS)M_PI, include/utils.h:97
    psx = fov / 180.0 * PI / (double)nx;          // cugridder.cu:48
    psy = fov / 180.0 * PI / (double)ny;          // cugridder.cu:49
}

extern "C" int ms2dirty_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
                          curig_cdouble *vis, double *wgt, curig_cdouble *dirty, double epsilon,
                          double sigma, int sign) {
    double psx, psy;
    ref_pixsizes(fov, nxdirty, nydirty, psx, psy);
    return oneshot(1, nrow, 1, nxdirty, nydirty, psx, psy, &freq, uvw, vis, wgt, dirty, epsilon, sigma,
                   sign, nullptr);
}

extern "C" int ms2dirty_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
                          curig_cdouble *vis, curig_cdouble *dirty, double epsilon, double sigma,
                          int sign) {
    return ms2dirty_2(nrow, nxdirty, nydirty, fov, freq, uvw, vis, nullptr, dirty, epsilon, sigma, sign);
}

extern "C" int dirty2ms_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
                          curig_cdouble *vis, double *wgt, curig_cdouble *dirty, double epsilon,
                          double sigma, int sign) {
    double psx, psy;
    ref_pixsizes(fov, nxdirty, nydirty, psx, psy);
    return oneshot(2, nrow, 1, nxdirty, nydirty, psx, psy, &freq, uvw, vis, wgt, dirty, epsilon, sigma,
                   sign, nullptr);
}

extern "C" int dirty2ms_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
                          curig_cdouble *vis, curig_cdouble *dirty, double epsilon, double sigma,
                          int sign) {
    return dirty2ms_2(nrow, nxdirty, nydirty, fov, freq, uvw, vis, nullptr, dirty, epsilon, sigma, sign);
}

extern "C" int curig_ms2dirty(int64_t nrow, int nchan, int nx, int ny, double psx, double psy,
                              const double *freq, const double *uvw, const void *vis, const void *wgt,
                              void *dirty, double eps, double sigma, int sign, const curig_opts *opts) {
    return oneshot(1, nrow, nchan, nx, ny, psx, psy, freq, uvw, const_cast<void *>(vis), wgt, dirty, eps,
                   sigma, sign, opts);
}

extern "C" int curig_dirty2ms(int64_t nrow, int nchan, int nx, int ny, double psx, double psy,
                              const double *freq, const double *uvw, void *vis, const void *wgt,
                              const void *dirty, double eps, double sigma, int sign,
                              const curig_opts *opts) {
    return oneshot(2, nrow, nchan, nx, ny, psx, psy, freq, uvw, vis, wgt, const_cast<void *>(dirty), eps,
                   sigma, sign, opts);
}

// ------------------------------------------------------------------ plan API
struct curig_plan_s {
    Plan *p;
};

extern "C" int curig_makeplan(int type, int nx, int ny, double psx, double psy, double eps, double sigma,
                              int sign, const curig_opts *opts, curig_plan *out) {
    if (!out) return fail(ERR_ARG, "null plan pointer");
    *out = nullptr;
    Plan *p = nullptr;
    int s = plan_create(type, nx, ny, psx, psy, eps, sigma, sign, to_options(opts), &p);
    if (s != OK) return fail(s, "plan creation failed");
    *out = new curig_plan_s{p};
    return OK;
}

// ------------------------------------------------------------------ generic NUFFT
// Type 1 (points -> modes) and type 2 (modes -> points) in one or two
// dimensions on the w-free gridder: a point (x, y) becomes the row
// (s x / 2pi, s y / 2pi, 0) at frequency c with unit pixel sizes, so the
// gridder's phases e^{+-i 2pi (l u + m v)} are e^{+-i (k1 x + k2 y)}; s = +iflag
// for type 1 (ms2dirty's sign) and -iflag for type 2 (dirty2ms's).  Modes are
// [n1][n2] with mode k = index - n/2, as the dirty image.  Plays the part of
// the reference's cunufft_setting / cunufft exec path (cuft.cu:249) for types
// 1 and 2 with the same kernel-width, grid-size and correction rules.
struct curig_nufft_s {
    Plan *p = nullptr;
    Nufft3 *t3 = nullptr;                 // type 3
    curig_opts opts{};
    int type = 1, dim = 1, n1 = 0, n2 = 1, n3 = 1, iflag = 1;
    double *d_uvw = nullptr;
    const double *d_z = nullptr;          // 3-D: the third coordinate, for setpts
};

extern "C" int curig_nufft_makeplan(int type, int dim, int n1, int n2, double eps, int iflag, double sigma,
                                    const curig_opts *opts, curig_nufft *out) {
    if (!out) return fail(ERR_ARG, "null plan pointer");
    *out = nullptr;
    if ((type != 1 && type != 2 && type != 3) || (dim != 1 && dim != 2) || (type == 3 && dim != 1) || n1 <= 0 ||
        (dim == 2 && n2 <= 0) || (iflag != 1 && iflag != -1))
        return fail(ERR_ARG, "invalid NUFFT plan arguments");
    if (type == 3) {                                   // sizes come with the points (curig_nufft_setpts3)
        KernelParams kp;
        int st = setup_kernel(eps, sigma, kp);
        if (st != OK) return fail(st, "invalid NUFFT tolerance or upsampling factor");
        if (opts && opts->precision != 0 && opts->precision != 1) return fail(ERR_ARG, "invalid precision");
        *out = new curig_nufft_s;
        (*out)->type = 3;
        (*out)->dim = 1;
        (*out)->n1 = n1;
        (*out)->iflag = iflag;
        if (opts) (*out)->opts = *opts;
        else curig_default_opts(&(*out)->opts);
        (*out)->t3 = nufft3_create(iflag, eps, sigma, (*out)->opts.precision, (cudaStream_t)(*out)->opts.stream);
        return OK;
    }
    Options o = to_options(opts);
    o.w_term = 1;
    Plan *p = nullptr;
    const int ny = dim == 2 ? n2 : 1;
    int s = plan_create(type, n1, ny, 1.0, 1.0, eps, sigma, 1, o, &p);
    if (s != OK) return fail(s, "NUFFT plan creation failed");
    *out = new curig_nufft_s;
    (*out)->p = p;
    (*out)->type = type;
    (*out)->dim = dim;
    (*out)->n1 = n1;
    (*out)->n2 = ny;
    (*out)->iflag = iflag;
    return OK;
}

// Generic 3-D NUFFT of types 1 and 2: the w-free gridder with a periodic third
// axis of the NUFFT's own grid size (opts n3): a point (x, y, z) becomes the
// row s (x, y, z) / 2pi at frequency c, and the third axis is transformed and
// corrected like the first two (k_correct3_m2d / k_correct3_d2m).  Modes
// [n1][n2][n3], mode k = index - n/2 on every axis.
extern "C" int curig_nufft3d_makeplan(int type, int n1, int n2, int n3, double eps, int iflag, double sigma,
                                      const curig_opts *opts, curig_nufft *out) {
    if (!out) return fail(ERR_ARG, "null plan pointer");
    *out = nullptr;
    if ((type != 1 && type != 2) || n1 <= 0 || n2 <= 0 || n3 <= 0 || (iflag != 1 && iflag != -1))
        return fail(ERR_ARG, "invalid 3-D NUFFT plan arguments");
    Options o = to_options(opts);
    o.w_term = 0;
    o.n3 = n3;
    Plan *p = nullptr;
    int s = plan_create(type, n1, n2, 1.0, 1.0, eps, sigma, 1, o, &p);
    if (s != OK) return fail(s, "3-D NUFFT plan creation failed");
    *out = new curig_nufft_s;
    (*out)->p = p;
    (*out)->type = type;
    (*out)->dim = 3;
    (*out)->n1 = n1;
    (*out)->n2 = n2;
    (*out)->n3 = n3;
    (*out)->iflag = iflag;
    return OK;
}

extern "C" int curig_nufft3d_setpts(curig_nufft h, int64_t m, const double *d_x, const double *d_y,
                                    const double *d_z) {
    if (!h || h->dim != 3 || !d_y || !d_z) return fail(ERR_ARG, "not a 3-D plan, or missing coordinates");
    h->d_z = d_z;
    return curig_nufft_setpts(h, m, d_x, d_y);
}

extern "C" int curig_nufft_setpts3(curig_nufft h, int64_t m, const double *d_x, int64_t n, const double *d_s) {
    if (!h || h->type != 3) return fail(ERR_ARG, "not a type-3 plan");
    int s = nufft3_setpts(h->t3, m, d_x, n, d_s, &h->opts);
    if (s != OK) return fail(s, "type-3 NUFFT setpts failed");
    return OK;
}

extern "C" int curig_nufft_info3(curig_nufft h, int *nf, double *dinfo) {
    if (!h || h->type != 3) return fail(ERR_ARG, "not a type-3 plan");
    nufft3_info(h->t3, nf, dinfo);
    return OK;
}

extern "C" int curig_nufft_setpts(curig_nufft h, int64_t m, const double *d_x, const double *d_y) {
    if (!h || !d_x || m <= 0 || (h->dim >= 2 && !d_y) || (h->dim == 3 && !h->d_z))
        return fail(ERR_ARG, "invalid NUFFT points");
    if (h->type == 3) return fail(ERR_ARG, "type-3 plans take their points with curig_nufft_setpts3");
    Plan *p = h->p;
    if (h->d_uvw) cudaFreeAsync(h->d_uvw, p->st);
    h->d_uvw = nullptr;
    if (alloc_async((void **)&h->d_uvw, 3 * m * sizeof(double), p->st) != cudaSuccess)
        return fail(ERR_NOMEM, "out of device memory");
    const double sgn = h->type == 1 ? (double)h->iflag : -(double)h->iflag;
    launch_nupts_uvw(m, d_x, h->dim >= 2 ? d_y : nullptr, h->dim == 3 ? h->d_z : nullptr, sgn, h->d_uvw, p->st);
    const double freq = SPEEDOFLIGHT;                   // f / c = 1
    int s = plan_setpts(p, m, 1, h->d_uvw, h->d_uvw + 1, h->d_uvw + 2, 3, &freq);
    if (s != OK) return fail(s, p->last_error.empty() ? "NUFFT setpts failed" : p->last_error);
    return OK;
}

extern "C" int curig_nufft_execute(curig_nufft h, void *d_c, void *d_fk) {
    if (!h || !d_c || !d_fk) return fail(ERR_ARG, "invalid NUFFT execute arguments");
    if (h->type == 3) {
        int s = nufft3_execute(h->t3, d_c, d_fk);
        if (s != OK) return fail(s, "type-3 NUFFT execute failed");
        return OK;
    }
    int s = plan_execute(h->p, d_c, nullptr, d_fk, h->type);
    if (s != OK) return fail(s, h->p->last_error.empty() ? "NUFFT execute failed" : h->p->last_error);
    return OK;
}

extern "C" int curig_nufft_destroy(curig_nufft h) {
    if (!h) return OK;
    if (h->type == 3) {
        nufft3_destroy(h->t3);
        delete h;
        return OK;
    }
    if (h->d_uvw) cudaFreeAsync(h->d_uvw, h->p->st);
    plan_destroy(h->p);
    delete h;
    return OK;
}

extern "C" int curig_setpts_uvw(curig_plan h, int64_t nrow, int nchan, const double *du, const double *dv,
                                const double *dw, int stride, const double *freq) {
    if (!h) return fail(ERR_ARG, "null plan");
    int s = plan_setpts(h->p, nrow, nchan, du, dv, dw, stride, freq);
    if (s != OK) return fail(s, h->p->last_error.empty() ? "setpts failed" : h->p->last_error);
    return OK;
}

extern "C" int curig_setpts(curig_plan h, int64_t nrow, int nchan, const double *d_uvw, const double *freq) {
    if (!d_uvw) return fail(ERR_ARG, "null uvw");
    return curig_setpts_uvw(h, nrow, nchan, d_uvw, d_uvw + 1, d_uvw + 2, 3, freq);
}

extern "C" int curig_execute(curig_plan h, void *d_vis, const void *d_wgt, void *d_dirty) {
    if (!h) return fail(ERR_ARG, "null plan");
    int s = plan_execute(h->p, d_vis, d_wgt, d_dirty);
    if (s != OK) return fail(s, h->p->last_error.empty() ? "execute failed" : h->p->last_error);
    return OK;
}

extern "C" int curig_execute_dir(curig_plan h, int type, void *d_vis, const void *d_wgt, void *d_dirty) {
    if (!h) return fail(ERR_ARG, "null plan");
    int s = plan_execute(h->p, d_vis, d_wgt, d_dirty, type);
    if (s != OK) return fail(s, h->p->last_error.empty() ? "execute failed" : h->p->last_error);
    return OK;
}

extern "C" void curig_set_timing(int on) { set_timing(on != 0); }

extern "C" int curig_plan_timings(curig_plan h, double *out, int n) {
    if (!h || !out) return fail(ERR_ARG, "null argument");
    return plan_timings(h->p, out, n);
}

extern "C" int64_t curig_launch_count(void) { return launch_count(); }

extern "C" int curig_plan_status(curig_plan h) {
    if (!h) return fail(ERR_ARG, "null plan");
    const int s = plan_device_status(h->p);
    if (s != OK) return fail(s, h->p->last_error.empty() ? "device status" : h->p->last_error);
    return OK;
}

extern "C" void curig_test_tile_wait(int64_t polls, int noissue) { set_tile_wait(polls, noissue); }

extern "C" void curig_test_gather_scratch(int on) { set_gather_scratch(on); }

extern "C" int curig_destroy(curig_plan h) {
    if (!h) return OK;
    plan_destroy(h->p);
    delete h;
    return OK;
}

extern "C" int curig_plan_info(curig_plan h, int *info, double *dinfo) {
    if (!h || !h->p->ready) return fail(ERR_ARG, "plan has no points");
    const Plan *p = h->p;
    if (info) {
        info[0] = p->gp.nf1; info[1] = p->gp.nf2; info[2] = p->gp.nf3; info[3] = p->gp.kp.kw;
        info[4] = p->tg.bx; info[5] = p->tg.bz; info[6] = (int)p->tg.nbins(); info[7] = p->win.kind;
    }
    if (dinfo) {
        dinfo[0] = p->gp.kp.beta; dinfo[1] = p->gp.gamma; dinfo[2] = p->gp.h;
        dinfo[3] = p->gp.i_center; dinfo[4] = p->gp.i_half; dinfo[5] = p->gp.o_center;
    }
    return OK;
}

// Relative L2 error of a plan's results against the FP64 direct transform,
// estimated from its parts (added in quadrature), each calibrated on this
// library's measurements against the FP64 DFT:
//  * window: the ES window at sigma 2 measured per width W (256^2, 3000
//    visibilities, w-stacking; W = 4..8: 2.0e-3, 1.08e-4, 1.12e-5, 1.32e-6,
//    1.62e-7, a factor of about 8.5 per width beyond), scaled by
//    exp(-pi W (sqrt(1 - 1/sigma) - sqrt(1/2))) for other sigma; a learned
//    window's own measured error (eps_reached);
//  * arithmetic: FP32 gridding 3.5e-7 (two-word tiles against FP64 over the
//    whole 4096^2 image: 2.9e-7 to 3.6e-7), FP64 1e-13;
//  * accumulation: FP32 one-word tiles 1.5e-6 (against the exact two-word
//    tiles at full density: 1.3e-6 to 1.6e-6), otherwise 0.
static double es_window_error(int W, double sigma) {
    static const double tab[5] = {2.0e-3, 1.08e-4, 1.12e-5, 1.32e-6, 1.62e-7};   // W = 4..8
    double e = W < 4 ? tab[0] * std::pow(8.5, 4 - W) : W > 8 ? tab[4] * std::pow(8.5, -(W - 8)) : tab[W - 4];
    return e * std::exp(-PI_D * W * (std::sqrt(1.0 - 1.0 / sigma) - std::sqrt(0.5)));
}

extern "C" int curig_plan_error(curig_plan h, double *est) {
    if (!h || !h->p->ready || !est) return fail(ERR_ARG, "plan has no points");
    const Plan *p = h->p;
    const double win = p->win.kind == 1 ? p->win.eps_reached : es_window_error(p->gp.kp.kw, p->gp.kp.upsampfac);
    const bool f32 = p->opt.precision == 1;
    const double arith = f32 ? 3.5e-7 : 1e-13;
    const double acc = f32 && p->dg.smode == 2 ? 1.5e-6 : 0.0;
    est[1] = win;
    est[2] = arith;
    est[3] = acc;
    est[0] = std::sqrt(win * win + arith * arith + acc * acc);
    return OK;
}

extern "C" int curig_set_window(int kw, int degree, const double *coef, double eps_reached) {
    int s = registry_set_window(kw, degree, coef, eps_reached);
    return s == OK ? OK : fail(s, "invalid window table");
}

extern "C" void curig_clear_windows(void) { registry_clear(); }

extern "C" int curig_grid_params(int nx, int ny, double psx, double psy, double wmin, double wmax,
                                 double eps, double sigma, int *iout, double *dout) {
    GridParams gp;
    int s = grid_params(nx, ny, psx, psy, wmin, wmax, eps, sigma, 1, gp);
    if (s != OK) return fail(s, "invalid grid parameters");
    if (iout) { iout[0] = gp.nf1; iout[1] = gp.nf2; iout[2] = gp.nf3; iout[3] = gp.kp.kw; }
    if (dout) {
        dout[0] = gp.kp.beta; dout[1] = gp.gamma; dout[2] = gp.h;
        dout[3] = gp.i_center; dout[4] = gp.i_half; dout[5] = gp.o_center;
    }
    return OK;
}

extern "C" int curig_psi_hat(int nf, double eps, double sigma, double *out) {
    KernelParams kp;
    int s = setup_kernel(eps, sigma, kp);
    if (s != OK) return fail(s, "invalid kernel parameters");
    if (nf < 2 || !out) return fail(ERR_ARG, "invalid argument");
    std::vector<double> v;
    psi_hat_grid(nf, kp, Window(), v);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
    return OK;
}

// ------------------------------------------------------------------ C++ gridder_* mirror
int gridder_setting(int N1, int N2, int method, int kerevalmeth, int w_term_method, double tol,
                    int direction, double sigma, int iflag, int batchsize, int M, int channel,
                    double fov, visibility *pv, double *d_u, double *d_v, double *d_w,
                    cuDoubleComplex *d_c, curafft_plan *plan, ragridder_plan *gplan) {
    (void)kerevalmeth; (void)iflag; (void)batchsize;
    if (!plan || !gplan || !pv || !pv->frequency || M <= 0) return ERR_ARG;
    if (method != 0 || w_term_method != 1) return ERR_UNSUPPORTED;
    double psx, psy;
    ref_pixsizes(fov, N2, N1, psx, psy);
    Options opt;
    Plan *p = nullptr;
    int s = plan_create(direction == 1 ? 1 : 2, N2, N1, psx, psy, tol, sigma, pv->sign, opt, &p);
    if (s != OK) return s;
    s = plan_setpts(p, M, 1, d_u, d_v, d_w, 1, pv->frequency);
    if (s != OK) { plan_destroy(p); return s; }
    plan->impl = p;
    plan->d_c = d_c; plan->d_u = d_u; plan->d_v = d_v; plan->d_w = d_w;
    plan->dim = 3; plan->type = direction == 1 ? 1 : 2; plan->M = M;
    plan->nf1 = p->gp.nf1; plan->nf2 = p->gp.nf2; plan->nf3 = p->gp.nf3;
    plan->ms = N1; plan->mt = N2; plan->mu = 1;
    plan->iflag = direction == 1 ? 1 : -1; plan->batchsize = p->gp.nf3; plan->direction = direction;
    gplan->kv = *pv;
    gplan->fov = fov; gplan->pixelsize_x = psx; gplan->pixelsize_y = psy;
    gplan->num_w = p->gp.nf3; gplan->width = N1; gplan->height = N2;
    gplan->channel = channel; gplan->nrow = M; gplan->w_term_method = w_term_method;
    gplan->speedoflight = 299792458;
    return OK;
}

int gridder_execution(curafft_plan *plan, ragridder_plan *gplan) {
    if (!plan || !plan->impl || !plan->fk || !plan->d_c) return ERR_ARG;
    Plan *p = static_cast<Plan *>(plan->impl);
    double *d_wgt = nullptr;
    if (gplan && gplan->kv.weight) {               // ra_exec.cu:98-104 uploads per call
        if (alloc_async((void **)&d_wgt, (size_t)p->nrow * sizeof(double), p->st) != cudaSuccess)
            return ERR_NOMEM;
        cudaMemcpyAsync(d_wgt, gplan->kv.weight, (size_t)p->nrow * sizeof(double), cudaMemcpyHostToDevice,
                        p->st);
    }
    int s = plan_execute(p, plan->d_c, d_wgt, plan->fk);
    if (d_wgt) cudaFreeAsync(d_wgt, p->st);
    if (cudaStreamSynchronize(p->st) != cudaSuccess && s == OK) s = ERR_CUDA;
    return s;
}

int gridder_destroy(curafft_plan *plan, ragridder_plan *gplan) {
    if (plan && plan->impl) {
        plan_destroy(static_cast<Plan *>(plan->impl));
        plan->impl = nullptr;
    }
    if (gplan) {                                   // cugridder.cu:297-303
        free(gplan->dirty_image); gplan->dirty_image = nullptr;
        free(gplan->kv.u); free(gplan->kv.v); free(gplan->kv.w); free(gplan->kv.vis);
        free(gplan->kv.frequency); free(gplan->kv.weight);
        gplan->kv.u = gplan->kv.v = gplan->kv.w = nullptr;
        gplan->kv.vis = nullptr; gplan->kv.frequency = nullptr; gplan->kv.weight = nullptr;
    }
    return OK;
}
