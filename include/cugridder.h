/*
 * C++ plan API with the reference's names and argument meaning
 * (include/cugridder.h:8-11, src/astro/cugridder.cu:105-307), for C++ callers
 * that drive the gridder with their own device arrays:
 *
 *   gridder_setting(N1 = nydirty, N2 = nxdirty, method, kerevalmeth,
 *                   w_term_method, tol, direction (1: vis->image, 0: image->vis),
 *                   sigma, iflag, batchsize, M, channel, fov (degrees),
 *                   pointer_v (host: frequency[0], sign, weight), d_u, d_v, d_w
 *                   (device, M each), d_c (device vis), plan, gridder_plan)
 *   caller sets plan->fk (device dirty image [N2][N1]) and, for direction 0,
 *   plan->d_c (device output vis), then gridder_execution(plan, gridder_plan).
 *
 * Differences from the reference, by design: d_u/d_v/d_w are read, not
 * rescaled in place; only method 0 / w_term_method 1 exist (as in the
 * reference); gridder_destroy releases the library state and the host arrays
 * held in gridder_plan->kv (as the reference does) but not the two plan
 * structs, which the caller owns (the reference calls free() on a new-ed
 * object, cugridder.cu:296).
 */
#ifndef CURIG_CUGRIDDER_H
#define CURIG_CUGRIDDER_H

#include <complex>
#include <cuComplex.h>

struct visibility {            /* include/ragridder_plan.h:6-31 */
    double *u;
    double *v;
    double *w;
    std::complex<double> *vis;
    double *weight;
    bool *flag;
    double *frequency;
    int pirange;
    int sign;
};

struct ragridder_plan {        /* include/ragridder_plan.h:33-54 */
    visibility kv;
    double fov;
    double pixelsize_x;
    double pixelsize_y;
    double w_max;
    double w_min;
    double w_s_r;
    int num_w;
    double w_0;
    double delta_w;
    int speedoflight;
    std::complex<double> *dirty_image;
    int width;
    int height;
    int channel;
    int nrow;
    int cur_channel;
    int w_term_method;
};

struct curafft_plan {          /* the fields of include/curafft_plan.h:50-122 that callers use */
    cuDoubleComplex *d_c;      /* device visibilities (input of direction 1, output of 0) */
    cuDoubleComplex *fk;       /* device dirty image [N2][N1] */
    double *d_u, *d_v, *d_w;
    int dim;
    int type;
    int M;
    int nf1, nf2, nf3;
    int ms, mt, mu;
    int iflag;
    int batchsize;
    int direction;
    void *impl;                /* library state */
};

int gridder_setting(int N1, int N2, int method, int kerevalmeth, int w_term_method, double tol,
                    int direction, double sigma, int iflag, int batchsize, int M, int channel,
                    double fov, visibility *pointer_v, double *d_u, double *d_v, double *d_w,
                    cuDoubleComplex *d_c, curafft_plan *plan, ragridder_plan *gridder_plan);
int gridder_execution(curafft_plan *plan, ragridder_plan *gridder_plan);
int gridder_destroy(curafft_plan *plan, ragridder_plan *gridder_plan);

#endif
