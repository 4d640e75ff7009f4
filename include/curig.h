/*
 * curig_b200 -- C ABI of the B200-native ms2dirty / dirty2ms gridder.
 *
 * Shared library: curig_b200/libcurafft.so (same file name as the reference's
 * build product, Makefile:177-178 / setup.py:24).  All entry points are
 * extern "C", take plain pointers and sizes, and return an int status:
 *   0 ok, 1 generic error (the reference's code), 2 bad sigma, 3 bad argument,
 *   4 CUDA error, 5 cuFFT error, 6 out of device memory, 7 NaN/Inf input,
 *   8 unsupported option, 9 no learned window reaches the requested epsilon.
 * No entry point calls exit(); errors are returned (the reference exits the
 * process through checkCudaErrors, include/cuda_sample/helper_cuda.h:583-595).
 *
 * Conventions shared with the reference (include/cugridder.h:12-21,
 * src/astro/cugridder.cu:330-612):
 *   uvw    [nrow][3] float64, metres (u, v, w per row)
 *   vis    [nrow] (reference ABI) or [nrow][nchan] complex
 *   wgt    same shape as vis, real, may be NULL; it multiplies in both
 *          directions (src/astro/ra_exec.cu:103, ra_exec.cu:81 -> utils.cu:189)
 *   dirty  [nxdirty][nydirty] complex, row-major; pixel (ix, iy) is at
 *          l = (ix - nxdirty/2) * pixsize_x, m = (iy - nydirty/2) * pixsize_y
 *   sign   sign of the w term: phase = f/c (u l + v m + sign w (n - 1))
 *   ms2dirty: dirty = sum wgt vis e^{+2 pi i phase} / n
 *   dirty2ms: vis   = wgt sum_pix dirty / n e^{-2 pi i phase}
 */
#ifndef CURIG_H
#define CURIG_H

#include <stdint.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> curig_cdouble;
extern "C" {
#else
#include <complex.h>
typedef double _Complex curig_cdouble;
#endif

/* ---------------------------------------------------------------- reference ABI
 * Single channel (freq), FP64, host buffers; the library allocates, copies and
 * frees all device memory inside the call.  fov in degrees; pixel sizes are
 * fov/180*pi/nxdirty and fov/180*pi/nydirty (src/astro/cugridder.cu:48-49).
 */
/* replaces ms2dirty_1, include/cugridder.h:15-16 (src/astro/cugridder.cu:594-599) */
int ms2dirty_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               curig_cdouble *vis, curig_cdouble *dirty, double epsilon, double sigma, int sign);
/* replaces ms2dirty_2, include/cugridder.h:13-14 (src/astro/cugridder.cu:587-592) */
int ms2dirty_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               curig_cdouble *vis, double *wgt, curig_cdouble *dirty, double epsilon, double sigma,
               int sign);
/* replaces dirty2ms_1, include/cugridder.h:17-18 (src/astro/cugridder.cu:601-606); vis is the output */
int dirty2ms_1(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               curig_cdouble *vis, curig_cdouble *dirty, double epsilon, double sigma, int sign);
/* replaces dirty2ms_2, include/cugridder.h:19-20 (src/astro/cugridder.cu:608-612) */
int dirty2ms_2(int nrow, int nxdirty, int nydirty, double fov, double freq, double *uvw,
               curig_cdouble *vis, double *wgt, curig_cdouble *dirty, double epsilon, double sigma,
               int sign);

/* ---------------------------------------------------------------- options */
typedef struct curig_opts {
    int precision;        /* 0: FP64 (default), 1: FP32 gridding (FP64 w-phase and correction) */
    int window;           /* 0: ES kernel (default), 1: learned window (curig_set_window) */
    int bin_xy;           /* bin edge in cells, 0 = automatic */
    int sub;              /* visibilities per sub-problem (tile chunk), 0 = automatic: 16384
                             for one-word FP32 tiles (requests up to 65536), 4096 otherwise
                             (also the largest value the two- and three-word tiles take) */
    int64_t smem_budget;  /* shared-memory bytes per tile CTA, 0 = automatic */
    void *stream;         /* cudaStream_t for the device-pointer API, NULL = legacy stream */
    int accumulate;       /* FP32 tile accumulation: 0 automatic (default: one-word when
                             epsilon >= 1e-5, else two-word), 1 float atomics, 2 one-word
                             int32 fixed point (22-bit terms, deterministic), 3 two-word
                             int32 fixed point (exact sums, deterministic).  FP64 tiles:
                             1 double atomics, any other value three-word int32 fixed point
                             (exact sums, deterministic) */
    int w_term;           /* 0: improved w-stacking (default); 1: w ignored -- 2-D gridding
                             without the n-1 term or the 1/n factor (the Nifty gridder's
                             do_wstacking = False; no counterpart in the reference, whose
                             w_term_method 0 is not functional, ra_exec.cu:124) */
    int grid_x;           /* oversampled grid size along the nxdirty axis (the Nifty gridder's
                             nx), even and >= nxdirty; 0 = sigma rule (cugridder.cu:180-181) */
    int grid_y;           /* the same along the nydirty axis (Nifty's ny); both or neither */
    int bin_z;            /* w-planes per tile slab (1 .. nf3 - 1), 0 = automatic (all planes in
                             one tile unless a w support could wrap) */
    int slabs;            /* one-shot calls only: row slabs of the copy / compute pipeline
                             (1 .. 8; ms2dirty spreads slab k while slab k+1 is uploaded,
                             dirty2ms downloads slab k while slab k+1 is interpolated);
                             0 = automatic (3 from 1 GiB of visibilities and weights,
                             2 from 384 MiB, else 1).  Plans ignore it. */
    int sparse;           /* tile spreaders: a chunk of fewer visibilities than this adds its
                             taps straight to the grid instead of through a shared-memory tile
                             (0: automatic, 128 in FP32, 64 in FP64; negative: always the tile) */
} curig_opts;

void curig_default_opts(curig_opts *opts);

/* ---------------------------------------------------------------- one-shot, host buffers
 * Multi-channel generalisation of the reference ABI (which uses freq[0] only,
 * python/curagridder/curagridder.py:92): all nchan channels are folded into one
 * transform and the dirty image is their sum.  vis/wgt/dirty element type
 * follows opts->precision (complex128/float64 or complex64/float32).  pixsize
 * in radians.  Replaces per-channel loops over ms2dirty_2 / dirty2ms_2.
 */
int curig_ms2dirty(int64_t nrow, int nchan, int nxdirty, int nydirty, double pixsize_x,
                   double pixsize_y, const double *freq, const double *uvw, const void *vis,
                   const void *wgt, void *dirty, double epsilon, double sigma, int sign,
                   const curig_opts *opts);
int curig_dirty2ms(int64_t nrow, int nchan, int nxdirty, int nydirty, double pixsize_x,
                   double pixsize_y, const double *freq, const double *uvw, void *vis,
                   const void *wgt, const void *dirty, double epsilon, double sigma, int sign,
                   const curig_opts *opts);

/* ---------------------------------------------------------------- plan API, device pointers
 * C counterpart of gridder_setting / gridder_execution / gridder_destroy
 * (include/cugridder.h:8-11): create once, set points once (device uvw,
 * host frequencies), execute many times on new visibilities / images.
 * type 1: ms2dirty (vis -> dirty), type 2: dirty2ms (dirty -> vis).
 * The uvw buffer must stay valid while the plan executes.
 */
typedef struct curig_plan_s *curig_plan;
int curig_makeplan(int type, int nxdirty, int nydirty, double pixsize_x, double pixsize_y,
                   double epsilon, double sigma, int sign, const curig_opts *opts,
                   curig_plan *plan);
int curig_setpts(curig_plan plan, int64_t nrow, int nchan, const double *d_uvw,
                 const double *h_freq);
/* separate u, v, w device arrays with an element stride (1: SoA, 3: AoS) */
int curig_setpts_uvw(curig_plan plan, int64_t nrow, int nchan, const double *d_u,
                     const double *d_v, const double *d_w, int stride, const double *h_freq);
int curig_execute(curig_plan plan, void *d_vis, const void *d_wgt, void *d_dirty);
/* execute in either direction with the same points: type 1 ms2dirty, 2 dirty2ms */
int curig_execute_dir(curig_plan plan, int type, void *d_vis, const void *d_wgt, void *d_dirty);
int curig_destroy(curig_plan plan);
/* info[0..7] = nf1, nf2, nf3, kw, bin_xy, bin_z, n_bins, window kind;
 * dinfo[0..5] = beta, gamma, h, w centre, w half width, n-1 centre */
int curig_plan_info(curig_plan plan, int *info, double *dinfo);
/* The error of this plan's results against the FP64 direct transform, stated
 * per result: est[0] = estimated relative L2 error, from est[1] the window
 * (ES per width and sigma, or the learned window's measured error), est[2] the
 * arithmetic (FP32 gridding with FP64 w-phase and correction, or FP64) and
 * est[3] the tile accumulation (FP32 one-word fixed point), added in
 * quadrature; the parts are calibrated on measurements against the FP64 DFT
 * (4096^2, 1.6e8 visibilities).  No counterpart in the reference. */
int curig_plan_error(curig_plan plan, double *est);

/* ---------------------------------------------------------------- learned window
 * Register a piecewise-polynomial window for support width kw: coef is
 * [kw][degree+1], interval d covers t in [d - kw/2, d + 1 - kw/2], variable
 * s = 2 (t - d + kw/2) - 1 in [-1, 1], highest power first.  eps_reached is
 * the relative error the window reaches against the exact DFT; a plan with
 * opts.window = 1 picks the narrowest registered window with
 * eps_reached <= epsilon.  No counterpart in the reference (its kernel is the
 * fixed ES function, src/fourier/conv.cu:17-25).
 */
int curig_set_window(int kw, int degree, const double *coef, double eps_reached);
void curig_clear_windows(void);

/* Learned window: phi(t) = exp(beta (sqrt(1 - x^2) - 1) + g(x^2)), x = 2t/W, with
 * g a 1-32-32-32-1 tanh MLP (FP32 parameters, curig_window_nparams() of them:
 * W1[32] b1[32] W2[32][32] b2[32] W3[32][32] b3[32] Wo[32] bo).  The objective
 * is log of the RMS error, over fractional offsets and the image band
 * |xi| <= 1/(2 sigma), of gridding one visibility, transforming and correcting
 * by the window's Fourier transform, against the exact DFT (per axis).
 * curig_train_window runs `iters` Adam steps on the current GPU in place on
 * params (loss_hist[iters] optional); curig_window_loss_grad evaluates the RMS
 * error and the gradient of its log; curig_window_table tabulates the window
 * (normalised to max 1) as [W][degree+1] Horner coefficients for
 * curig_set_window.  No counterpart in the reference. */
int curig_window_nparams(void);
int curig_train_window(int W, double sigma, int iters, double lr, float *params, double *loss_hist);
/* The same training on method-generated random visibilities: every step draws
 * 64 visibility positions (fractional cell offsets, uniform, from `seed`) and
 * takes the gradient of their gridding error against the exact DFT over the
 * image band; iters steps see 64 * iters random visibilities. */
int curig_train_window_mc(int W, double sigma, int iters, double lr, uint64_t seed, float *params,
                          double *loss_hist);
int curig_window_loss_grad(int W, double sigma, const float *params, double *loss, float *grad);
int curig_window_table(int W, double sigma, const float *params, int degree, double *coef);

/* Same result as curig_window_loss_grad, but allocates nothing on the device:
 * for callers that cannot call cudaMalloc where they need the objective (their
 * device memory is reserved up front by another framework's pool, or their
 * pipeline forbids allocation after initialisation).  Its scratch lives in one
 * 64 KiB file-scope device array that every GPU loading the library holds until
 * exit; the array's device address is looked up once per device, on the first
 * call with that device current, so make that first call before any stream
 * capture (and do not call it again on a device after cudaDeviceReset, which
 * reloads the module at a new address).  Calls
 * share the array: calls that overlap on the GPU race.  W above 12 is rejected
 * (status 3).  params, loss and grad are host pointers.  No counterpart in the
 * reference. */
int curig_window_loss_grad_static(int W, double sigma, const float *params, double *loss, float *grad);

/* ---------------------------------------------------------------- host-only helpers
 * Sizes and scalars a transform would use, computed on the host without a GPU:
 * iout[0..3] = nf1, nf2, nf3, kw; dout[0..5] = beta, gamma, h, w centre,
 * w half width, n-1 centre.  wmin/wmax are the effective (f/c * sign * 2 pi)
 * w extremes.  Restates setup_conv_opts (src/fourier/conv_interp_invoker.cu:46-116),
 * get_num_cells (conv_interp_invoker.cu:29-44), set_nhg_type3
 * (contrib/common.cpp:161-195) and setup_gridder_plan (src/astro/cugridder.cu:29-101).
 */
int curig_grid_params(int nxdirty, int nydirty, double pixsize_x, double pixsize_y, double wmin,
                      double wmax, double epsilon, double sigma, int *iout, double *dout);
/* Kernel Fourier transform of the ES window on fine-grid indices 0..nf/2,
 * including the (-1)^k half-grid factor; out has nf/2+1 entries and equals the
 * reference's fwkerhalf (src/fourier/deconv.cu:13-24, 60-102) times e^-beta. */
int curig_psi_hat(int nf, double epsilon, double sigma, double *out);

/* ---------------------------------------------------------------- instrumentation
 * Per-stage CUDA-event timing (the reference's -DTIME stage timers,
 * src/astro/cugridder.cu:348-450, ra_exec.cu:163-307), off by default.
 * curig_plan_timings synchronises the plan's stream and writes up to n
 * durations in ms: [0] setpts, [1] binning part of setpts, [2] vis prep,
 * [3] grid zero, [4] spread, [5] FFT (ms2dirty), [6] screen+correction,
 * [7] correction+screen (dirty2ms), [8] FFT (dirty2ms), [9] interpolation,
 * [10] vis output; -1 where a stage did not run.  curig_launch_count returns
 * the number of kernels this library has launched in the process. */
void curig_set_timing(int on);
int curig_plan_timings(curig_plan plan, double *out, int n);
int64_t curig_launch_count(void);

/* Flags the plan's kernels raised since its points were set: waits for the
 * plan's stream and returns 0, or 4 (CUDA) when an interpolator tile load did
 * not complete within its bounded wait, or 1 when an index check of the
 * bounds-checked build failed (curig_last_error says which).  The one-shot
 * calls check this themselves; the plan API leaves it to the caller, so that
 * execute stays asynchronous.  No counterpart in the reference (its kernels
 * report nothing). */
int curig_plan_status(curig_plan plan);

/* Test hook for the interpolator's bounded wait on its TMA tile loads: plans
 * whose points are set after this call poll a load's barrier at most `polls`
 * times (<= 0: the default, about a second) before raising the error that the
 * one-shot calls report as status 4 ("a tile load did not complete (timed
 * out)").  noissue != 0 arms the barrier without issuing the load, so the wait
 * runs out with nothing in flight; (0, 0) restores normal operation.  No
 * counterpart in the reference, which has no bounded waits. */
void curig_test_tile_wait(int64_t polls, int noissue);

/* Test hook for ms2dirty's weighted gather: with on = 0 the visibilities and
 * weights are gathered into bin order in one pass, the path taken when the
 * vis * wgt scratch (one complex value per visibility, from the device's
 * stream-ordered pool) cannot be allocated; on = 1 (the default) forms vis * wgt
 * in input order first.  The two differ only in the rounding order of the
 * products.  No counterpart in the reference. */
void curig_test_gather_scratch(int on);

/* Generic NUFFT, types 1 (points -> modes) and 2 (modes -> points) in one or two
 * dimensions, on the w-free gridder (same kernel-width, grid-size and correction
 * rules as the gridder; takes the place of the reference's cunufft_setting /
 * exec path for these types, src/fourier/cuft.cu:249).  Points x (and y for
 * dim 2) are device float64 arrays of m coordinates in radians (periodic,
 * any range); strengths c are device complex [m] (complex64 when
 * opts->precision = 1); modes fk are device complex [n1][n2] (dim 1: [n1]), mode
 * k = index - n/2.  Type 1: fk[k] = sum_j c_j e^{i iflag k.x_j}; type 2: c_j =
 * sum_k fk[k] e^{i iflag k.x_j}.  sigma: upsampling factor (2 = reference rule). */
typedef struct curig_nufft_s *curig_nufft;
int curig_nufft_makeplan(int type, int dim, int n1, int n2, double epsilon, int iflag, double sigma,
                         const curig_opts *opts, curig_nufft *plan);
int curig_nufft_setpts(curig_nufft plan, int64_t m, const double *d_x, const double *d_y);
int curig_nufft_execute(curig_nufft plan, void *d_c, void *d_fk);
int curig_nufft_destroy(curig_nufft plan);

/* Generic NUFFT type 3 in one dimension (nonuniform points to nonuniform
 * frequencies): f_k = sum_j c_j e^{i iflag s_k x_j}, j < m, k < n; the
 * reference's cunufft_setting type 3, dim 1 (src/fourier/cuft.cu:249-424, with
 * its pre/post stages cuft.cu:19-124; test/nufft_1d_3_1_test.cu).  Make the plan
 * with curig_nufft_makeplan(3, 1, n, 1, epsilon, iflag, sigma, opts, &plan) (n1:
 * the number of frequencies, informative), then give the device float64
 * points x[m] and frequencies s[n] here; curig_nufft_execute(plan, d_c, d_f)
 * maps strengths c[m] to values f[n] (complex, complex64 when
 * opts->precision = 1).  Sizes (grid nf, scale gamma, cell h) follow the
 * reference's set_nhg_type3 (contrib/common.cpp:161-195). */
int curig_nufft_setpts3(curig_nufft plan, int64_t m, const double *d_x, int64_t n, const double *d_s);

/* Generic NUFFT, types 1 and 2 in three dimensions (the reference's
 * cunufft_setting with dim 3, src/fourier/cuft.cu:293-305): modes fk
 * [n1][n2][n3] (n3 fastest), mode k = index - n/2 on every axis; points
 * x, y, z (device float64, radians, periodic).  Type 1: fk[k] = sum_j c_j
 * e^{i iflag k.x_j}; type 2: c_j = sum_k fk[k] e^{i iflag k.x_j}.  Execute and
 * destroy with curig_nufft_execute / curig_nufft_destroy. */
int curig_nufft3d_makeplan(int type, int n1, int n2, int n3, double epsilon, int iflag, double sigma,
                           const curig_opts *opts, curig_nufft *plan);
int curig_nufft3d_setpts(curig_nufft plan, int64_t m, const double *d_x, const double *d_y, const double *d_z);
/* nf and dinfo[0..5] = input centre, input half width, output centre, output
 * half width, gamma, h of a type-3 plan with points */
int curig_nufft_info3(curig_nufft plan, int *nf, double *dinfo);

/* Last error text of this thread (static storage, empty if none). */
const char *curig_last_error(void);

/* Device memory: calls and plans allocate from the current device's default
 * stream-ordered pool, which keeps freed memory for the next call (no
 * cudaMalloc per call).  This returns the pool's unused memory to the driver,
 * e.g. before another library needs it, and destroys the cached cuFFT
 * handles that no live plan holds (at most 16 such handles are kept between
 * calls; the rest are destroyed when released).  Call it when no call or plan
 * of this library is executing on the device.  No counterpart in the
 * reference, which allocates and frees with cudaMalloc / cudaFree in every
 * call. */
int curig_release_memory(void);

#ifdef __cplusplus
}
#endif
#endif /* CURIG_H */
