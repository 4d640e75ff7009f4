// Plan object of the B200 gridder (host side).
#pragma once

#include "curig_internal.h"
#include "kernels.cuh"

#include <string>

namespace curig {

struct Options {
    int precision = 0;        // 0: FP64 (the reference's only precision), 1: FP32
    int window = 0;           // 0: ES kernel, 1: learned window table (see set_window)
    int bin_xy = 0;           // bin edge in cells (0: chosen from the shared-memory budget)
    int sub = 0;              // visibilities per sub-problem (0: default)
    size_t smem_budget = 0;   // bytes of shared memory per CTA for tiles (0: default)
    cudaStream_t stream = nullptr;
};

struct Plan {
    int type = 1;             // 1: ms2dirty (vis -> dirty), 2: dirty2ms (dirty -> vis)
    int nx = 0, ny = 0;
    double psx = 0, psy = 0, eps = 1e-6, sigma = 2.0;
    int sign = 1;
    Options opt;
    cudaStream_t st = nullptr;
    int device = 0, nsm = 148;

    // set by setpts
    bool ready = false;
    long long nrow = 0;
    int nchan = 0;
    std::vector<double> freq;
    const double *du = nullptr, *dv = nullptr, *dw = nullptr;
    int stride = 3;
    GridParams gp;
    TileGeom tg;
    DevGeom dg{};
    DevCorr dc{};
    Window win;
    size_t smem = 0;
    double wmin_eff = 0, wmax_eff = 0;

    // device buffers owned by the plan
    double *d_foc = nullptr, *d_quad = nullptr, *d_psi1 = nullptr, *d_psi2 = nullptr, *d_wcoef = nullptr;
    int *d_bin_count = nullptr, *d_bin_start = nullptr, *d_nsub = nullptr, *d_sub_end = nullptr;
    int *d_rank = nullptr, *d_perm = nullptr, *d_err = nullptr;
    unsigned long long *d_keys = nullptr;
    void *d_rec = nullptr, *d_cs = nullptr, *d_grid = nullptr, *d_scan_tmp = nullptr;
    size_t scan_bytes = 0;

    cufftHandle fft_main = 0, fft_rest = 0;
    int fft_batch = 0, fft_rest_batch = 0;

    // learned-window tables per width (coefficients [kw][deg+1]); empty -> ES only
    std::vector<Window> learned;
    std::string last_error;
};

int plan_create(int type, int nx, int ny, double psx, double psy, double eps, double sigma, int sign,
                const Options &opt, Plan **out);
int plan_setpts(Plan *p, long long nrow, int nchan, const double *du, const double *dv,
                const double *dw, int stride, const double *h_freq);
int plan_execute(Plan *p, void *d_vis, const void *d_wgt, void *d_dirty);
int plan_destroy(Plan *p);
void plan_release_points(Plan *p);

// launchers (kernels.cu)
void launch_wrange(const double *w, int stride, long long nrow, unsigned long long *keys, int *err,
                   cudaStream_t st);
void launch_bin_count(const DevGeom &g, const double *u, const double *v, const double *w,
                      const double *foc, int *bin_count, int *rank, int *err, cudaStream_t st);
void launch_nsub(const int *count, int *nsub, long long nb, int sub, cudaStream_t st);
size_t scan_temp_bytes(long long n);
int scan_exclusive(void *tmp, size_t tmpb, const int *in, int *out, long long n, cudaStream_t st);
int scan_inclusive(void *tmp, size_t tmpb, const int *in, int *out, long long n, cudaStream_t st);
size_t tile_smem_bytes(const TileGeom &tg, int esize, int kw, int wdeg);
template <typename T>
void launch_bin_scatter(const DevGeom &g, const double *u, const double *v, const double *w,
                        const double *foc, const int *bin_start, const int *rank, void *rec, int *perm,
                        cudaStream_t st);
template <typename T>
void launch_vis_prep(const DevGeom &g, const double *w, const double *foc, const void *vis,
                     const void *wgt, const int *perm, void *cs, cudaStream_t st);
template <typename T>
void launch_vis_out(const DevGeom &g, const double *w, const double *foc, const void *os,
                    const int *perm, const void *wgt, void *vis, cudaStream_t st);
template <typename T>
int launch_spread(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                  const void *rec, const void *cs, void *grid, const double *wc, int nsm, cudaStream_t st);
template <typename T>
int launch_interp(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                  const void *rec, const void *grid, void *os, const double *wc, int nsm, cudaStream_t st);
template <typename T>
void launch_correct_m2d(const DevCorr &cc, const void *grid, void *dirty, cudaStream_t st);
template <typename T>
void launch_correct_d2m(const DevCorr &cc, const void *dirty, void *grid, cudaStream_t st);
template <typename T>
void launch_zero_pad(int nx, int ny, int nf1, int nf2, int nf3, void *grid, cudaStream_t st);

// global learned-window registry (set through the C ABI)
int registry_set_window(int kw, int degree, const double *coef, double eps_reached);
// smallest registered width whose reached error is <= eps (nullptr: none)
const Window *registry_pick_window(double eps);
const Window *registry_get_window(int kw);
void registry_clear();

}  // namespace curig
