// Internal declarations of the B200 gridder: parameters, plan state, kernels.
//
// Layout in HBM (one plan):
//   grid      [nf3][nf2][nf1] complex<T>, plane-major, x (nf1, pairs with v and
//             nydirty) fastest -- the batched 2-D cuFFT layout.
//   records   visibilities in bin order: SoA {packed start cell, fractional
//             offsets (ux,uy,uz) in [0,1)} plus, per execute, the weighted and
//             phase-shifted values c.
//   dirty     [nxdirty][nydirty] complex<T>, row-major (the reference's layout).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <cstdint>
#include <cstddef>
#include <vector>

namespace curig {

// cudaMallocAsync whose failure is reported by its return value only: the
// runtime's last-error state is cleared again, so the launch checks
// (cudaGetLastError) of this or a later call do not report the failed
// allocation a second time.  After an out-of-memory failure the device's
// default pool is trimmed: a request larger than the device can leave the
// pool holding what it mapped before giving up (the pool keeps freed memory,
// its release threshold being raised), which other processes then lack.
inline cudaError_t alloc_async(void **ptr, size_t bytes, cudaStream_t st) {
    const cudaError_t e = cudaMallocAsync(ptr, bytes, st);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        int dev = 0;
        cudaMemPool_t pool;
        if (e == cudaErrorMemoryAllocation && cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
            cudaMemPoolTrimTo(pool, 0);
        (void)cudaGetLastError();
    }
    return e;
}

// ------------------------------------------------------------------ errors
enum Status : int {
    OK = 0,
    ERR_GENERIC = 1,      // the reference's only error code (cugridder.cu:403-406)
    ERR_SIGMA = 2,        // bad upsampling factor (conv_interp_invoker.cu:53-116 returns 2)
    ERR_ARG = 3,          // invalid sizes / null pointers
    ERR_CUDA = 4,         // CUDA runtime error
    ERR_CUFFT = 5,        // cuFFT error
    ERR_NOMEM = 6,        // allocation failed
    ERR_NONFINITE = 7,    // NaN / Inf in uvw or frequencies
    ERR_UNSUPPORTED = 8,  // option combination not supported
    ERR_WINDOW = 9,       // learned window missing for the requested width
};

constexpr double SPEEDOFLIGHT = 299792458.0;
constexpr double PI_D = 3.14159265358979323846;
constexpr double INV_2PI = 0.159154943091895336;   // the reference's M_1_2PI
constexpr int MAX_KW = 28;                         // the reference's MAX_KERNEL_WIDTH
constexpr int MAX_QUAD = 128;                      // quadrature nodes on the half line
constexpr int MAX_POLY = 16;                       // piecewise-polynomial window degree + 1

// ------------------------------------------------------------------ params
struct KernelParams {
    int kw = 0;            // support width in cells
    double beta = 0;       // ES beta
    double c = 0;          // ES c = 4/kw^2
    double upsampfac = 2;  // sigma
    int ier = 0;           // 1 = eps clamped (warning), as the reference
};

// Window used by the spreader / interpolator and the correction.
//   kind 0: ES exp(beta*(sqrt(1-c t^2)-1)) evaluated directly (normalised by
//           e^-beta; the correction uses the same normalisation).
//   kind 1: piecewise polynomial on kw unit intervals (learned window tables or
//           the ES approximated by Horner polynomials).
struct Window {
    int kind = 0;
    int kw = 0;
    int degree = 0;                       // polynomial degree (kind 1)
    std::vector<double> coef;             // [kw][degree+1], highest power first
    double eps_reached = 0;               // error the table reaches against the exact DFT
};

struct GridParams {
    int nx = 0, ny = 0;          // nxdirty (N2), nydirty (N1)
    int nf1 = 0, nf2 = 0, nf3 = 0;
    double pixsize_x = 0, pixsize_y = 0;
    double i_center = 0, i_half = 0;   // w range (effective units)
    double o_center = 0, o_half = 0;   // n-1 range
    double gamma = 1, h = 0;
    int sign = 1;
    int no_w = 0;                // w ignored: one plane, n = 1, no w phase
    KernelParams kp;
};

int setup_kernel(double eps, double sigma, KernelParams &kp);
int next235beven(int n, int b);
int get_num_cells(int ms, const KernelParams &kp);
void set_nhg_type3(double S, double X, const KernelParams &kp, int &nf, double &h, double &gam);
void gauss_legendre(int n, double *x, double *w);
// nodes (grid units, >= 0) and weights g = alpha*w*phi for the kernel FT
int quadrature_terms(const KernelParams &kp, const Window &win, double *xs, double *g);
double window_value(const KernelParams &kp, const Window &win, double t);
void psi_hat_grid(int nf, const KernelParams &kp, const Window &win, std::vector<double> &out);
// Optional sizing requests: an explicit oversampled grid (grid_x along the
// nxdirty axis, grid_y along nydirty; 0 = the sigma rule) and the no-w mode.
struct GridRequest {
    int grid_x = 0, grid_y = 0;
    int no_w = 0;
};
int grid_params(int nx, int ny, double pixsize_x, double pixsize_y, double wmin_eff,
                double wmax_eff, double eps, double sigma, int sign, GridParams &gp,
                int kw_override = 0, const GridRequest &req = GridRequest());
void es_horner_window(const KernelParams &kp, int degree, Window &win);

// ------------------------------------------------------------------ tiles
struct TileGeom {
    int bx = 16, by = 16, bz = 0;      // bin size in cells (bz = nf3: one z bin)
    int tx = 0, ty = 0, tz = 0;        // shared tile extent = bin + kw (z: nf3 if unpadded)
    int nbx = 0, nby = 0, nbz = 0;     // number of bins per axis
    int zpad = 1;                      // 1: tile z = bz + kw with offset; 0: tile z = nf3
    int sub = 1024;                    // visibilities per sub-problem
    int fix = 0;                       // spreader tile: 1 two-word, 2 one-word int32 fixed point, 3 three-word int32 (FP64)
    size_t smem_bytes = 0;
    long long nbins() const { return (long long)nbx * nby * nbz; }
};

}  // namespace curig
