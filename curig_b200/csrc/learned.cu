// Learned gridding window: a 1 -> 32 -> 32 -> 32 -> 1 tanh MLP g(x^2) that
// multiplies the ES window, phi(t) = exp(beta (sqrt(1 - x^2) - 1) + g(x^2)),
// x = 2t/W, on |t| < W/2.  No counterpart in the reference (its window is the
// fixed ES function, src/fourier/conv.cu:17-25); the correction of a learned
// window comes from the same Gauss-Legendre quadrature (src/fourier/deconv.cu:13-197).
//
// Training objective, per axis (the 3-D error is, to first order, the sum of
// the axes' errors): grid one visibility at fractional offset f, transform,
// divide by the window's continuous Fourier transform psi(xi) and compare with
// the exact DFT e^{2 pi i xi u} over the image band |xi| <= 1/(2 sigma):
//   S(f, xi) = sum_d phi(t_d) e^{2 pi i xi t_d},  t_d = ceil(f - W/2) + d - f
//   e(f, xi) = S / psi - 1,   L = sqrt(mean_{f, xi} |e|^2)
// The forward, the backward (through the error model and the MLP) and the Adam
// update run in one CTA: one warp per point, lane k <-> hidden unit k.
#include "plan.h"

#include "../../include/curig.h"

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

namespace curig {

constexpr int H = 32;                               // hidden units
constexpr int NPAR = H + H + H * H + H + H * H + H + H + 1;   // 2209
constexpr int OFF_W1 = 0, OFF_B1 = 32, OFF_W2 = 64, OFF_B2 = 64 + H * H, OFF_W3 = OFF_B2 + H,
              OFF_B3 = OFF_W3 + H * H, OFF_WO = OFF_B3 + H, OFF_BO = OFF_WO + H;
constexpr int TNF = 64, TNXI = 64, TNQ = 96, TMAXW = 12;
constexpr int TNP = TNF * TMAXW + TNQ;                // point capacity
constexpr int TTHREADS = 256, TWARPS = TTHREADS / 32;

struct TrainGeom {
    int W, nf, nxi, nq, np;                          // np = nf*W + nq
    double beta, sigma;
    double lr, b1, b2, eps;
    int step;                                        // Adam step (1-based)
    int want_update;                                 // 0: loss / gradient only
    int mc;                                          // 1: random visibility offsets per step
    unsigned long long seed;                         // their stream
};

// Uniform [0, 1) from (seed, step, i): splitmix64 of the three, top 53 bits.
__device__ __forceinline__ double mc_uniform(unsigned long long seed, int step, int i) {
    unsigned long long z = seed + 0x9e3779b97f4a7c15ULL * ((unsigned long long)step * 1048576ULL + (unsigned)i + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double es_log(double x2, double beta) {
    // beta * (sqrt(1 - x^2) - 1) written without cancellation
    return -beta * x2 / (sqrt(fmax(1.0 - x2, 0.0)) + 1.0);
}

// Warp-cooperative MLP forward for one input z = x^2: lane k returns h1[k],
// h2[k], h3[k]; the output g is reduced over lanes.
__device__ __forceinline__ double mlp_forward(const float *__restrict__ P, double z, int lane, double &h1,
                                              double &h2, double &h3) {
    h1 = tanh((double)P[OFF_W1 + lane] * z + (double)P[OFF_B1 + lane]);
    double a = P[OFF_B2 + lane];
#pragma unroll 8
    for (int m = 0; m < H; ++m) a += (double)P[OFF_W2 + lane * H + m] * __shfl_sync(0xffffffffu, h1, m);
    h2 = tanh(a);
    a = P[OFF_B3 + lane];
#pragma unroll 8
    for (int m = 0; m < H; ++m) a += (double)P[OFF_W3 + lane * H + m] * __shfl_sync(0xffffffffu, h2, m);
    h3 = tanh(a);
    double g = (double)P[OFF_WO + lane] * h3;
    for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
    return g + (double)P[OFF_BO];
}

__device__ __forceinline__ double point_t(const TrainGeom &G, const double *__restrict__ qx, int p) {
    if (p < G.nf * G.W) {
        // visibility i at fractional cell offset f: a fixed grid of offsets, or
        // (Monte-Carlo training) offsets drawn afresh at every step
        int i = p / G.W, d = p - i * G.W;
        double f = G.mc ? mc_uniform(G.seed, G.step, i) : (i + 0.5) / G.nf;
        return ceil(f - 0.5 * G.W) + d - f;
    }
    return qx[p - G.nf * G.W] * 0.5 * G.W;          // Gauss-Legendre node on [-W/2, W/2]
}

// One training step (or a loss / gradient evaluation): params (FP32) and Adam
// moments in global memory; out[0] = loss before the update.
__global__ void __launch_bounds__(TTHREADS, 1)
k_window_step(TrainGeom G, float *__restrict__ P, float *__restrict__ m1, float *__restrict__ m2,
              const double *__restrict__ qx, const double *__restrict__ qw, double *__restrict__ out,
              float *__restrict__ grad_out) {
    __shared__ float sp[NPAR];
    __shared__ double phi[TNP], gphi[TNP];
    __shared__ double psi[TNXI], gpsi[TNXI];
    __shared__ double red[TWARPS];
    __shared__ double gsum[NPAR];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < NPAR; i += TTHREADS) { sp[i] = P[i]; gsum[i] = 0.0; }
    __syncthreads();
    // 1. window values at every point
    for (int p = warp; p < G.np; p += TWARPS) {
        double t = point_t(G, qx, p);
        double x = 2.0 * t / G.W;
        double z = x * x;
        double h1, h2, h3;
        double g = mlp_forward(sp, fmin(z, 1.0), lane, h1, h2, h3);
        double v = (fabs(t) < 0.5 * G.W) ? exp(es_log(z, G.beta) + g) : 0.0;
        if (lane == 0) phi[p] = v;
    }
    __syncthreads();
    // 2. psi(xi_j) by quadrature
    const double xi0 = -0.5 / G.sigma, dxi = (G.nxi > 1) ? (1.0 / G.sigma) / (G.nxi - 1) : 0.0;
    const int nT = G.nf * G.W;
    for (int j = tid; j < G.nxi; j += TTHREADS) {
        double xi = xi0 + j * dxi, s = 0;
        for (int q = 0; q < G.nq; ++q) s += qw[q] * 0.5 * G.W * phi[nT + q] * cos(2.0 * PI_D * xi * point_t(G, qx, nT + q));
        psi[j] = s;
        gpsi[j] = 0;
    }
    for (int p = tid; p < G.np; p += TTHREADS) gphi[p] = 0;
    __syncthreads();
    // 3. error and its gradient with respect to S (per (i, j) pair)
    double acc = 0;
    const int npair = G.nf * G.nxi;
    for (int k = tid; k < npair; k += TTHREADS) {
        int i = k / G.nxi, j = k - i * G.nxi;
        double xi = xi0 + j * dxi, sr = 0, si = 0;
        for (int d = 0; d < G.W; ++d) {
            double t = point_t(G, qx, i * G.W + d), s, c;
            sincos(2.0 * PI_D * xi * t, &s, &c);
            sr += phi[i * G.W + d] * c;
            si += phi[i * G.W + d] * s;
        }
        double er = sr / psi[j] - 1.0, ei = si / psi[j];
        acc += er * er + ei * ei;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    double m = 0;
    for (int w = 0; w < TWARPS; ++w) m += red[w];
    m /= npair;
    const double L = sqrt(m);
    // objective log(L): d log L / d m = 1 / (2 m)
    const double dm = 1.0 / (2.0 * m) / npair;
    for (int k = tid; k < npair; k += TTHREADS) {
        int i = k / G.nxi, j = k - i * G.nxi;
        double xi = xi0 + j * dxi, sr = 0, si = 0;
        double cs[TMAXW], sn[TMAXW];
        for (int d = 0; d < G.W; ++d) {
            double t = point_t(G, qx, i * G.W + d);
            sincos(2.0 * PI_D * xi * t, &sn[d], &cs[d]);
            sr += phi[i * G.W + d] * cs[d];
            si += phi[i * G.W + d] * sn[d];
        }
        double er = sr / psi[j] - 1.0, ei = si / psi[j];
        double gsr = dm * 2.0 * er / psi[j], gsi = dm * 2.0 * ei / psi[j];   // dObj/dSr, dObj/dSi
        double gp = -(gsr * sr + gsi * si) / psi[j];                         // dObj/dpsi_j
        atomicAdd(&gpsi[j], gp);
        for (int d = 0; d < G.W; ++d) atomicAdd(&gphi[i * G.W + d], gsr * cs[d] + gsi * sn[d]);
    }
    __syncthreads();
    for (int q = tid; q < G.nq; q += TTHREADS) {
        double tq = point_t(G, qx, nT + q), s = 0;
        for (int j = 0; j < G.nxi; ++j) s += gpsi[j] * qw[q] * 0.5 * G.W * cos(2.0 * PI_D * (xi0 + j * dxi) * tq);
        gphi[nT + q] += s;
    }
    __syncthreads();
    // 4. backward through exp and the MLP, warp per point, lane k <-> unit k
    double gW1 = 0, gB1 = 0, gB2 = 0, gB3 = 0, gWo = 0, gBo = 0;
    double gW2[H], gW3[H];                            // lane k: row k of dW2 / dW3 (FP64: terms cancel)
#pragma unroll
    for (int mm = 0; mm < H; ++mm) { gW2[mm] = 0; gW3[mm] = 0; }
    for (int p = warp; p < G.np; p += TWARPS) {
        double t = point_t(G, qx, p);
        if (!(fabs(t) < 0.5 * G.W)) continue;
        double x = 2.0 * t / G.W, z = fmin(x * x, 1.0);
        double h1, h2, h3;
        mlp_forward(sp, z, lane, h1, h2, h3);
        double dg = gphi[p] * phi[p];                  // d/dg exp(es + g) = phi
        // output layer
        gWo += dg * h3;
        gBo += dg;
        double d3 = dg * (double)sp[OFF_WO + lane] * (1.0 - h3 * h3);
        gB3 += d3;
#pragma unroll
        for (int mm = 0; mm < H; ++mm) gW3[mm] += d3 * __shfl_sync(0xffffffffu, h2, mm);
        double d2 = 0;
#pragma unroll 8
        for (int k = 0; k < H; ++k) d2 += (double)sp[OFF_W3 + k * H + lane] * __shfl_sync(0xffffffffu, d3, k);
        d2 *= (1.0 - h2 * h2);
        gB2 += d2;
#pragma unroll
        for (int mm = 0; mm < H; ++mm) gW2[mm] += d2 * __shfl_sync(0xffffffffu, h1, mm);
        double d1 = 0;
#pragma unroll 8
        for (int k = 0; k < H; ++k) d1 += (double)sp[OFF_W2 + k * H + lane] * __shfl_sync(0xffffffffu, d2, k);
        d1 *= (1.0 - h1 * h1);
        gB1 += d1;
        gW1 += d1 * z;
    }
    // per-warp partial gradients -> shared sums (lane k owns row k of W2/W3)
    atomicAdd(&gsum[OFF_W1 + lane], gW1);
    atomicAdd(&gsum[OFF_B1 + lane], gB1);
    atomicAdd(&gsum[OFF_B2 + lane], gB2);
    atomicAdd(&gsum[OFF_B3 + lane], gB3);
    atomicAdd(&gsum[OFF_WO + lane], gWo);
    if (lane == 0) atomicAdd(&gsum[OFF_BO], gBo);
#pragma unroll
    for (int mm = 0; mm < H; ++mm) {
        atomicAdd(&gsum[OFF_W2 + lane * H + mm], gW2[mm]);
        atomicAdd(&gsum[OFF_W3 + lane * H + mm], gW3[mm]);
    }
    __syncthreads();
    if (tid == 0) out[0] = L;
    if (grad_out)
        for (int i = tid; i < NPAR; i += TTHREADS) grad_out[i] = gsum[i];
    if (!G.want_update) return;
    // 5. Adam
    const double c1 = 1.0 - pow(G.b1, G.step), c2 = 1.0 - pow(G.b2, G.step);
    for (int i = tid; i < NPAR; i += TTHREADS) {
        double g = gsum[i];
        double a = G.b1 * m1[i] + (1.0 - G.b1) * g;
        double b = G.b2 * m2[i] + (1.0 - G.b2) * g * g;
        m1[i] = (float)a;
        m2[i] = (float)b;
        P[i] = (float)((double)sp[i] - G.lr * (a / c1) / (sqrt(b / c2) + G.eps));
    }
}

static double es_beta_for(int W, double sigma) {
    KernelParams kp;
    setup_kernel(std::pow(10.0, 1.0 - W), sigma, kp);       // the reference's beta rule for this width
    if (sigma == 2.0) {
        double bon = W == 2 ? 2.20 : W == 3 ? 2.26 : W == 4 ? 2.38 : 2.30;
        return bon * W;
    }
    return kp.beta / kp.kw * W;
}

struct TrainBuffers {
    float *P = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr;
    double *qx = nullptr, *qw = nullptr, *out = nullptr;
    ~TrainBuffers() {
        cudaFree(P); cudaFree(m1); cudaFree(m2); cudaFree(grad); cudaFree(qx); cudaFree(qw); cudaFree(out);
    }
};

static int train_setup(int W, double sigma, const float *params, TrainBuffers &B, TrainGeom &G) {
    if (W < 2 || W > TMAXW || !(sigma > 1.0)) return ERR_ARG;
    G = TrainGeom{};
    G.W = W; G.nf = TNF; G.nxi = TNXI; G.nq = TNQ; G.np = TNF * W + TNQ;
    G.beta = es_beta_for(W, sigma); G.sigma = sigma;
    G.b1 = 0.9; G.b2 = 0.999; G.eps = 1e-8;
    std::vector<double> x(TNQ), w(TNQ);
    gauss_legendre(TNQ, x.data(), w.data());
    if (cudaMalloc(&B.P, NPAR * 4) || cudaMalloc(&B.m1, NPAR * 4) || cudaMalloc(&B.m2, NPAR * 4) ||
        cudaMalloc(&B.grad, NPAR * 4) || cudaMalloc(&B.qx, TNQ * 8) || cudaMalloc(&B.qw, TNQ * 8) ||
        cudaMalloc(&B.out, 8)) {
        (void)cudaGetLastError();              // reported here, not by a later launch check
        return ERR_NOMEM;
    }
    cudaMemcpy(B.P, params, NPAR * 4, cudaMemcpyHostToDevice);
    cudaMemset(B.m1, 0, NPAR * 4);
    cudaMemset(B.m2, 0, NPAR * 4);
    cudaMemcpy(B.qx, x.data(), TNQ * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(B.qw, w.data(), TNQ * 8, cudaMemcpyHostToDevice);
    return OK;
}

// Host evaluation of the trained window (for tabulation and quadrature).
double mlp_window_value(int W, double beta, const float *P, double t) {
    if (!(std::fabs(t) < 0.5 * W)) return 0.0;
    double x = 2.0 * t / W, z = std::min(x * x, 1.0);
    double h1[H], h2[H], h3[H];
    for (int k = 0; k < H; ++k) h1[k] = std::tanh((double)P[OFF_W1 + k] * z + P[OFF_B1 + k]);
    for (int k = 0; k < H; ++k) {
        double a = P[OFF_B2 + k];
        for (int m = 0; m < H; ++m) a += (double)P[OFF_W2 + k * H + m] * h1[m];
        h2[k] = std::tanh(a);
    }
    for (int k = 0; k < H; ++k) {
        double a = P[OFF_B3 + k];
        for (int m = 0; m < H; ++m) a += (double)P[OFF_W3 + k * H + m] * h2[m];
        h3[k] = std::tanh(a);
    }
    double g = P[OFF_BO];
    for (int k = 0; k < H; ++k) g += (double)P[OFF_WO + k] * h3[k];
    return std::exp(-beta * z / (std::sqrt(std::max(1.0 - z, 0.0)) + 1.0) + g);
}

}  // namespace curig

using namespace curig;

extern "C" int curig_window_nparams(void) { return NPAR; }

extern "C" int curig_window_loss_grad(int W, double sigma, const float *params, double *loss, float *grad) {
    if (!params) return ERR_ARG;
    TrainBuffers B;
    TrainGeom G;
    int s = train_setup(W, sigma, params, B, G);
    if (s) return s;
    G.want_update = 0;
    count_launch();
    k_window_step<<<1, TTHREADS>>>(G, B.P, B.m1, B.m2, B.qx, B.qw, B.out, B.grad);
    if (cudaDeviceSynchronize() != cudaSuccess) return ERR_CUDA;
    if (loss) cudaMemcpy(loss, B.out, 8, cudaMemcpyDeviceToHost);
    if (grad) cudaMemcpy(grad, B.grad, NPAR * 4, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA;
}

static int train_loop(int W, double sigma, int iters, double lr, int mc, unsigned long long seed, float *params,
                      double *loss_hist) {
    if (!params || iters < 0) return ERR_ARG;
    TrainBuffers B;
    TrainGeom G;
    int s = train_setup(W, sigma, params, B, G);
    if (s) return s;
    G.want_update = 1;
    G.lr = lr;
    G.mc = mc;
    G.seed = seed;
    for (int it = 0; it < iters; ++it) {
        G.step = it + 1;
        count_launch();
        k_window_step<<<1, TTHREADS>>>(G, B.P, B.m1, B.m2, B.qx, B.qw, B.out, nullptr);
        if (loss_hist) cudaMemcpyAsync(&loss_hist[it], B.out, 8, cudaMemcpyDeviceToHost);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return ERR_CUDA;
    cudaMemcpy(params, B.P, NPAR * 4, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA;
}

extern "C" int curig_train_window(int W, double sigma, int iters, double lr, float *params,
                                  double *loss_hist) {
    return train_loop(W, sigma, iters, lr, 0, 0, params, loss_hist);
}

extern "C" int curig_train_window_mc(int W, double sigma, int iters, double lr, uint64_t seed, float *params,
                                     double *loss_hist) {
    return train_loop(W, sigma, iters, lr, 1, seed, params, loss_hist);
}

// Piecewise Chebyshev interpolation of the trained window (normalised to a
// maximum of 1) on the kw unit intervals -> [kw][degree+1] Horner coefficients.
extern "C" int curig_window_table(int W, double sigma, const float *params, int degree, double *coef) {
    if (!params || !coef || W < 2 || W > MAX_KW || degree < 1 || degree + 1 > MAX_POLY) return ERR_ARG;
    double beta = es_beta_for(W, sigma);
    double vmax = 0;
    for (int k = 0; k <= 4000; ++k) vmax = std::max(vmax, mlp_window_value(W, beta, params, -0.5 * W + W * k / 4000.0));
    if (!(vmax > 0)) return ERR_ARG;
    const int n = degree + 1;
    std::vector<double> fv(n), a(n), tkm1(n), tk(n), tkp1(n), m(n);
    for (int d = 0; d < W; ++d) {
        for (int j = 0; j < n; ++j) {
            double sn = std::cos(PI_D * (j + 0.5) / n);
            fv[j] = mlp_window_value(W, beta, params, (sn + 1.0) * 0.5 + d - 0.5 * W) / vmax;
        }
        for (int k = 0; k < n; ++k) {
            double s = 0;
            for (int j = 0; j < n; ++j) s += fv[j] * std::cos(PI_D * k * (j + 0.5) / n);
            a[k] = s * (k == 0 ? 1.0 : 2.0) / n;
        }
        std::fill(m.begin(), m.end(), 0.0);
        std::fill(tkm1.begin(), tkm1.end(), 0.0);
        std::fill(tk.begin(), tk.end(), 0.0);
        tkm1[0] = 1.0;
        if (n > 1) tk[1] = 1.0;
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
        for (int i = 0; i < n; ++i) coef[(size_t)d * n + i] = m[degree - i];
    }
    return OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of curig_window_loss_grad.
//
// Some callers cannot allocate device memory at the point where they need the
// window objective: processes whose device memory is reserved up front by
// another framework's pool (nothing is left for cudaMalloc), and real-time or
// embedded pipelines that forbid allocation after initialisation so that
// latency stays bounded.  This entry point runs the same kernel with its
// scratch (parameter copy, Adam moments, gradient, quadrature nodes and the
// loss) in a file-scope device array instead of cudaMalloc'd buffers.
//
// The array is g_window_scratch below: WSCRATCH_BYTES (64 KiB) per GPU, held
// by every GPU that loads the library until the process exits.  Host code must
// not hand the symbol itself to a kernel (in host code it is only a stand-in,
// not a device address); its device address is looked up once per device with
// cudaGetSymbolAddress, on the first call made with that device current.  Make
// that first call before any stream capture.  All calls share the one array and
// it keeps the last call's contents, so calls that overlap on the GPU (other
// threads, other streams) race; this entry point serialises on the legacy
// stream and returns only when its results are copied out.
// ---------------------------------------------------------------------------
namespace curig {

constexpr size_t WSCRATCH_BYTES = 64 * 1024;
static __device__ __align__(256) unsigned char g_window_scratch[WSCRATCH_BYTES];

// Device address of g_window_scratch on the current device, looked up once per
// device (std::call_once: threads making their first call on one device at the
// same time wait for a single lookup).  A failed lookup is retried on the next
// call.  The cached address belongs to the device's current context: after
// cudaDeviceReset the module is loaded again and this cache is stale, so a
// process that resets a device must not call this entry point afterwards.
constexpr int MAX_DEVICES = 64;
static std::once_flag g_scratch_once[MAX_DEVICES];
static std::atomic<void *> g_scratch_addr[MAX_DEVICES];
static std::mutex g_scratch_retry;

static void *window_scratch_ptr(int &status) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) { status = ERR_CUDA; return nullptr; }
    std::call_once(g_scratch_once[dev], [dev] {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_window_scratch) == cudaSuccess) g_scratch_addr[dev].store(p);
    });
    void *p = g_scratch_addr[dev].load();
    if (!p) {                                     // the first lookup failed: try again, serialised
        std::lock_guard<std::mutex> lk(g_scratch_retry);
        if (!g_scratch_addr[dev].load() && cudaGetSymbolAddress(&p, g_window_scratch) == cudaSuccess)
            g_scratch_addr[dev].store(p);
        p = g_scratch_addr[dev].load();
    }
    status = p ? OK : ERR_CUDA;
    return p;
}

}  // namespace curig

extern "C" int curig_window_loss_grad_static(int W, double sigma, const float *params, double *loss,
                                             float *grad) {
    using namespace curig;
    if (!params || W < 2 || W > TMAXW || !(sigma > 1.0)) return ERR_ARG;   // W beyond 12 does not fit
    // layout in the static array: P, m1, m2, grad (NPAR floats each), qx, qw (TNQ doubles), out (1 double)
    const size_t fbytes = NPAR * sizeof(float), nodes = TNQ * sizeof(double);
    const size_t o_m1 = fbytes, o_m2 = 2 * fbytes, o_g = 3 * fbytes;
    const size_t o_qx = (4 * fbytes + 255) & ~(size_t)255, o_qw = o_qx + nodes, o_out = o_qw + nodes;
    static_assert((4 * NPAR * sizeof(float) + 255) / 256 * 256 + 2 * TNQ * sizeof(double) + sizeof(double) <=
                      WSCRATCH_BYTES, "window scratch too small");
    int st = OK;
    unsigned char *base = static_cast<unsigned char *>(window_scratch_ptr(st));
    if (st != OK) return st;
    TrainGeom G{};
    G.W = W; G.nf = TNF; G.nxi = TNXI; G.nq = TNQ; G.np = TNF * W + TNQ;
    G.beta = es_beta_for(W, sigma); G.sigma = sigma;
    G.b1 = 0.9; G.b2 = 0.999; G.eps = 1e-8;
    G.want_update = 0;
    std::vector<double> x(TNQ), w(TNQ);
    gauss_legendre(TNQ, x.data(), w.data());
    float *P = reinterpret_cast<float *>(base), *m1 = reinterpret_cast<float *>(base + o_m1);
    float *m2 = reinterpret_cast<float *>(base + o_m2), *g = reinterpret_cast<float *>(base + o_g);
    double *qx = reinterpret_cast<double *>(base + o_qx), *qw = reinterpret_cast<double *>(base + o_qw);
    double *out = reinterpret_cast<double *>(base + o_out);
    // every region the kernel reads is written first; the moments (unused
    // without an update) are cleared so no stale state of an earlier call remains
    if (cudaMemcpy(P, params, fbytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m1, 0, 2 * fbytes) != cudaSuccess ||
        cudaMemcpy(qx, x.data(), nodes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(qw, w.data(), nodes, cudaMemcpyHostToDevice) != cudaSuccess)
        return ERR_CUDA;
    count_launch();
    k_window_step<<<1, TTHREADS>>>(G, P, m1, m2, qx, qw, out, g);
    if (cudaDeviceSynchronize() != cudaSuccess) return ERR_CUDA;
    if (loss && cudaMemcpy(loss, out, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return ERR_CUDA;
    if (grad && cudaMemcpy(grad, g, fbytes, cudaMemcpyDeviceToHost) != cudaSuccess) return ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA;
}
