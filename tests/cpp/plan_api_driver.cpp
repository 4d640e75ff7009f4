// C++ caller of the plan API with the reference's names (include/cugridder.h),
// written the way the reference's own test mains drive it
// (test/w_s_gridder_test.cu:105-222,274 and test/w_s_degridder_test.cu:195-229):
// host u/v/w/vis/frequency/weight arrays from malloc, device copies of u, v, w
// and vis, a visibility struct with sign -1, gridder_setting, plan->fk set by
// the caller, gridder_execution, and gridder_destroy (which frees the host
// arrays held in gridder_plan->kv, as the reference's does).
//
//   plan_api_driver <in.bin> <out.bin>
//
// in.bin:  int32 nrow, nx, ny; float64 fov, freq, eps, sigma;
//          float64 u[nrow], v[nrow], w[nrow]; complex128 vis[nrow];
//          float64 wgt[nrow]; complex128 dirty[nx][ny]
// out.bin: complex128 dirty_w[nx][ny], dirty_nw[nx][ny], vis_w[nrow], vis_nw[nrow]
//          (ms2dirty with / without weights, dirty2ms with / without weights)
// Exit status: 0 ok, 2 I/O error, 3 CUDA error, 10 + status of a failing call.
#include "cugridder.h"

#include <cuda_runtime.h>

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef std::complex<double> CPX;

#define CUDA_OK(x)                                                         \
    do {                                                                   \
        if ((x) != cudaSuccess) {                                          \
            std::fprintf(stderr, "CUDA error at %s:%d\n", __FILE__, __LINE__); \
            std::exit(3);                                                  \
        }                                                                  \
    } while (0)

struct Inputs {
    int nrow = 0, nx = 0, ny = 0;
    double fov = 0, freq = 0, eps = 0, sigma = 0;
    std::vector<double> u, v, w, wgt;
    std::vector<CPX> vis, dirty;
};

static bool read_inputs(const char *path, Inputs &in) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    int hdr[3];
    double d[4];
    bool ok = std::fread(hdr, sizeof(int), 3, f) == 3 && std::fread(d, sizeof(double), 4, f) == 4;
    if (ok) {
        in.nrow = hdr[0]; in.nx = hdr[1]; in.ny = hdr[2];
        in.fov = d[0]; in.freq = d[1]; in.eps = d[2]; in.sigma = d[3];
        const size_t n = in.nrow, npix = (size_t)in.nx * in.ny;
        in.u.resize(n); in.v.resize(n); in.w.resize(n); in.wgt.resize(n);
        in.vis.resize(n); in.dirty.resize(npix);
        ok = std::fread(in.u.data(), 8, n, f) == n && std::fread(in.v.data(), 8, n, f) == n &&
             std::fread(in.w.data(), 8, n, f) == n && std::fread(in.vis.data(), 16, n, f) == n &&
             std::fread(in.wgt.data(), 8, n, f) == n && std::fread(in.dirty.data(), 16, npix, f) == npix;
    }
    std::fclose(f);
    return ok;
}

template <typename X>
static X *host_copy(const std::vector<X> &src) {      // malloc'd: gridder_destroy frees it
    X *p = static_cast<X *>(std::malloc(src.size() * sizeof(X)));
    std::memcpy(p, src.data(), src.size() * sizeof(X));
    return p;
}

// One plan life cycle in the reference's order.  direction 1: vis -> image
// (result in image), 0: image -> vis (result in vis_out).
static int run(const Inputs &in, int direction, bool with_wgt, std::vector<CPX> &image, std::vector<CPX> &vis_out) {
    const int nrow = in.nrow, nx = in.nx, ny = in.ny;
    double *d_u, *d_v, *d_w;
    cuDoubleComplex *d_vis, *d_fk;
    CUDA_OK(cudaMalloc((void **)&d_u, nrow * sizeof(double)));
    CUDA_OK(cudaMalloc((void **)&d_v, nrow * sizeof(double)));
    CUDA_OK(cudaMalloc((void **)&d_w, nrow * sizeof(double)));
    CUDA_OK(cudaMalloc((void **)&d_vis, nrow * sizeof(cuDoubleComplex)));
    CUDA_OK(cudaMemcpy(d_u, in.u.data(), nrow * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_v, in.v.data(), nrow * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_w, in.w.data(), nrow * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_vis, in.vis.data(), nrow * sizeof(cuDoubleComplex), cudaMemcpyHostToDevice));

    curafft_plan *plan = new curafft_plan();
    ragridder_plan *gplan = new ragridder_plan();
    std::memset(plan, 0, sizeof(curafft_plan));
    std::memset(gplan, 0, sizeof(ragridder_plan));
    visibility *pv = static_cast<visibility *>(std::malloc(sizeof(visibility)));
    pv->u = host_copy(in.u);
    pv->v = host_copy(in.v);
    pv->w = host_copy(in.w);
    pv->vis = host_copy(in.vis);
    pv->frequency = static_cast<double *>(std::malloc(sizeof(double)));
    pv->frequency[0] = in.freq;
    pv->weight = with_wgt ? host_copy(in.wgt) : nullptr;
    pv->flag = nullptr;
    pv->pirange = 0;
    pv->sign = -1;
    int ier = gridder_setting(ny, nx, 0, 0, 1, in.eps, direction, in.sigma, 0, 1, nrow, 1, in.fov, pv, d_u, d_v,
                              d_w, d_vis, plan, gplan);
    std::free(pv);
    if (ier != 0) return 10 + ier;
    CUDA_OK(cudaMalloc((void **)&d_fk, sizeof(cuDoubleComplex) * nx * ny));
    plan->fk = d_fk;
    if (direction == 0)
        CUDA_OK(cudaMemcpy(d_fk, in.dirty.data(), sizeof(cuDoubleComplex) * nx * ny, cudaMemcpyHostToDevice));
    ier = gridder_execution(plan, gplan);
    if (ier != 0) return 10 + ier;
    if (direction == 1) {
        image.resize((size_t)nx * ny);
        CUDA_OK(cudaMemcpy(image.data(), d_fk, sizeof(cuDoubleComplex) * nx * ny, cudaMemcpyDeviceToHost));
    } else {
        vis_out.resize(nrow);
        CUDA_OK(cudaMemcpy(vis_out.data(), plan->d_c, sizeof(cuDoubleComplex) * nrow, cudaMemcpyDeviceToHost));
    }
    ier = gridder_destroy(plan, gplan);
    if (ier != 0) return 10 + ier;
    delete plan;
    delete gplan;
    cudaFree(d_u);
    cudaFree(d_v);
    cudaFree(d_w);
    cudaFree(d_vis);
    cudaFree(d_fk);
    return 0;
}

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    Inputs in;
    if (!read_inputs(argv[1], in)) return 2;
    std::vector<CPX> dw, dnw, vw, vnw, unused;
    int s;
    if ((s = run(in, 1, true, dw, unused)) || (s = run(in, 1, false, dnw, unused)) ||
        (s = run(in, 0, true, unused, vw)) || (s = run(in, 0, false, unused, vnw)))
        return s;
    FILE *f = std::fopen(argv[2], "wb");
    if (!f) return 2;
    bool ok = std::fwrite(dw.data(), 16, dw.size(), f) == dw.size() &&
              std::fwrite(dnw.data(), 16, dnw.size(), f) == dnw.size() &&
              std::fwrite(vw.data(), 16, vw.size(), f) == vw.size() &&
              std::fwrite(vnw.data(), 16, vnw.size(), f) == vnw.size();
    std::fclose(f);
    return ok ? 0 : 2;
}
