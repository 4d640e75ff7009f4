// Host orchestration of one ms2dirty / dirty2ms plan: set points (w range,
// sizing, tile binning), execute (spread -> cuFFT -> screen+correction, or the
// adjoint chain), destroy.  Mirrors the reference's plan life cycle
// (gridder_setting / gridder_execution / gridder_destroy, src/astro/cugridder.cu:105-328)
// with device memory from the stream-ordered pool and no host synchronisation
// inside execute.
#include "plan.h"

#include <cudaTypedefs.h>        // PFN_cuTensorMapEncodeTiled

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>

namespace curig {

#define CU_TRY(x)                                   \
    do {                                            \
        cudaError_t e_ = (x);                       \
        if (e_ != cudaSuccess) {                    \
            p->last_error = cudaGetErrorString(e_); \
            return e_ == cudaErrorMemoryAllocation ? ERR_NOMEM : ERR_CUDA; \
        }                                           \
    } while (0)

template <typename X>
static cudaError_t dalloc(X **ptr, size_t bytes, cudaStream_t st) {
    *ptr = nullptr;
    if (bytes == 0) bytes = 16;
    return alloc_async((void **)ptr, bytes, st);
}

template <typename X>
static void dfree(X *&ptr, cudaStream_t st) {
    if (ptr) cudaFreeAsync((void *)ptr, st);
    ptr = nullptr;
}

static void keep_pool_memory(int device) {
    static bool done[64] = {false};
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        unsigned long long thr = ULLONG_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[device] = true;
}

static int encode_grid_map(Plan *p);

// ------------------------------------------------------------------ cuFFT plan cache
// Rank-1 batched in-place plans keyed by (device, length, element stride,
// batch distance, batch, precision, stream, host thread).  Handles are made
// without a work area of their own (auto-allocation off): every transform pass
// takes one from the stream-ordered pool on the plan's stream and returns it,
// so cached handles hold no large buffers and the pool's memory serves all of
// them.  A handle's stream and work area are per-call state, hence one handle
// per stream and host thread.  Plans hold references to the handles they use;
// released handles stay cached for the next plan of the same shape, at most
// FFT_KEEP of them (least recently released destroyed first), and
// fft_cache_trim (called by curig_release_memory) destroys all of them.
namespace {
struct FftEntry {
    cufftHandle h;
    size_t work;
    int refs;
    unsigned long long released;   // release tick, for the least-recently-released eviction
};
using FftKey = std::tuple<int, int, int, int, int, int, uintptr_t, std::thread::id>;
std::mutex g_fft_mu;
std::map<FftKey, FftEntry> g_fft;
unsigned long long g_fft_tick = 0;
constexpr int FFT_KEEP = 16;
}

static int fft_plan1(Plan *p, int n, int stride, int dist, int batch, int prec, cufftHandle &out, size_t &work) {
    std::lock_guard<std::mutex> lk(g_fft_mu);
    FftKey key = std::make_tuple(p->device, n, stride, dist, batch, prec, (uintptr_t)p->st,
                                 std::this_thread::get_id());
    auto it = g_fft.find(key);
    if (it != g_fft.end()) {
        ++it->second.refs;
        p->fft_keys.push_back(key);
        out = it->second.h;
        work = it->second.work;
        return OK;
    }
    cufftHandle h;
    if (cufftCreate(&h) != CUFFT_SUCCESS) return ERR_CUFFT;
    int nn[1] = {n}, emb[1] = {n};
    size_t ws = 0;
    if (cufftSetAutoAllocation(h, 0) != CUFFT_SUCCESS ||
        cufftMakePlanMany(h, 1, nn, emb, stride, dist, emb, stride, dist, prec ? CUFFT_C2C : CUFFT_Z2Z, batch,
                          &ws) != CUFFT_SUCCESS) {
        cufftDestroy(h);
        return ERR_CUFFT;
    }
    g_fft[key] = FftEntry{h, ws, 1, 0};
    p->fft_keys.push_back(key);
    out = h;
    work = ws;
    return OK;
}

// Drop the plan's references; keep at most FFT_KEEP unreferenced handles.
static void fft_release(Plan *p) {
    std::lock_guard<std::mutex> lk(g_fft_mu);
    for (const FftKey &k : p->fft_keys) {
        auto it = g_fft.find(k);
        if (it != g_fft.end() && it->second.refs > 0 && --it->second.refs == 0) it->second.released = ++g_fft_tick;
    }
    p->fft_keys.clear();
    for (;;) {
        int idle = 0;
        auto oldest = g_fft.end();
        for (auto it = g_fft.begin(); it != g_fft.end(); ++it)
            if (it->second.refs == 0) {
                ++idle;
                if (oldest == g_fft.end() || it->second.released < oldest->second.released) oldest = it;
            }
        if (idle <= FFT_KEEP) break;
        cufftDestroy(oldest->second.h);
        g_fft.erase(oldest);
    }
}

int fft_cache_trim() {
    std::lock_guard<std::mutex> lk(g_fft_mu);
    int n = 0;
    for (auto it = g_fft.begin(); it != g_fft.end();) {
        if (it->second.refs == 0) {
            cufftDestroy(it->second.h);
            it = g_fft.erase(it);
            ++n;
        } else {
            ++it;
        }
    }
    return n;
}

int fft_cache_size() {
    std::lock_guard<std::mutex> lk(g_fft_mu);
    return (int)g_fft.size();
}

// ------------------------------------------------------------------ learned-window registry
namespace {
std::mutex g_win_mu;
std::vector<Window> g_windows;
}

int registry_set_window(int kw, int degree, const double *coef, double eps_reached) {
    if (kw < 2 || kw > MAX_KW || degree < 1 || degree + 1 > MAX_POLY || !coef) return ERR_ARG;
    Window w;
    w.kind = 1;
    w.kw = kw;
    w.degree = degree;
    w.coef.assign(coef, coef + (size_t)kw * (degree + 1));
    w.eps_reached = eps_reached;
    std::lock_guard<std::mutex> lk(g_win_mu);
    for (auto &x : g_windows)
        if (x.kw == kw) { x = w; return OK; }
    g_windows.push_back(w);
    return OK;
}

bool registry_pick_window(double eps, Window &out) {
    std::lock_guard<std::mutex> lk(g_win_mu);
    const Window *best = nullptr;
    for (auto &x : g_windows)
        if (x.eps_reached <= eps && (!best || x.kw < best->kw)) best = &x;
    if (best) out = *best;                       // a copy: the registry may grow meanwhile
    return best != nullptr;
}

bool registry_get_window(int kw, Window &out) {
    std::lock_guard<std::mutex> lk(g_win_mu);
    for (auto &x : g_windows)
        if (x.kw == kw) {
            out = x;
            return true;
        }
    return false;
}

void registry_clear() {
    std::lock_guard<std::mutex> lk(g_win_mu);
    g_windows.clear();
}

// ------------------------------------------------------------------ instrumentation
namespace {
std::atomic<long long> g_launches{0};
std::atomic<bool> g_timing{false};
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }
void set_timing(bool on) { g_timing.store(on); }

static void mark(Plan *p, int slot) {
    if (!g_timing.load()) return;
    if (!p->ev[slot]) cudaEventCreate(&p->ev[slot]);
    cudaEventRecord(p->ev[slot], p->st);
    p->ev_recorded[slot] = true;
}

int plan_timings(Plan *p, double *out, int n) {
    static const int pairs[11][2] = {{EV_SET_BEGIN, EV_SET_END}, {EV_SET_WRANGE, EV_SET_END},
                                     {EV_M2D_BEGIN, EV_M2D_PREP}, {EV_M2D_PREP, EV_M2D_ZERO},
                                     {EV_M2D_ZERO, EV_M2D_SPREAD}, {EV_M2D_SPREAD, EV_M2D_FFT},
                                     {EV_M2D_FFT, EV_M2D_END}, {EV_D2M_BEGIN, EV_D2M_CORRECT},
                                     {EV_D2M_CORRECT, EV_D2M_FFT}, {EV_D2M_FFT, EV_D2M_INTERP},
                                     {EV_D2M_INTERP, EV_D2M_END}};
    if (cudaStreamSynchronize(p->st) != cudaSuccess) return ERR_CUDA;
    for (int i = 0; i < n && i < 11; ++i) {
        out[i] = -1.0;
        int a = pairs[i][0], b = pairs[i][1];
        float ms = 0;
        if (p->ev_recorded[a] && p->ev_recorded[b] && cudaEventElapsedTime(&ms, p->ev[a], p->ev[b]) == cudaSuccess)
            out[i] = ms;
    }
    return OK;
}

// ------------------------------------------------------------------ tile-load wait
// Polls of the interpolator's tile-load barrier before it gives up (about a
// second at the default); a test can shorten it and suppress the load so that
// the wait runs out on purpose (nothing is in flight when the CTA leaves).
namespace {
std::atomic<long long> g_tma_polls{DEFAULT_TMA_POLLS};
std::atomic<int> g_tma_noissue{0};
}

void set_tile_wait(long long polls, int noissue) {
    g_tma_polls.store(polls > 0 ? polls : DEFAULT_TMA_POLLS);
    g_tma_noissue.store(noissue ? 1 : 0);
}

// ms2dirty's weighted gather takes a scratch vis * wgt from the pool, or, when
// that allocation fails (or a test turns the scratch off), gathers vis and wgt
// in one pass.
namespace {
std::atomic<int> g_gather_scratch{1};
}

void set_gather_scratch(int on) { g_gather_scratch.store(on ? 1 : 0); }

template <typename T>
static void *gather_scratch(const void *d_wgt, long long M, cudaStream_t st) {
    void *vw = nullptr;
    if (d_wgt && g_gather_scratch.load() && dalloc(&vw, (size_t)M * 2 * sizeof(T), st) != cudaSuccess)
        vw = nullptr;
    return vw;
}

// ------------------------------------------------------------------ plan
int plan_create(int type, int nx, int ny, double psx, double psy, double eps, double sigma, int sign,
                const Options &opt, Plan **out) {
    *out = nullptr;
    if ((type != 1 && type != 2) || nx <= 0 || ny <= 0 || nx > (1 << 24) || ny > (1 << 24))
        return ERR_ARG;
    if (opt.precision != 0 && opt.precision != 1) return ERR_ARG;
    if (opt.smode < 0 || opt.smode > 3) return ERR_ARG;
    if (opt.w_term < 0 || opt.w_term > 1 || opt.grid_x < 0 || opt.grid_y < 0 || (opt.grid_x > 0) != (opt.grid_y > 0))
        return ERR_ARG;
    if (opt.bin_z < 0) return ERR_ARG;
    if (!std::isfinite(psx) || !std::isfinite(psy) || !(psx > 0) || !(psy > 0)) return ERR_ARG;
    KernelParams kp;
    int st = setup_kernel(eps, sigma, kp);
    if (st != OK) return st;
    Plan *p = new Plan();
    p->type = type;
    p->nx = nx;
    p->ny = ny;
    p->psx = psx;
    p->psy = psy;
    p->eps = eps;
    p->sigma = sigma;
    p->sign = sign >= 0 ? 1 : -1;
    p->opt = opt;
    p->st = opt.stream;
    if (cudaGetDevice(&p->device) != cudaSuccess) { delete p; return ERR_CUDA; }
    cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->device);
    keep_pool_memory(p->device);
    *out = p;
    return OK;
}

void plan_release_points(Plan *p) {
    cudaStream_t st = p->st;
    dfree(p->d_foc, st); dfree(p->d_quad, st); dfree(p->d_psi1, st); dfree(p->d_psi2, st); dfree(p->d_psi3, st);
    dfree(p->d_wcoef, st); dfree(p->d_bin_count, st); dfree(p->d_bin_start, st);
    dfree(p->d_nsub, st); dfree(p->d_sub_end, st); dfree(p->d_keys_in, st); dfree(p->d_kcount, st);
    dfree(p->d_cbin, st); p->dg.cbin = nullptr; p->dg.ccls = nullptr;
    dfree(p->d_idx, st); dfree(p->d_err, st); dfree(p->d_keys, st); dfree(p->d_scan, st);
    dfree(p->d_tmp, st); dfree(p->d_bcur, st);
    dfree(p->d_rec, st); dfree(p->d_ph, st); dfree(p->d_cs, st); dfree(p->d_grid, st);
    dfree(p->d_tgrid, st);
    fft_release(p);
    p->fft_hx = p->fft_hx_rest = p->fft_hy = p->fft_hy_rest = 0;
    p->ready = false;
    p->geom_ready = false;
}

int plan_destroy(Plan *p) {
    if (!p) return OK;
    plan_release_points(p);
    cudaStreamSynchronize(p->st);
    for (auto &e : p->ev)
        if (e) cudaEventDestroy(e);
    delete p;
    return OK;
}

// Bin / tile geometry: among the xy bin sizes whose tile (bin + kw halo, all
// w-planes when the w support never wraps, else 8- or 4-plane slabs) fits the
// shared-memory budget, the one with the smallest tile/core cell ratio (the
// halo overhead of zeroing, staging and flushing a tile).
// FP32 tile accumulation of the spreader (kernel numbering: 0 two-word int32,
// 1 float atomics, 2 one-word int32).  Automatic: one word when the requested
// epsilon is at least 1e-5 (its rounding, about 1.5e-6 relative, stays well
// inside the error budget), else the exact two-word form.  FP64 tiles take the
// exact three-word int32 form in every mode but 1 (double atomics).
static int tile_mode(const Plan *p) {
    switch (p->opt.smode) {
    case 1: return 1;
    case 2: return 2;
    case 3: return 0;
    default: return p->eps >= 1e-5 ? 2 : 0;
    }
}

static int choose_tiles(Plan *p, int esize, bool force_slabs) {
    const GridParams &gp = p->gp;
    const int kw = gp.kp.kw;
    TileGeom &t = p->tg;
    // FP32 spreader: int32 fixed point, two words (exact) or one word per component;
    // FP64: three-word int32 fixed point (exact)
    const int mode = tile_mode(p);
    t.fix = kw > TAB_KW ? 0 : esize == 4 ? (mode == 0 ? 1 : mode == 2 ? 2 : 0) : (mode != 1 ? 3 : 0);
    // FP32 tiles: two CTAs per SM (<= 112 KB each); FP64 fixed-point tiles: one
    // CTA per SM (its registers), so a larger tile with less halo
    size_t budget = p->opt.smem_budget ? p->opt.smem_budget
                    : (t.fix == 3 ? 200 * 1024 : t.fix ? 112 * 1024 : esize == 4 ? 72 * 1024 : 100 * 1024);
    int wdeg = p->win.kind ? p->win.degree : 0;
    // does the w support stay inside [0, nf3)?  (z grows monotonically with w;
    // same arithmetic as the binning kernel, which rejects any start outside)
    auto zstart = [&](double we) {
        double wp = (we - gp.i_center) / gp.gamma;
        double gz = (wp * INV_2PI + 0.5) * gp.nf3;
        return std::ceil(gz - 0.5 * kw);
    };
    double z0 = zstart(p->wmin_eff), z1 = zstart(p->wmax_eff);
    bool nowrap = gp.no_w || (!force_slabs && z0 >= 0.0 && z1 <= gp.nf3 - kw && gp.nf3 <= 4000);
    if (p->opt.n3 > 0) nowrap = false;                  // 3-D NUFFT: the third axis is periodic
    const int cand[] = {96, 64, 48, 32, 24, 20, 16, 12, 10, 8, 6, 4, 2};
    double best = 1e30;
    int bb = 0, bz_best = 0;
    auto consider = [&](int b, int bz, int tz) {
        if ((p->opt.bin_xy && b != p->opt.bin_xy) || b > gp.nf1 || b > gp.nf2) return;
        TileGeom q;
        q.tx = b + kw; q.ty = b + kw; q.tz = tz; q.fix = t.fix;
        if (q.tx > 1024 || tz > 4096 || tile_smem_bytes(q, esize, kw, wdeg) > budget) return;
        double ratio = (double)q.tx * q.ty * tz / ((double)b * b * bz);
        if (ratio < best - 1e-9) { best = ratio; bb = b; bz_best = bz; }
    };
    std::vector<int> edges(cand, cand + sizeof(cand) / sizeof(cand[0]));
    if (p->opt.bin_xy > 0) edges.assign(1, p->opt.bin_xy);   // a requested edge, any size
    if (p->opt.bin_z > 0 && !gp.no_w) {                 // requested slab depth
        if (p->opt.bin_z >= gp.nf3) return ERR_ARG;
        nowrap = false;
        for (int b : edges) consider(b, p->opt.bin_z, p->opt.bin_z + kw);
    } else {
        for (int b : edges) {
            if (nowrap) consider(b, gp.nf3, gp.nf3);
            for (int bz : {8, 4, 2}) if (bz < gp.nf3) consider(b, bz, bz + kw);
        }
    }
    if (!bb) return ERR_UNSUPPORTED;
    if (nowrap && bz_best == gp.nf3) {
        t.zpad = 0; t.bz = gp.nf3; t.tz = gp.nf3; t.nbz = 1;
    } else {
        t.zpad = 1; t.bz = bz_best; t.tz = bz_best + kw; t.nbz = (gp.nf3 + bz_best - 1) / bz_best;
    }
    t.bx = t.by = bb;
    t.tx = bb + kw; t.ty = bb + kw;
    t.nbx = (gp.nf1 + bb - 1) / bb;
    t.nby = (gp.nf2 + bb - 1) / bb;
    // visibilities per chunk: the two- and three-word tiles' per-cell headroom
    // assumes <= 4096; the one-word tiles bound their scale per chunk, so their
    // chunks may be larger: fewer tile flushes and reloads per bin (bench size,
    // 1.6e8 visibilities, ~4900 per bin: 67.4 ms per step at 4096, 66.2 at
    // 8192, 65.5-65.7 at 16384, no further change at 32768 or 65536)
    const int one_word = t.fix == 2;
    t.sub = std::min(p->opt.sub > 0 ? p->opt.sub : one_word ? 16384 : 4096, one_word ? 65536 : 4096);
    t.smem_bytes = tile_smem_bytes(t, esize, kw, wdeg);
    if (t.nbins() > INT_MAX / 2) return ERR_UNSUPPORTED;
    return OK;
}

static double key_to_double(unsigned long long k) {
    unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
    double d;
    std::memcpy(&d, &b, 8);
    return d;
}

int plan_setpts_geometry(Plan *p, long long nrow, int nchan, const double *du, const double *dv,
                         const double *dw, int stride, const double *h_freq) {
    if (!p) return ERR_ARG;
    if (nrow <= 0 || nchan <= 0 || !du || !dv || !dw || !h_freq || stride <= 0) return ERR_ARG;
    if (nrow * (long long)nchan >= INT_MAX) return ERR_ARG;
    for (int c = 0; c < nchan; ++c)
        if (!std::isfinite(h_freq[c]) || !(h_freq[c] > 0)) return ERR_NONFINITE;
    plan_release_points(p);
    cudaStream_t st = p->st;
    p->nrow = nrow;
    p->nchan = nchan;
    p->freq.assign(h_freq, h_freq + nchan);
    p->du = du; p->dv = dv; p->dw = dw; p->stride = stride;
    const int esize = p->opt.precision ? 4 : 8;

    // 1. raw w range -> effective range over channels (precomp.cu:61-69, utils.cu:42-53)
    mark(p, EV_SET_BEGIN);
    CU_TRY(dalloc(&p->d_keys, 2 * sizeof(unsigned long long), st));
    CU_TRY(dalloc(&p->d_err, sizeof(int), st));
    unsigned long long hk[2] = {ULLONG_MAX, 0ULL};
    CU_TRY(cudaMemcpyAsync(p->d_keys, hk, sizeof(hk), cudaMemcpyHostToDevice, st));
    CU_TRY(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
    launch_wrange(dw, stride, nrow, p->d_keys, p->d_err, st);
    int herr = 0;
    CU_TRY(cudaMemcpyAsync(hk, p->d_keys, sizeof(hk), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(&herr, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    CU_TRY(cudaGetLastError());
    if (herr & EF_NONFINITE) return ERR_NONFINITE;
    double wmin = key_to_double(hk[0]), wmax = key_to_double(hk[1]);
    double lo = INFINITY, hi = -INFINITY;
    std::vector<double> foc(nchan);
    for (int c = 0; c < nchan; ++c) {
        foc[c] = h_freq[c] / SPEEDOFLIGHT;
        double a = foc[c] * p->sign;
        for (double w : {wmin, wmax}) {
            double v = (w * a) * (2 * PI_D);
            lo = std::min(lo, v);
            hi = std::max(hi, v);
        }
    }
    p->wmin_eff = lo;
    p->wmax_eff = hi;

    // 2. sizes (cugridder.cu:29-101, 180-186) and window
    int kw_override = 0;
    p->win = Window();
    if (p->opt.window == 1) {
        if (!registry_pick_window(p->eps, p->win)) return ERR_WINDOW;
        kw_override = p->win.kw;
    }
    GridRequest req;
    req.grid_x = p->opt.grid_x;
    req.grid_y = p->opt.grid_y;
    req.no_w = p->opt.w_term == 1 || p->opt.n3 > 0;
    int s = grid_params(p->nx, p->ny, p->psx, p->psy, lo, hi, p->eps, p->sigma, p->sign, p->gp, kw_override, req);
    if (s != OK) return s;
    if (req.no_w && p->gp.kp.kw > TAB_KW) return ERR_UNSUPPORTED;   // thread-per-visibility kernels only
    if (p->opt.n3 > 0) {        // generic 3-D NUFFT: a periodic third axis of the NUFFT's own size
        GridParams &g3 = p->gp;
        g3.no_w = 0;
        g3.nf3 = get_num_cells(p->opt.n3, g3.kp);
        g3.gamma = 1.0;
        g3.i_center = g3.i_half = g3.o_center = g3.o_half = 0.0;
        g3.h = 2 * PI_D / g3.nf3;
    }
    p->win.kw = p->gp.kp.kw;
    // 3. correction tables (deconv.cu:60-197): psi1, psi2 on the grid, quadrature for psi3
    //    (psi1 / psi2 evaluated on the device from the quadrature: no host work
    //    while the GPU waits)
    const GridParams &gp = p->gp;
    double qx[MAX_QUAD], qg[MAX_QUAD];
    int nq = quadrature_terms(gp.kp, p->win, qx, qg);
    CU_TRY(dalloc(&p->d_foc, nchan * sizeof(double), st));
    CU_TRY(dalloc(&p->d_quad, 2 * MAX_QUAD * sizeof(double), st));
    CU_TRY(dalloc(&p->d_psi1, (gp.nf1 / 2 + 1) * sizeof(double), st));
    CU_TRY(dalloc(&p->d_psi2, (gp.nf2 / 2 + 1) * sizeof(double), st));
    CU_TRY(cudaMemcpyAsync(p->d_foc, foc.data(), nchan * sizeof(double), cudaMemcpyHostToDevice, st));
    CU_TRY(cudaMemcpyAsync(p->d_quad, qx, nq * sizeof(double), cudaMemcpyHostToDevice, st));
    CU_TRY(cudaMemcpyAsync(p->d_quad + MAX_QUAD, qg, nq * sizeof(double), cudaMemcpyHostToDevice, st));
    launch_psi_grid(gp.nf1 / 2 + 1, nq, p->d_quad, p->d_quad + MAX_QUAD, p->d_psi1, st);
    launch_psi_grid(gp.nf2 / 2 + 1, nq, p->d_quad, p->d_quad + MAX_QUAD, p->d_psi2, st);
    if (p->opt.n3 > 0) {
        CU_TRY(dalloc(&p->d_psi3, (gp.nf3 / 2 + 1) * sizeof(double), st));
        launch_psi_grid(gp.nf3 / 2 + 1, nq, p->d_quad, p->d_quad + MAX_QUAD, p->d_psi3, st);
    }
    if (p->win.kind == 1) {
        CU_TRY(dalloc(&p->d_wcoef, p->win.coef.size() * sizeof(double), st));
        CU_TRY(cudaMemcpyAsync(p->d_wcoef, p->win.coef.data(), p->win.coef.size() * sizeof(double),
                               cudaMemcpyHostToDevice, st));
    }
    DevCorr &cc = p->dc;
    cc.nx = p->nx; cc.ny = p->ny; cc.nf1 = gp.nf1; cc.nf2 = gp.nf2; cc.nf3 = gp.nf3;
    cc.psx = gp.pixsize_x; cc.psy = gp.pixsize_y; cc.o_center = gp.o_center; cc.i_center = gp.i_center;
    cc.gamma = gp.gamma; cc.h = gp.h; cc.nquad = nq; cc.no_w = gp.no_w;
    cc.qx = p->d_quad; cc.qg = p->d_quad + MAX_QUAD; cc.psi1 = p->d_psi1; cc.psi2 = p->d_psi2;
    cc.n3 = p->opt.n3; cc.psi3 = p->d_psi3; cc.dbg = p->d_err;

    // 4. fine grid and FFT plans
    size_t gbytes = (size_t)gp.nf1 * gp.nf2 * gp.nf3 * 2 * esize;
    CU_TRY(dalloc(&p->d_grid, gbytes, st));

    // 2-D transforms as two passes of contiguous rows: x rows of every plane
    // (length nf1), and y rows (length nf2) of the image's columns only, kept
    // transposed in d_tgrid [nf3][ny][nf2]
    CU_TRY(dalloc(&p->d_tgrid, (size_t)gp.nf3 * p->ny * gp.nf2 * 2 * esize, st));
    const long long nxrows = (long long)gp.nf2 * gp.nf3, nyrows = (long long)p->ny * gp.nf3;
    p->fft_bx = (int)std::max(1LL, std::min(nxrows, (1LL << 28) / gp.nf1));
    p->fft_bx_rest = (int)(nxrows % p->fft_bx);
    p->fft_by = (int)std::max(1LL, std::min(nyrows, (1LL << 28) / gp.nf2));
    p->fft_by_rest = (int)(nyrows % p->fft_by);
    const int pr = p->opt.precision;
    p->fft_hx_rest = p->fft_hy_rest = 0;
    p->fft_wx = p->fft_wx_rest = p->fft_wy = p->fft_wy_rest = 0;
    if (fft_plan1(p, gp.nf1, 1, gp.nf1, p->fft_bx, pr, p->fft_hx, p->fft_wx)) return ERR_CUFFT;
    if (p->fft_bx_rest &&
        fft_plan1(p, gp.nf1, 1, gp.nf1, p->fft_bx_rest, pr, p->fft_hx_rest, p->fft_wx_rest))
        return ERR_CUFFT;
    if (fft_plan1(p, gp.nf2, 1, gp.nf2, p->fft_by, pr, p->fft_hy, p->fft_wy)) return ERR_CUFFT;
    if (p->fft_by_rest &&
        fft_plan1(p, gp.nf2, 1, gp.nf2, p->fft_by_rest, pr, p->fft_hy_rest, p->fft_wy_rest))
        return ERR_CUFFT;
    p->geom_ready = true;
    return OK;
}

// Tiles, bins, the sort and the per-visibility records, on stream st (the
// plan's stream, or a second stream that the caller joins before executing).
int plan_setpts_bin(Plan *p, cudaStream_t st) {
    if (!p || !p->geom_ready) return ERR_ARG;
    const int esize = p->opt.precision ? 4 : 8;
    const long long nrow = p->nrow;
    const int nchan = p->nchan;
    const long long M = nrow * nchan;
    const double *du = p->du, *dv = p->dv, *dw = p->dw;
    const int stride = p->stride;
    int herr = 0, s;
    mark(p, EV_SET_WRANGE);
    bool force_slabs = false;
retry_tiles:
    s = choose_tiles(p, esize, force_slabs);
    if (s != OK) return s;
    const GridParams &gp = p->gp;
    const TileGeom &tg = p->tg;
    p->smem = tg.smem_bytes;
    {
        TileGeom ti = tg;
        ti.fix = 0;
        p->smem_interp = tile_smem_bytes(ti, esize, gp.kp.kw, p->win.kind ? p->win.degree : 0);
    }

    DevGeom &g = p->dg;
    g = DevGeom{};
    g.dbg = p->d_err;                                   // index checks of the bounds-checked build
    g.nf1 = gp.nf1; g.nf2 = gp.nf2; g.nf3 = gp.nf3;
    g.kw = gp.kp.kw; g.hkw = gp.kp.kw / 2;
    g.bx = tg.bx; g.by = tg.by; g.bz = tg.bz; g.nbx = tg.nbx; g.nby = tg.nby; g.nbz = tg.nbz;
    g.ibx = 1.0 / tg.bx; g.iby = 1.0 / tg.by; g.ibz = tg.bz > 0 ? 1.0 / tg.bz : 0.0;
    g.tx = tg.tx; g.ty = tg.ty; g.tz = tg.tz; g.zpad = tg.zpad; g.sub = tg.sub;
    g.sparse_n = p->opt.sparse < 0 ? 0 : p->opt.sparse > 0 ? p->opt.sparse
                 : esize == 4 ? DEFAULT_SPARSE_N : DEFAULT_SPARSE_N64;
    g.tpitch = (tg.tx + 2) & ~1;
    g.use_tma = 0;                          // set once the grid's TMA descriptor exists
    g.tma_polls = g_tma_polls.load();
    g.tma_test_noissue = g_tma_noissue.load();
    // row slabs (tile kernels only): bins of slab k are k * nbins_slab + bin
    int nslab = std::max(1, std::min(p->opt.slabs, MAX_SLABS));
    if (g.kw > TAB_KW || nrow < nslab || (long long)nslab * tg.nbins() > INT_MAX / 2) nslab = 1;
    p->nslab = nslab;
    g.nslab = nslab;
    g.nbins_slab = tg.nbins();
    g.nbins = nslab * tg.nbins();
    g.sub_lo = g.sub_hi = 0;
    p->slab_row.resize(nslab + 1);
    for (int k = 0; k <= nslab; ++k) p->slab_row[k] = slab_first_row(nrow, nslab, k);
    g.beta = gp.kp.beta; g.c = gp.kp.c;
    g.wkind = p->win.kind; g.wdeg = p->win.kind ? p->win.degree : 0;
    g.smode = tile_mode(p);
    g.no_w = gp.no_w;
    // window table for the thread-per-visibility kernels: the learned window, or
    // in FP32 the ES window as degree-(TAB_DEG-1) Horner polynomials
    p->htab.clear();
    if (g.kw <= TAB_KW && (p->win.kind == 1 || p->opt.precision == 1)) {
        Window src = p->win;
        if (src.kind == 0) es_horner_window(gp.kp, TAB_DEG - 1, src);
        if (src.degree <= TAB_DEG - 1) {
            p->htab.assign((size_t)g.kw * TAB_DEG, 0.0);
            for (int d = 0; d < g.kw; ++d)
                for (int i = 0; i <= src.degree; ++i)
                    p->htab[d * TAB_DEG + (TAB_DEG - 1 - src.degree) + i] = src.coef[(size_t)d * (src.degree + 1) + i];
            g.wkind = 1;
        }
    }
    // bounds on the window (sampled table maxima, 1% margin): per tap index d
    // over all offsets (wenv), of one tap's product (wmax3) and of the z factor;
    // they set the scale of the one-word fixed-point spreader
    g.wmax3 = 8.0f;
    g.wzmax = g.no_w ? 1.0f : 2.0f;
    for (int d = 0; d < TAB_KW; ++d) g.wenv[d] = 2.0f;
    if (!p->htab.empty()) {
        double wm = 0.0;
        for (int d = 0; d < g.kw; ++d) {
            double wd = 0.0;
            for (int k = 0; k <= 1024; ++k) {
                double x = 2.0 * k / 1024.0 - 1.0, v = 0.0;
                for (int i = 0; i < TAB_DEG; ++i) v = v * x + p->htab[(size_t)d * TAB_DEG + i];
                wd = std::max(wd, std::fabs(v));
            }
            g.wenv[d] = (float)(wd * 1.01);
            wm = std::max(wm, wd);
        }
        g.wmax3 = (float)(std::max(wm * wm, wm * wm * wm) * 1.01);   // 2-D: two factors
        if (!g.no_w) g.wzmax = (float)(wm * 1.01);
    }
    g.nrow = nrow; g.nchan = nchan; g.uvw_stride = stride;
    g.psx = gp.pixsize_x; g.psy = gp.pixsize_y; g.i_center = gp.i_center; g.gamma = gp.gamma;
    g.o_center = gp.o_center; g.sign = (double)gp.sign;

    // binning: key per visibility (bin, start-cell residue) and its count, a
    //    scan of the counts, per-bin bounds and sub-problems, the scatter of the
    //    input indices into bin order, then records in bin order (replaces the
    //    transpose and the unsorted point order of the reference)
    const long long nb = g.nbins;
    int binbits = 1;
    while ((1LL << binbits) < nb) ++binbits;
    // start-cell residue in the key: mod 16 for the FP32 tile kernels (their
    // class schedule needs it), mod 32 for the FP64 ones (bin-only keys beyond 31 bits)
    const bool f32tile = esize == 4 && g.kw <= TAB_KW;
    int cbits = f32tile ? 4 : (binbits + 5 <= 31 ? 5 : 0);
    if (binbits > 31 || binbits + cbits > 31) return ERR_UNSUPPORTED;
    g.cbits = cbits;
    const long long nkeys = nb << cbits;
    CU_TRY(dalloc(&p->d_keys_in, M * sizeof(unsigned), st));
    CU_TRY(dalloc(&p->d_kcount, nkeys * sizeof(int), st));
    CU_TRY(dalloc(&p->d_tmp, M * sizeof(int), st));
    CU_TRY(dalloc(&p->d_bcur, nb * sizeof(int), st));
    CU_TRY(dalloc(&p->d_bin_start, nb * sizeof(int), st));
    CU_TRY(dalloc(&p->d_bin_count, nb * sizeof(int), st));
    CU_TRY(dalloc(&p->d_nsub, nb * sizeof(int), st));
    CU_TRY(dalloc(&p->d_sub_end, nb * sizeof(int), st));
    CU_TRY(dalloc(&p->d_scan, std::max(scan_temp_ints(nkeys), scan_temp_ints(nb)) * sizeof(int), st));
    CU_TRY(cudaMemsetAsync(p->d_kcount, 0, nkeys * sizeof(int), st));
    launch_bin_count(g, du, dv, dw, p->d_foc, p->d_keys_in, p->d_kcount, p->d_err, st);
    scan_ints(p->d_kcount, p->d_kcount, nkeys, false, p->d_scan, st);          // in place: first position per key
    launch_bins_from_keys(p->d_kcount, p->d_scan, nb, cbits, g.sub, p->d_bin_start, p->d_bin_count, p->d_nsub,
                          p->d_bcur, st);
    launch_bin_scatter(M, p->d_keys_in, cbits, p->d_bcur, p->d_tmp, st);
    scan_ints(p->d_nsub, p->d_sub_end, nb, true, p->d_scan, st);
    p->slab_sub_end.assign(nslab, 0);               // last sub-problem end of every slab
    for (int k = 0; k < nslab; ++k)
        CU_TRY(cudaMemcpyAsync(&p->slab_sub_end[k], p->d_sub_end + (k + 1) * g.nbins_slab - 1, sizeof(int),
                               cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(&herr, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    CU_TRY(cudaGetLastError());
    if (herr & EF_NONFINITE) return ERR_NONFINITE;
    if (herr & EF_BOUNDS) {
        p->last_error = "an index left its buffer (bounds-checked build)";
        return ERR_GENERIC;
    }
    if (herr & EF_RANGE) {
        if (p->tg.zpad == 0 && !force_slabs) {          // a w support reached the grid edge: use z slabs
            force_slabs = true;
            herr = 0;
            CU_TRY(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
            dfree(p->d_keys_in, st); dfree(p->d_kcount, st); dfree(p->d_tmp, st); dfree(p->d_bcur, st);
            dfree(p->d_bin_start, st); dfree(p->d_bin_count, st);
            dfree(p->d_nsub, st); dfree(p->d_sub_end, st); dfree(p->d_scan, st);
            goto retry_tiles;
        }
        return ERR_GENERIC;
    }
    CU_TRY(dalloc(&p->d_rec, M * 4 * (size_t)esize, st));
    CU_TRY(dalloc(&p->d_ph, M * 2 * (size_t)esize, st));
    CU_TRY(dalloc(&p->d_cs, M * 2 * (size_t)esize, st));
    CU_TRY(dalloc(&p->d_idx, M * sizeof(int), st));
    // each bin's visibilities (tmp) placed by residue; the key cursors start at
    // the scanned key counts
    if (p->opt.precision)
        launch_records<float>(g, du, dv, dw, p->d_foc, p->d_tmp, M, p->d_kcount, p->d_rec, p->d_ph, p->d_idx, st);
    else
        launch_records<double>(g, du, dv, dw, p->d_foc, p->d_tmp, M, p->d_kcount, p->d_rec, p->d_ph, p->d_idx, st);
    dfree(p->d_keys_in, st);
    dfree(p->d_scan, st);
    dfree(p->d_tmp, st);
    dfree(p->d_bcur, st);
    // the key cursors now hold the end of every (bin, residue) run: the class
    // boundaries of the FP32 tile kernels; every sub-problem's bin
    if (f32tile) {
        g.ccls = p->d_kcount;
    } else {
        dfree(p->d_kcount, st);
        g.ccls = nullptr;
    }
    const int nsubs = p->slab_sub_end.empty() ? 0 : p->slab_sub_end.back();
    g.cbin = nullptr;
    if (nsubs > 0) {
        CU_TRY(dalloc(&p->d_cbin, (size_t)nsubs * sizeof(int), st));
        launch_chunk_bins(nb, p->d_sub_end, p->d_cbin, st);
        g.cbin = p->d_cbin;
    }
    // TMA descriptor of the grid for the interpolator's interior tile boxes
    // ({tpitch, ty, tz} cells in 8-byte elements: one per FP32 cell, two per
    // FP64 cell; box edges <= 256 elements, x starts 16-byte aligned)
    if (g.tpitch * (p->opt.precision ? 1 : 2) <= 256 && g.ty <= 256 && g.tz <= 256)
        g.use_tma = encode_grid_map(p) == OK ? 1 : 0;
    mark(p, EV_SET_END);
    p->ready = true;
    return OK;
}

int plan_setpts(Plan *p, long long nrow, int nchan, const double *du, const double *dv,
                const double *dw, int stride, const double *h_freq) {
    int s = plan_setpts_geometry(p, nrow, nchan, du, dv, dw, stride, h_freq);
    return s != OK ? s : plan_setpts_bin(p, p->st);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void *f = nullptr;                            // initialised once, thread-safe
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        return nullptr;
    }();
    return fn;
}

static int encode_grid_map(Plan *p) {
    auto enc = tensor_map_encoder();
    if (!enc) return ERR_UNSUPPORTED;
    const GridParams &gp = p->gp;
    const DevGeom &g = p->dg;
    // 8-byte elements: one complex cell in FP32, one component in FP64 (a cell = 2 elements)
    const int per = p->opt.precision ? 1 : 2;
    cuuint64_t dims[3] = {(cuuint64_t)gp.nf1 * per, (cuuint64_t)gp.nf2, (cuuint64_t)gp.nf3};
    cuuint64_t strides[2] = {(cuuint64_t)gp.nf1 * per * 8, (cuuint64_t)gp.nf1 * gp.nf2 * per * 8};
    cuuint32_t box[3] = {(cuuint32_t)(g.tpitch * per), (cuuint32_t)g.ty, (cuuint32_t)g.tz};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&p->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, p->d_grid, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? OK : ERR_UNSUPPORTED;
}

static int fft_exec(Plan *p, cufftHandle h, void *base, long long offset, int dir) {
    if (cufftSetStream(h, p->st) != CUFFT_SUCCESS) return ERR_CUFFT;
    cufftResult r;
    if (p->opt.precision) {
        cufftComplex *d = reinterpret_cast<cufftComplex *>(base) + offset;
        r = cufftExecC2C(h, d, d, dir);
    } else {
        cufftDoubleComplex *d = reinterpret_cast<cufftDoubleComplex *>(base) + offset;
        r = cufftExecZ2Z(h, d, d, dir);
    }
    return r == CUFFT_SUCCESS ? OK : ERR_CUFFT;
}

// Batched contiguous row transforms of length n over nrows rows of buf, with
// one work area from the stream-ordered pool for the pass.
static int fft_rows(Plan *p, void *buf, long long nrows, int n, cufftHandle h, size_t wh, int b,
                    cufftHandle h_rest, size_t wr, int b_rest, int dir) {
    const size_t ws = std::max(wh, h_rest ? wr : (size_t)0);
    void *work = nullptr;
    if (ws) CU_TRY(alloc_async(&work, ws, p->st));
    int s = OK;
    if (cufftSetWorkArea(h, work) != CUFFT_SUCCESS || (h_rest && cufftSetWorkArea(h_rest, work) != CUFFT_SUCCESS))
        s = ERR_CUFFT;
    for (long long r = 0; s == OK && r < nrows;) {
        const bool full = nrows - r >= b;
        s = fft_exec(p, full ? h : h_rest, buf, r * n, dir);
        r += full ? b : b_rest;
    }
    if (work) cudaFreeAsync(work, p->st);
    return s;
}

// 2-D transform of every plane (cuft.cu:127-143) restricted to what the image
// needs.  ms2dirty: x rows of the whole grid, then the image's columns are
// transposed into d_tgrid and transformed along y there (the correction reads
// d_tgrid).  dirty2ms: the correction writes d_tgrid, y rows are transformed,
// the columns go back into the grid (other columns zeroed), then x rows.
template <typename T>
static int plane_fft(Plan *p, int dir, bool m2d) {
    const GridParams &gp = p->gp;
    const long long nx_rows = (long long)gp.nf2 * gp.nf3, ny_rows = (long long)p->ny * gp.nf3;
    int s;
    if (m2d) {
        if ((s = fft_rows(p, p->d_grid, nx_rows, gp.nf1, p->fft_hx, p->fft_wx, p->fft_bx, p->fft_hx_rest, p->fft_wx_rest,
                      p->fft_bx_rest, dir)))
            return s;
        launch_cols_to_t<T>(p->ny, gp.nf1, gp.nf2, gp.nf3, p->d_grid, p->d_tgrid, p->st);
        return fft_rows(p, p->d_tgrid, ny_rows, gp.nf2, p->fft_hy, p->fft_wy, p->fft_by, p->fft_hy_rest, p->fft_wy_rest,
                      p->fft_by_rest, dir);
    }
    if ((s = fft_rows(p, p->d_tgrid, ny_rows, gp.nf2, p->fft_hy, p->fft_wy, p->fft_by, p->fft_hy_rest, p->fft_wy_rest,
                      p->fft_by_rest, dir)))
        return s;
    launch_t_to_grid<T>(p->ny, gp.nf1, gp.nf2, gp.nf3, p->d_tgrid, p->d_grid, p->st);
    return fft_rows(p, p->d_grid, nx_rows, gp.nf1, p->fft_hx, p->fft_wx, p->fft_bx, p->fft_hx_rest, p->fft_wx_rest,
                      p->fft_bx_rest, dir);
}

template <typename T>
static int execute_t(Plan *p, int type, void *d_vis, const void *d_wgt, void *d_dirty) {
    cudaStream_t st = p->st;
    const DevGeom &g = p->dg;
    const GridParams &gp = p->gp;
    size_t gbytes = (size_t)gp.nf1 * gp.nf2 * gp.nf3 * 2 * sizeof(T);
    const long long M = p->nrow * p->nchan;
    int s;
    if (type == 1) {
        mark(p, EV_M2D_BEGIN);
        void *vw = gather_scratch<T>(d_wgt, M, st);   // vis * wgt in input order (the pool's memory)
        launch_vis_prep<T>(0, M, p->d_idx, p->d_ph, d_vis, d_wgt, vw, p->d_cs, st);
        dfree(vw, st);
        mark(p, EV_M2D_PREP);
        CU_TRY(cudaMemsetAsync(p->d_grid, 0, gbytes, st));
        mark(p, EV_M2D_ZERO);
        const VisIO io{p->d_idx, p->d_ph, d_wgt, d_vis};
        s = launch_spread<T>(g, p->smem, p->d_bin_start, p->d_bin_count, p->d_sub_end, p->d_rec, p->d_cs,
                             p->d_grid, p->d_wcoef, p->htab.empty() ? nullptr : p->htab.data(), io, M, p->nsm,
                             st);
        if (s) return s;
        mark(p, EV_M2D_SPREAD);
        s = plane_fft<T>(p, CUFFT_INVERSE, true);    // +1, cuft.cu:127-143
        if (s) return s;
        mark(p, EV_M2D_FFT);
        if (p->opt.n3 > 0) launch_correct3_m2d<T>(p->dc, p->d_tgrid, d_dirty, st);
        else launch_correct_m2d<T>(p->dc, p->d_tgrid, d_dirty, st);
        mark(p, EV_M2D_END);
    } else {
        mark(p, EV_D2M_BEGIN);
        launch_zero_tpad<T>(p->nx, p->ny, gp.nf2, gp.nf3, p->d_tgrid, st);
        if (p->opt.n3 > 0) launch_correct3_d2m<T>(p->dc, d_dirty, p->d_tgrid, st);
        else launch_correct_d2m<T>(p->dc, d_dirty, p->d_tgrid, st);
        mark(p, EV_D2M_CORRECT);
        s = plane_fft<T>(p, CUFFT_FORWARD, false);   // -1
        if (s) return s;
        mark(p, EV_D2M_FFT);
        const VisIO io{p->d_idx, p->d_ph, nullptr, d_vis};   // weights applied after the scatter
        s = launch_interp<T>(g, p->smem_interp, p->d_bin_start, p->d_bin_count, p->d_sub_end, p->d_rec, p->d_grid,
                             p->d_cs, p->d_wcoef, p->htab.empty() ? nullptr : p->htab.data(), io, M, &p->tmap,
                             p->d_err, p->nsm, st);
        if (s) return s;
        mark(p, EV_D2M_INTERP);                  // the scatter runs inside the interpolator
        launch_vis_scale<T>(0, M, d_vis, d_wgt, st);
        mark(p, EV_D2M_END);
    }
    CU_TRY(cudaGetLastError());
    return OK;
}

template <typename T>
static int execute_slabs_t(Plan *p, int type, void *d_vis, const void *d_wgt, void *d_dirty,
                           const cudaEvent_t *ready, const cudaEvent_t *done, int nev, bool prologue_done) {
    cudaStream_t st = p->st;
    const GridParams &gp = p->gp;
    const int ns = p->nslab;
    if (nev != ns && !(ns == 1 && nev > 0)) return ERR_ARG;
    auto wait_slab = [&](int k) {
        if (!ready) return cudaSuccess;
        if (ns == nev) return cudaStreamWaitEvent(st, ready[k], 0);
        for (int e = 0; e < nev; ++e) {               // one plan slab: every upload
            cudaError_t r = cudaStreamWaitEvent(st, ready[e], 0);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    };
    auto done_slab = [&](int k) {
        if (!done) return cudaSuccess;
        if (ns == nev) return cudaEventRecord(done[k], st);
        for (int e = 0; e < nev; ++e) {
            cudaError_t r = cudaEventRecord(done[e], st);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    };
    // launch geometry of slab k: its sub-problem window
    auto slab_geom = [&](int k, DevGeom &gk) {
        gk = p->dg;
        gk.sub_lo = k ? p->slab_sub_end[k - 1] : 0;
        gk.sub_hi = p->slab_sub_end[k];
        return gk.sub_hi > gk.sub_lo;
    };
    const VisIO io{p->d_idx, p->d_ph, d_wgt, d_vis};
    const double *ht = p->htab.empty() ? nullptr : p->htab.data();
    int s;
    if (type == 1) {
        const size_t gbytes = (size_t)gp.nf1 * gp.nf2 * gp.nf3 * 2 * sizeof(T);
        CU_TRY(cudaMemsetAsync(p->d_grid, 0, gbytes, st));
        void *vw = gather_scratch<T>(d_wgt, p->nrow * p->nchan, st);   // vis * wgt in input order
        for (int k = 0; k < ns; ++k) {
            if (cudaError_t e = wait_slab(k)) {
                dfree(vw, st);
                CU_TRY(e);
            }
            const long long i0 = p->slab_row[k] * p->nchan, i1 = p->slab_row[k + 1] * p->nchan;
            launch_vis_prep<T>(i0, i1 - i0, p->d_idx, p->d_ph, d_vis, d_wgt, vw, p->d_cs, st);
            DevGeom gk;
            if (slab_geom(k, gk) &&
                (s = launch_spread<T>(gk, p->smem, p->d_bin_start, p->d_bin_count, p->d_sub_end, p->d_rec, p->d_cs,
                                      p->d_grid, p->d_wcoef, ht, io, p->nrow * p->nchan, p->nsm, st))) {
                dfree(vw, st);
                return s;
            }
        }
        dfree(vw, st);
        if ((s = plane_fft<T>(p, CUFFT_INVERSE, true))) return s;
        launch_correct_m2d<T>(p->dc, p->d_tgrid, d_dirty, st);
    } else {
        if (!prologue_done) {
            launch_zero_tpad<T>(p->nx, p->ny, gp.nf2, gp.nf3, p->d_tgrid, st);
            launch_correct_d2m<T>(p->dc, d_dirty, p->d_tgrid, st);
            if ((s = plane_fft<T>(p, CUFFT_FORWARD, false))) return s;
        }
        const VisIO io_out{p->d_idx, p->d_ph, nullptr, d_vis};   // weights applied after the scatter
        for (int k = 0; k < ns; ++k) {
            CU_TRY(wait_slab(k));
            DevGeom gk;
            if (slab_geom(k, gk) &&
                (s = launch_interp<T>(gk, p->smem_interp, p->d_bin_start, p->d_bin_count, p->d_sub_end, p->d_rec,
                                      p->d_grid, p->d_cs, p->d_wcoef, ht, io_out, p->nrow * p->nchan, &p->tmap,
                                      p->d_err, p->nsm, st)))
                return s;
            const long long i0 = p->slab_row[k] * p->nchan, i1 = p->slab_row[k + 1] * p->nchan;
            launch_vis_scale<T>(i0, i1 - i0, d_vis, d_wgt, st);
            CU_TRY(done_slab(k));
        }
    }
    CU_TRY(cudaGetLastError());
    return OK;
}

int plan_execute_slabs(Plan *p, int type, void *d_vis, const void *d_wgt, void *d_dirty,
                       const cudaEvent_t *ready, const cudaEvent_t *done, int nev, bool prologue_done) {
    if (!p || !p->ready || !d_vis || !d_dirty || (type != 1 && type != 2)) return ERR_ARG;
    return p->opt.precision
               ? execute_slabs_t<float>(p, type, d_vis, d_wgt, d_dirty, ready, done, nev, prologue_done)
               : execute_slabs_t<double>(p, type, d_vis, d_wgt, d_dirty, ready, done, nev, prologue_done);
}

template <typename T>
static int d2m_prologue_t(Plan *p, const void *d_dirty, cudaEvent_t image_ready) {
    const GridParams &gp = p->gp;
    launch_zero_tpad<T>(p->nx, p->ny, gp.nf2, gp.nf3, p->d_tgrid, p->st);   // needs no image
    if (image_ready) CU_TRY(cudaStreamWaitEvent(p->st, image_ready, 0));
    launch_correct_d2m<T>(p->dc, d_dirty, p->d_tgrid, p->st);
    int s = plane_fft<T>(p, CUFFT_FORWARD, false);
    if (s) return s;
    CU_TRY(cudaGetLastError());
    return OK;
}

int plan_d2m_prologue(Plan *p, const void *d_dirty, cudaEvent_t image_ready) {
    if (!p || !p->geom_ready || !d_dirty) return ERR_ARG;
    return p->opt.precision ? d2m_prologue_t<float>(p, d_dirty, image_ready)
                            : d2m_prologue_t<double>(p, d_dirty, image_ready);
}

// Error flags raised by kernels of earlier executes (an interpolator tile load
// that never completed); waits for the plan's stream.
int plan_device_status(Plan *p) {
    if (!p || !p->d_err) return OK;
    int herr = 0;
    CU_TRY(cudaMemcpyAsync(&herr, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, p->st));
    CU_TRY(cudaStreamSynchronize(p->st));
    if (herr & EF_TIMEOUT) {
        p->last_error = "a tile load did not complete (timed out)";
        return ERR_CUDA;
    }
    if (herr & EF_BOUNDS) {
        p->last_error = "an index left its buffer (bounds-checked build)";
        return ERR_GENERIC;
    }
    return OK;
}

int plan_execute(Plan *p, void *d_vis, const void *d_wgt, void *d_dirty, int type) {
    if (!p || !p->ready || !d_vis || !d_dirty) return ERR_ARG;
    if (type == 0) type = p->type;
    if (type != 1 && type != 2) return ERR_ARG;
    return p->opt.precision ? execute_t<float>(p, type, d_vis, d_wgt, d_dirty)
                            : execute_t<double>(p, type, d_vis, d_wgt, d_dirty);
}

}  // namespace curig
