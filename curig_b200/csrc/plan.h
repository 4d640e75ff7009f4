// Plan object of the B200 gridder (host side).
#pragma once

#include "curig_internal.h"
#include "kernels.cuh"

#include <cstdint>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

struct curig_opts;                 // include/curig.h

namespace curig {

struct Options {
    int precision = 0;        // 0: FP64 (the reference's only precision), 1: FP32
    int window = 0;           // 0: ES kernel, 1: learned window table (see set_window)
    int bin_xy = 0;           // bin edge in cells (0: chosen from the shared-memory budget)
    int sub = 0;              // visibilities per sub-problem (0: default)
    int smode = 0;            // FP32 tile accumulation: 0 automatic, 1 float atomics,
                              // 2 one-word int32 fixed point, 3 exact two-word int32 fixed point
                              // (FP64: 1 double atomics, else exact three-word int32)
    size_t smem_budget = 0;   // bytes of shared memory per CTA for tiles (0: default)
    cudaStream_t stream = nullptr;
    int w_term = 0;           // 0: improved w-stacking, 1: w ignored (2-D gridding, no n - 1, n = 1)
    int grid_x = 0, grid_y = 0;   // oversampled grid along the nxdirty / nydirty axes (0: sigma rule)
    int bin_z = 0;                // w-planes per tile slab (0: automatic)
    int slabs = 1;                // row slabs of the sort (one-shot copy / compute pipeline), 1..MAX_SLABS
    int sparse = 0;               // FP32 spreader: chunks below this skip the tile (0: automatic, < 0: never)
    int n3 = 0;                   // generic 3-D NUFFT: modes along the third axis (0: the gridder)
};

struct Plan {
    int type = 1;             // 1: ms2dirty (vis -> dirty), 2: dirty2ms (dirty -> vis)
    int nx = 0, ny = 0;
    double psx = 0, psy = 0, eps = 1e-6, sigma = 2.0;
    int sign = 1;
    Options opt;
    cudaStream_t st = nullptr;
    int device = 0, nsm = 148;

    // set by setpts (geometry stage, then binning stage)
    bool geom_ready = false;
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
    size_t smem = 0, smem_interp = 0;
    double wmin_eff = 0, wmax_eff = 0;
    std::vector<double> htab;   // window table [kw][TAB_DEG] for the thread-per-visibility kernels
    // row slabs: slab k holds rows [slab_row[k], slab_row[k+1]) and the
    // sub-problems [k ? slab_sub_end[k-1] : 0, slab_sub_end[k])
    int nslab = 1;
    std::vector<long long> slab_row;
    std::vector<int> slab_sub_end;

    // device buffers owned by the plan
    double *d_foc = nullptr, *d_quad = nullptr, *d_psi1 = nullptr, *d_psi2 = nullptr, *d_wcoef = nullptr;
    double *d_psi3 = nullptr;          // generic 3-D NUFFT: window transform on the third axis [nf3/2+1]
    int *d_bin_count = nullptr, *d_bin_start = nullptr, *d_nsub = nullptr, *d_sub_end = nullptr;
    unsigned *d_keys_in = nullptr;                      // sort key per visibility (input order)
    int *d_kcount = nullptr;                            // count / first position per key value; after the
                                                        // records (FP32 tiles): end of every key's run
    int *d_cbin = nullptr;                              // bin of every sub-problem
    int *d_bcur = nullptr, *d_tmp = nullptr;            // bin cursors; input index per position, bin order
    int *d_idx = nullptr;                               // input index per sorted position (bin order)
    int *d_err = nullptr;
    unsigned long long *d_keys = nullptr;
    int *d_scan = nullptr;                              // scan temporaries (total, block sums)
    void *d_rec = nullptr, *d_ph = nullptr, *d_cs = nullptr, *d_grid = nullptr;
    void *d_tgrid = nullptr;           // image columns of every plane, transposed: [nf3][ny][nf2]
    CUtensorMap tmap{};                // TMA descriptor of d_grid for the interpolator's tile boxes (FP32)

    // x transforms on grid rows, y transforms on rows of the column-transposed planes
    cufftHandle fft_hx = 0, fft_hx_rest = 0, fft_hy = 0, fft_hy_rest = 0;
    size_t fft_wx = 0, fft_wx_rest = 0, fft_wy = 0, fft_wy_rest = 0;      // work-area bytes
    int fft_bx = 0, fft_bx_rest = 0, fft_by = 0, fft_by_rest = 0;         // rows per call

    // cuFFT cache entries this plan holds a reference to (released with its points)
    std::vector<std::tuple<int, int, int, int, int, int, uintptr_t, std::thread::id>> fft_keys;

    // learned-window tables per width (coefficients [kw][deg+1]); empty -> ES only
    std::vector<Window> learned;
    std::string last_error;

    // optional per-stage CUDA events (enabled by set_timing), see STAGE_* below
    cudaEvent_t ev[16] = {};
    bool ev_recorded[16] = {};
};

// event slots: setpts 0..2, ms2dirty 3..8, dirty2ms 9..13
enum Stage : int {
    EV_SET_BEGIN = 0, EV_SET_WRANGE = 1, EV_SET_END = 2,
    EV_M2D_BEGIN = 3, EV_M2D_PREP = 4, EV_M2D_ZERO = 5, EV_M2D_SPREAD = 6, EV_M2D_FFT = 7, EV_M2D_END = 8,
    EV_D2M_BEGIN = 9, EV_D2M_CORRECT = 10, EV_D2M_FFT = 11, EV_D2M_INTERP = 12, EV_D2M_END = 13,
};
void set_timing(bool on);
// durations (ms) of the last setpts / executes: [0] setpts, [1] binning part of setpts,
// [2] vis prep, [3] grid zero, [4] spread, [5] FFT (m2d), [6] correct (m2d),
// [7] correct+zero (d2m), [8] FFT (d2m), [9] interp, [10] vis out; -1 when not recorded
int plan_timings(Plan *p, double *out, int n);
long long launch_count();
void count_launch(int n = 1);

int plan_create(int type, int nx, int ny, double psx, double psy, double eps, double sigma, int sign,
                const Options &opt, Plan **out);
int plan_setpts(Plan *p, long long nrow, int nchan, const double *du, const double *dv,
                const double *dw, int stride, const double *h_freq);
// plan_setpts in two stages: the geometry (w range, sizes, correction tables,
// grid buffers and FFT plans, on the plan's stream; synchronises once), then
// tiles, binning and records on stream st.  With st not the plan's stream, st
// must wait for the plan's stream first, and the plan's stream must wait for st
// before anything executes.
int plan_setpts_geometry(Plan *p, long long nrow, int nchan, const double *du, const double *dv,
                         const double *dw, int stride, const double *h_freq);
int plan_setpts_bin(Plan *p, cudaStream_t st);
// dirty2ms grid preparation (corrections, per-plane screens, transforms) on
// the plan's stream; needs only the geometry stage.  With image_ready, the
// stream waits for it after clearing the buffer rows the image does not fill.
int plan_d2m_prologue(Plan *p, const void *d_dirty, cudaEvent_t image_ready = nullptr);
int plan_execute(Plan *p, void *d_vis, const void *d_wgt, void *d_dirty, int type = 0);
// The same transform run slab by slab (the one-shot copy / compute pipeline).
// ms2dirty: before slab k the plan's stream waits for ready[k] (the upload of
// that slab's visibilities and weights), then gathers and spreads it; the grid
// transforms follow the last slab.  dirty2ms: the grid is prepared first (the
// image must be on the device), then slab k is interpolated after ready[k]
// (its weights) and done[k] is recorded (its rows of d_vis are final).  The
// events describe the caller's partition of the rows into nev slabs: it must
// equal the plan's (nev == nslab), or the plan has one slab and waits for /
// records all of them.  Either array may be null.  prologue_done: dirty2ms
// skips the grid preparation (already run by plan_d2m_prologue).
int plan_execute_slabs(Plan *p, int type, void *d_vis, const void *d_wgt, void *d_dirty,
                       const cudaEvent_t *ready, const cudaEvent_t *done, int nev, bool prologue_done = false);
constexpr int MAX_SLABS = 8;
// Tile spreaders: chunks with fewer visibilities spread straight to the grid
// (each cell of such a tile receives about one tap), one warp per visibility.
// Measured thresholds at 4096^2 (ms of the spreader): FP32 with 1.6e8
// visibilities 19.5 for 64-192, 20.7 for 384; FP64 (three-word tiles) with one
// channel (1e7 visibilities, the reference ABI's call) 21.7 with the tile only,
// 14.1 / 14.1 / 15.8 / 20.5 for 32 / 64 / 128 / 256, with 16 channels 69.1 tile
// only, 65.7 / 65.2 / 65.9 / 69.7.
constexpr int DEFAULT_SPARSE_N = 128;
constexpr int DEFAULT_SPARSE_N64 = 64;
// first row of slab k of nslab over nrow rows (k = nslab gives nrow)
inline long long slab_first_row(long long nrow, int nslab, int k) {
    return ((long long)k * nrow + nslab - 1) / nslab;
}
int plan_destroy(Plan *p);
void plan_release_points(Plan *p);

// launchers (kernels.cu)
void launch_wrange(const double *w, int stride, long long nrow, unsigned long long *keys, int *err,
                   cudaStream_t st);
// binning: a counting sort over (bin, residue) keys (kernels.cu)
void launch_bin_count(const DevGeom &g, const double *u, const double *v, const double *w, const double *foc,
                      unsigned *keys, int *count, int *err, cudaStream_t st);
void launch_bin_scatter(long long M, const unsigned *keys, int cbits, int *bcur, int *tmp, cudaStream_t st);
void launch_chunk_bins(long long nb, const int *sub_end, int *cbin, cudaStream_t st);
void launch_bins_from_keys(const int *kstart, const int *total, long long nb, int cbits, int sub, int *bin_start,
                           int *bin_count, int *nsub, int *bcur, cudaStream_t st);
// Prefix sum of n int32 values (exclusive or inclusive); tmp holds
// scan_temp_ints(n) ints, tmp[0] receives the total.
long long scan_temp_ints(long long n);
void scan_ints(const int *in, int *out, long long n, bool inclusive, int *tmp, cudaStream_t st);
size_t tile_smem_bytes(const TileGeom &tg, int esize, int kw, int wdeg);
template <typename T>
void launch_records(const DevGeom &g, const double *u, const double *v, const double *w, const double *foc,
                    const int *tmp, long long M, int *kcur, void *rec, void *ph, int *idx, cudaStream_t st);
// cs[i] = vis[j] wgt[j] e^{i o_c w} for sorted positions i in [i0, i0 + n), j = idx[i]
// (the input indices of the positions [i0, i0 + n) are [i0, i0 + n) too); with
// weights and a scratch vw of every visibility, vis * wgt is formed in input
// order first and the gather reads one array.
// vis[j] *= wgt[j] for j in [i0, i0 + n) (nothing without weights): the weights
// of dirty2ms, applied after the interpolator's unweighted scatter.
template <typename T>
void launch_vis_scale(long long i0, long long n, void *vis, const void *wgt, cudaStream_t st);
template <typename T>
void launch_vis_prep(long long i0, long long n, const int *idx, const void *ph, const void *vis, const void *wgt,
                     void *vw, void *cs, cudaStream_t st);
template <typename T>
void launch_vis_out(long long M, const int *idx, const void *ph, const void *os, const void *wgt, void *vis,
                    cudaStream_t st);
// Tile kernels.  launch_spread spreads cs (vis * wgt * phase in bin order,
// written by k_vis_prep); launch_interp interpolates and scatters
// wgt * conj(phase) * value to io.vis — inside the tile kernel for widths up to
// 12 (the random writes overlap the shared-memory work), through os and
// k_vis_out for the generic wider kernel.
template <typename T>
int launch_spread(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                  const void *rec, void *cs, void *grid, const double *wc, const double *ht, VisIO io,
                  long long M, int nsm, cudaStream_t st);
template <typename T>
int launch_interp(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                  const void *rec, const void *grid, void *os, const double *wc, const double *ht, VisIO io,
                  long long M, const CUtensorMap *tmap, int *err, int nsm, cudaStream_t st);
template <typename T>
void launch_correct_m2d(const DevCorr &cc, const void *grid, void *dirty, cudaStream_t st);
template <typename T>
void launch_correct_d2m(const DevCorr &cc, const void *dirty, void *grid, cudaStream_t st);
// generic 3-D NUFFT: modes fk [nx][ny][n3] from / to the transformed planes
template <typename T>
void launch_correct3_m2d(const DevCorr &cc, const void *tgrid, void *fk, cudaStream_t st);
template <typename T>
void launch_correct3_d2m(const DevCorr &cc, const void *fk, void *tgrid, cudaStream_t st);
template <typename T>
void launch_cols_to_t(int ny, int nf1, int nf2, int nf3, const void *grid, void *t, cudaStream_t st);
template <typename T>
void launch_t_to_grid(int ny, int nf1, int nf2, int nf3, const void *t, void *grid, cudaStream_t st);
template <typename T>
void launch_zero_tpad(int nx, int ny, int nf2, int nf3, void *t, cudaStream_t st);
void launch_psi_grid(int n, int nq, const double *qx, const double *qg, double *out, cudaStream_t st);
void launch_nupts_uvw(long long m, const double *x, const double *y, const double *z, double s, double *uvw,
                      cudaStream_t st);

int plan_device_status(Plan *p);
// Bound on the polls of the interpolator's tile-load wait for plans whose
// points are set afterwards (polls <= 0: the default); noissue != 0 makes the
// tile loads not happen, for tests of the timeout path.
constexpr long long DEFAULT_TMA_POLLS = 1LL << 26;
void set_tile_wait(long long polls, int noissue);
// on = 0: ms2dirty gathers vis and wgt in one pass (no vis * wgt scratch), as
// when the scratch cannot be allocated; tests compare the two paths
void set_gather_scratch(int on);
// destroy the cached cuFFT handles no plan holds (returns how many); number cached
int fft_cache_trim();
int fft_cache_size();

// Generic NUFFT type 3 in one dimension (nufft3.cu): points x[m] with
// strengths c -> frequencies s[n]; the grid's series by the type-2 NUFFT.
struct Nufft3;
Nufft3 *nufft3_create(int iflag, double eps, double sigma, int precision, cudaStream_t st);
int nufft3_setpts(Nufft3 *p, long long m, const double *d_x, long long n, const double *d_s,
                  const ::curig_opts *opts);
int nufft3_execute(Nufft3 *p, const void *d_c, void *d_f);
void nufft3_info(const Nufft3 *p, int *nf, double *dinfo);
void nufft3_destroy(Nufft3 *p);

// global learned-window registry (set through the C ABI)
int registry_set_window(int kw, int degree, const double *coef, double eps_reached);
// smallest registered width whose reached error is <= eps (nullptr: none)
bool registry_pick_window(double eps, Window &out);   // narrowest window reaching eps
bool registry_get_window(int kw, Window &out);
void registry_clear();

}  // namespace curig
