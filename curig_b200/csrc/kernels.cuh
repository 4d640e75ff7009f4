// Device kernels of the gridder (declarations shared by kernels.cu and plan.cu).
#pragma once

#include "curig_internal.h"

#include <cuda.h>                   // CUtensorMap (TMA descriptor of the grid)

namespace curig {

template <typename T> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };

// Tabulated windows (piecewise polynomials, see WinTab): widths up to TAB_KW,
// TAB_DEG coefficients per tap (degree 11).
constexpr int TAB_KW = 12, TAB_DEG = 12;

// Everything a binning / spreading / interpolation launch needs, by value.
struct DevGeom {
    int nf1, nf2, nf3;
    int kw, hkw;                   // kernel width, floor(kw/2)
    int bx, by, bz, nbx, nby, nbz;
    double ibx, iby, ibz;          // 1 / bx, 1 / by, 1 / bz
    int tx, ty, tz, zpad;
    int sub;                       // visibilities per sub-problem
    int sparse_n;                  // FP32 spreader: chunks of fewer visibilities skip the tile
    int cbits;                     // bits of the in-tile start cell in the sort key (0: bin only)
    int smode;                     // tile accumulation: 0 two-word int32, 1 float atomics, 2 one-word int32
                                   // (FP64: 1 double atomics, else three-word int32)
    int tpitch;                    // tile row pitch of the thread-per-visibility kernels: tx + 1 rounded up
                                   // to even (the interpolator's rows start at an even x for TMA)
    int use_tma;                   // interpolator stages interior tiles with one TMA box load
    long long tma_polls;           // polls of a tile load's barrier before the load counts as lost
    int tma_test_noissue;          // test only: arm the barrier but issue no load (the wait runs out)
    int no_w;                      // w ignored: one plane, no z taps (window factor 1)
    float wmax3;                   // bound on |kx ky kz| of the tabulated window
    float wenv[TAB_KW];            // bound on |k(d)| of tap d over all offsets (one-word box bound)
    float wzmax;                   // bound on |kz| (1 without w)
    long long nbins;               // bins of all row slabs: nslab * nbins_slab
    long long nbins_slab;          // bins of one row slab (nbx * nby * nbz)
    int nslab;                     // row slabs (sort key major part; 1 = none)
    int sub_lo, sub_hi;            // sub-problem window of one launch (sub_hi 0: all)
    const int *cbin;               // bin of every sub-problem (set by the binning)
    const int *ccls;               // FP32 tile kernels: per (bin, start-cell residue mod 16) key, the end
                                   // of its run in bin order (the class boundaries of every bin)
    int *dbg;                      // bounds-checked build: error flags raised by the index checks
    double beta, c;                // ES parameters
    int wkind, wdeg;               // window kind (0 ES, 1 polynomial), degree
    // visibility geometry
    long long nrow;
    int nchan;
    int uvw_stride;                // 3 for [nrow][3], 1 for separate arrays
    double psx, psy, i_center, gamma, o_center, sign;
};

// Quarter-pixel correction geometry (ms2dirty epilogue / dirty2ms prologue).
struct DevCorr {
    int nx, ny, nf1, nf2, nf3;
    int no_w;                      // n = 1, psi3 = 1, no w phase
    double psx, psy, o_center, i_center, gamma, h;
    int nquad;
    const double *qx;              // quadrature nodes (grid units)
    const double *qg;              // quadrature weights * window
    const double *psi1;            // [nf1/2+1]
    const double *psi2;            // [nf2/2+1]
    int n3;                        // generic 3-D NUFFT: modes along z (0: w-stacking or 2-D)
    const double *psi3;            // 3-D NUFFT: [nf3/2+1], like psi1 / psi2
    int *dbg;                      // bounds-checked build: error flags raised by the index checks
};

enum ErrFlag : int { EF_NONFINITE = 1, EF_RANGE = 2, EF_TIMEOUT = 4, EF_BOUNDS = 8 };

// Index checks of the bounds-checked build (compiled with -DCURIG_BOUNDS_CHECK,
// libcurafft_check.so): IN_BOUNDS(cond, flags) raises EF_BOUNDS in *flags and
// yields false when cond fails, so the guarded access is skipped; the regular
// build compiles it to true and never evaluates cond.  A debugging aid in
// place of compute-sanitizer, which is not available on every system.
#ifdef CURIG_BOUNDS_CHECK
__device__ __forceinline__ bool bounds_ok(bool ok, int *flags) {
    if (!ok && flags) atomicOr(flags, EF_BOUNDS);
    return ok;
}
#define IN_BOUNDS(cond, flags) bounds_ok((cond), (flags))
#else
#define IN_BOUNDS(cond, flags) true
#endif

// Piecewise-polynomial window passed by value (kernel-parameter space, so the
// Horner coefficients are uniform constant operands): c[d][i], interval d,
// highest power first.  Used by the thread-per-visibility kernels (kw <= 12).
template <typename T> struct WinTab {
    T c[TAB_KW][TAB_DEG];
};

// The caller's visibilities (input order [nrow][nchan]) and the plan's gather
// tables, for the tile kernels that read or write them directly.
struct VisIO {
    const int *idx;        // sorted position -> input index
    const void *ph;        // e^{i o_c w} per sorted position (complex T)
    const void *wgt;       // weights in input order (T), may be null
    void *vis;             // visibilities in input order (complex T)
};

}  // namespace curig
