// CUDA kernels of the B200 gridder (sm_100a).
//
// Replaces, on the ms2dirty / dirty2ms path of the reference:
//   get_effective_coordinate + rescaling + pre_stage_1/2 + transpose
//       (precomp.cu:48-79, utils.cu:56-154, cuft.cu:19-92)  -> k_bin_keys + radix sort + k_records / k_vis_prep
//   conv_3d_nputsdriven (conv.cu:144-228)                  -> k_spread_t / k_spread (tile-binned)
//   interp_3d_nputsdriven (interp.cu:143-227)              -> k_interp_t / k_interp (tile-staged)
//   w_term_dft + deconv_2d + w_term_deconv + div_n_lm
//       (cuft.cu:520-572, deconv.cu:236-417, ra_exec.cu:22-52) -> k_correct_m2d (one pass)
//   div_n_lm + w_term_deconv + deconv_2d + w_term_idft
//       (ra_exec.cu:325-373, cuft.cu:575-612)              -> k_correct_d2m + k_zero_tpad
//   cura_cufft plane transforms (cuft.cu:127-143)            -> cuFFT rows + k_cols_to_t / k_t_to_grid
//   matrix_elementwise_multiply + shift_corr (utils.cu:156-192, ra_exec.cu:56-89) -> k_vis_out / k_interp_t
//   thrust min/max over w (utils.cu:42-53)                  -> k_wrange
#include "kernels.cuh"
#include "plan.h"

namespace curig {

template <typename T> using C = typename cplx_t<T>::type;
template <typename T> struct rec_t;
template <> struct rec_t<float> { using type = float4; };
template <> struct rec_t<double> { using type = double4; };
template <typename T> using R = typename rec_t<T>::type;

constexpr int NTHREADS = 256;
constexpr int NWARPS = NTHREADS / 32;
// k_spread_t: 16 warps per CTA, two CTAs per SM at the shared-memory budget of
// one fixed-point tile.  k_interp_t: 8 warps per CTA, two CTAs per SM.
constexpr int TTHREADS = 512;
constexpr int TWARPS = TTHREADS / 32;
// (384-thread FP32 interpolator CTAs measured slower: 18.4 against 17.8 ms)
template <typename T> constexpr int interp_threads() { return 256; }
constexpr int KSTR = 32;                 // per-axis stride of the per-warp kernel-value scratch
constexpr double TWO_PI = 2.0 * PI_D;

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ unsigned long long ordered_key(double x) {
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}

__device__ __forceinline__ int wrap3(int v, int n) {   // valid for -n <= v < 3n
    if (v < 0) v += n;
    if (v >= n) v -= n;
    if (v >= n) v -= n;
    return v;
}

__device__ __forceinline__ float pack_cell_f(int lx, int ly, int lz) {
    return __int_as_float(lx | (ly << 10) | (lz << 20));
}
__device__ __forceinline__ double pack_cell_d(int lx, int ly, int lz) {
    return __longlong_as_double((long long)(lx | (ly << 10) | (lz << 20)));
}
__device__ __forceinline__ int cell_bits(float w) { return __float_as_int(w); }
__device__ __forceinline__ int cell_bits(double w) { return (int)__double_as_longlong(w); }

// Grid coordinates of one visibility in the reference's operation order:
// u,v,w *= f/c (w also * sign), *= 2 pi; u *= pixsize_x, v *= pixsize_y;
// w' = (w - i_c)/gamma; g = (x/(2 pi) + 0.5) * nf with x <- v, y <- u, z <- w'.
__device__ __forceinline__ bool grid_coords(const DevGeom &g, double u, double v, double w, double foc, double &gx,
                                            double &gy, double &gz) {
    double us = ((u * foc) * TWO_PI) * g.psx;
    double vs = ((v * foc) * TWO_PI) * g.psy;
    double we = (w * (foc * g.sign)) * TWO_PI;
    double wp = (we - g.i_center) / g.gamma;
    gx = (vs * INV_2PI + 0.5) * g.nf1;
    gy = (us * INV_2PI + 0.5) * g.nf2;
    gz = (wp * INV_2PI + 0.5) * g.nf3;
    return isfinite(gx) && isfinite(gy) && isfinite(gz);
}

__device__ __forceinline__ bool vis_grid(const DevGeom &g, const double *__restrict__ uu,
                                         const double *__restrict__ vv, const double *__restrict__ ww,
                                         long long row, double foc, double &gx, double &gy,
                                         double &gz) {
    const long long o = row * g.uvw_stride;
    return grid_coords(g, uu[o], vv[o], ww[o], foc, gx, gy, gz);
}

__device__ __forceinline__ double w_eff(const DevGeom &g, const double *__restrict__ ww, long long row,
                                        double foc) {
    return (ww[row * g.uvw_stride] * (foc * g.sign)) * TWO_PI;
}
__device__ __forceinline__ double w_eff_v(const DevGeom &g, double w, double foc) {
    return (w * (foc * g.sign)) * TWO_PI;
}

// Periodic wrap into [0, nf), start cell ceil(g - kw/2), offset u = start-g+kw/2
// in [0,1), bin index and start relative to the bin's tile origin.  Points
// already inside [0, nf) (all of them unless |u| pixsize reaches 1/2) skip the
// wrap's division; the bin index is floor(gw / B) from a multiply by 1/B,
// corrected by exact integer comparisons.
__device__ __forceinline__ void axis_loc(double gc, int nf, int B, double invB, int nb, int hkw, int kw,
                                         int &bin, int &lstart, double &u) {
    double gw = gc;
    if (!(gc >= 0.0 && gc < (double)nf)) {
        gw = gc - (double)nf * floor(gc / (double)nf);
        if (gw >= (double)nf) gw -= (double)nf;
        if (gw < 0.0) gw = 0.0;
    }
    double sd = ceil(gw - 0.5 * kw);
    u = (sd - gw) + 0.5 * kw;
    if (u < 0.0) u = 0.0;
    if (u >= 1.0) u = 0.99999999999999989;
    bin = (int)(gw * invB);
    if ((double)(bin + 1) * B <= gw) ++bin;
    else if ((double)bin * B > gw) --bin;
    if (bin >= nb) bin = nb - 1;
    lstart = (int)sd - (bin * B - hkw);
}

struct VisLoc {
    long long bin;
    int lx, ly, lz;
    double ux, uy, uz;
};

__device__ __forceinline__ int locate(const DevGeom &g, double gx, double gy, double gz, VisLoc &L) {
    int bxi, byi, bzi;
    axis_loc(gx, g.nf1, g.bx, g.ibx, g.nbx, g.hkw, g.kw, bxi, L.lx, L.ux);
    axis_loc(gy, g.nf2, g.by, g.iby, g.nby, g.hkw, g.kw, byi, L.ly, L.uy);
    if (g.no_w) {                                  // one plane, no z taps
        L.lz = 0;
        L.uz = 0.0;
        bzi = 0;
    } else if (g.zpad) {
        axis_loc(gz, g.nf3, g.bz, g.ibz, g.nbz, g.hkw, g.kw, bzi, L.lz, L.uz);
    } else {
        double sd = ceil(gz - 0.5 * g.kw);
        double u = (sd - gz) + 0.5 * g.kw;
        if (u < 0.0) u = 0.0;
        if (u >= 1.0) u = 0.99999999999999989;
        L.uz = u;
        bzi = 0;
        L.lz = (int)sd;
        if (!(sd >= 0.0 && sd <= (double)(g.nf3 - g.kw))) return EF_RANGE;
    }
    if (L.lx < 0 || L.lx > g.tx - g.kw || L.ly < 0 || L.ly > g.ty - g.kw || L.lz < 0 ||
        (!g.no_w && L.lz > g.tz - g.kw))
        return EF_RANGE;
    L.bin = ((long long)bzi * g.nby + byi) * g.nbx + bxi;
    return 0;
}

// ------------------------------------------------------------------ w range
__global__ void k_wrange(const double *__restrict__ w, int stride, long long nrow,
                         unsigned long long *keys, int *err) {
    double lo = INFINITY, hi = -INFINITY;
    int bad = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nrow;
         i += (long long)gridDim.x * blockDim.x) {
        double x = w[i * stride];
        if (!isfinite(x)) bad = 1;
        else { lo = fmin(lo, x); hi = fmax(hi, x); }
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (lo <= hi) {
            atomicMin(&keys[0], ordered_key(lo));
            atomicMax(&keys[1], ordered_key(hi));
        }
        if (bad) atomicOr(err, EF_NONFINITE);
    }
}

// ------------------------------------------------------------------ binning (counting sort)
// Sort key of one visibility: bin id in the high bits, then the residue of its
// start cell's index in the tile (mod 16 for the FP32 tile kernels' class
// schedule, mod 32 for the FP64 and wide-window kernels: the shared-memory
// bank of its first tap).  With row slabs the bin id is slab * nbins_slab + bin (slab = row *
// nslab / nrow), so each slab's visibilities are contiguous in sorted order.
// BAD_KEY marks a visibility that could not be placed.
//
// The sort is a counting sort over the key values (at most 2^31 of them):
// k_bin_count counts every key, an exclusive scan turns the counts into each
// key's first sorted position, and k_bin_scatter claims positions with atomics
// and writes the input index there.  Sorted order is bin-major and, inside a
// bin, residue-major; the order of visibilities that share a key is whatever
// order their atomics ran in (nothing downstream depends on it beyond the last
// bits of FP32 sums, whose flush order is free anyway).  Every visibility
// takes its own atomic (merging the lanes of a warp with equal keys first,
// with __match_any_sync, measured 2 % slower over the three kernels).
constexpr unsigned BAD_KEY = 0xffffffffu;

__device__ __forceinline__ unsigned vis_key(const DevGeom &g, const double *__restrict__ uu,
                                            const double *__restrict__ vv, const double *__restrict__ ww,
                                            const double *__restrict__ foc, long long j, int &e) {
    const long long row = j / g.nchan;
    const int ch = (int)(j - row * g.nchan);
    double gx, gy, gz;
    VisLoc L;
    e = vis_grid(g, uu, vv, ww, row, foc[ch], gx, gy, gz) ? locate(g, gx, gy, gz, L) : EF_NONFINITE;
    if (e) return BAD_KEY;
    const unsigned cell = (unsigned)((L.lz * g.ty + L.ly) * g.tpitch + L.lx) & ((1u << g.cbits) - 1u);
    const long long slab = g.nslab > 1 ? row * g.nslab / g.nrow : 0;
    return ((unsigned)(slab * g.nbins_slab + L.bin) << g.cbits) | cell;
}

// keys[j] for every visibility (input order) and count[key] += 1.
__global__ void k_bin_count(DevGeom g, const double *__restrict__ uu, const double *__restrict__ vv,
                            const double *__restrict__ ww, const double *__restrict__ foc,
                            unsigned *__restrict__ keys, int *__restrict__ count, int *err) {
    const long long M = g.nrow * g.nchan;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int bad = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < M; j += stride) {
        int e;
        const unsigned key = vis_key(g, uu, vv, ww, foc, j, e);
        bad |= e;
        keys[j] = key;
        if (key != BAD_KEY && IN_BOUNDS((long long)key < (g.nbins << g.cbits), g.dbg)) atomicAdd(count + key, 1);
    }
    if (bad) atomicOr(err, bad);
}

// Coarse placement: tmp[position] = j with position = the first position of
// j's bin + a rank claimed on the bin's cursor (bcur starts at bin_start).
// With one cursor per bin (not per key) the partly written sectors of tmp stay
// in L2 while the pass runs; k_records then orders each bin by residue.
__global__ void k_bin_scatter(long long M, const unsigned *__restrict__ keys, int cbits, int *__restrict__ bcur,
                              int *__restrict__ tmp) {
    // two visibilities per thread and step: both cursor atomics in flight at once
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long j0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; j0 < M; j0 += 2 * stride) {
        const long long j1 = j0 + stride;
        const unsigned k0 = keys[j0], k1 = j1 < M ? keys[j1] : BAD_KEY;
        const int p0 = k0 != BAD_KEY ? atomicAdd(bcur + (k0 >> cbits), 1) : -1;
        const int p1 = k1 != BAD_KEY ? atomicAdd(bcur + (k1 >> cbits), 1) : -1;
        if (p0 >= 0) tmp[p0] = (int)j0;
        if (p1 >= 0) tmp[p1] = (int)j1;
    }
}

// Per bin, from the scanned key counts: first sorted position, count and the
// number of sub-problems (chunks of at most `sub` visibilities).
// Bin of every sub-problem: bin b owns sub-problems [sub_end[b] - nsub, sub_end[b])
// (sub_end = inclusive scan of the per-bin counts).
__global__ void k_chunk_bins(long long nb, const int *__restrict__ sub_end, int *__restrict__ cbin) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb; b += stride) {
        const int lo = b ? sub_end[b - 1] : 0, hi = sub_end[b];
        for (int s = lo; s < hi; ++s) cbin[s] = (int)b;
    }
}

// Chunks larger than CLS_SUB (the one-word FP32 tiles) also keep every start-
// cell residue class at <= CLS_SUB visibilities per chunk: a bin whose
// visibilities crowd into a few cells (one class) is cut as if the chunk size
// were CLS_SUB, so that its tile's box bound, and with it the rounding step of
// the one-word fixed point, stays that of a CLS_SUB chunk.
constexpr int CLS_SUB = 4096;

__global__ void k_bins_from_keys(const int *__restrict__ kstart, const int *__restrict__ total, long long nb,
                                 int cbits, int sub, int *__restrict__ bin_start, int *__restrict__ bin_count,
                                 int *__restrict__ nsub, int *__restrict__ bcur) {
    for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb;
         b += (long long)gridDim.x * blockDim.x) {
        const int s = kstart[b << cbits];
        const int e = b + 1 < nb ? kstart[(b + 1) << cbits] : *total;
        bin_start[b] = s;
        bcur[b] = s;
        bin_count[b] = e - s;
        int ns = (e - s + sub - 1) / sub;
        if (sub > CLS_SUB && cbits > 0) {
            const int nq = 1 << cbits;
            int big = 0;
            for (int q = 0; q < nq; ++q) {
                const int a = kstart[(b << cbits) + q], z = q + 1 < nq ? kstart[(b << cbits) + q + 1] : e;
                big = max(big, z - a);
            }
            ns = max(ns, (big + CLS_SUB - 1) / CLS_SUB);
        }
        nsub[b] = ns;
    }
}

// ------------------------------------------------------------------ scan
// Prefix sums of int32 arrays (n < 2^31 summing below 2^31): per-block sums,
// one block scanning the block sums, then each block's items scanned with its
// offset.  SCAN_T threads x SCAN_I consecutive items per block, staged in
// shared memory so that global loads and stores are coalesced.
constexpr int SCAN_T = 512, SCAN_I = 8, SCAN_B = SCAN_T * SCAN_I;

// Exclusive scan over the block (all SCAN_T threads call it, wsum has 32
// entries); tot = the block's total.
__device__ __forceinline__ int block_exclusive(int v, int *wsum, int &tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = lane < SCAN_T / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    const int r = (warp ? wsum[warp - 1] : 0) + x - v;
    tot = wsum[SCAN_T / 32 - 1];
    __syncthreads();                     // wsum may be reused by the caller
    return r;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_sums(const int *__restrict__ in, long long n, int *__restrict__ bsum) {
    const long long b0 = (long long)blockIdx.x * SCAN_B;
    int s = 0;
    for (int k = threadIdx.x; k < SCAN_B; k += SCAN_T)
        if (b0 + k < n) s += in[b0 + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ int ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < SCAN_T / 32; ++w) t += ws[w];
        bsum[blockIdx.x] = t;
    }
}

// One block: exclusive scan of the nblk block sums in place; *total = their sum.
__global__ void __launch_bounds__(SCAN_T) k_scan_top(int *__restrict__ bsum, long long nblk, int *__restrict__ total) {
    __shared__ int ws[32];
    int carry = 0;
    for (long long c0 = 0; c0 < nblk; c0 += SCAN_T) {
        const long long i = c0 + threadIdx.x;
        const int v = i < nblk ? bsum[i] : 0;
        int tot;
        const int ex = block_exclusive(v, ws, tot);
        if (i < nblk) bsum[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_apply(const int *__restrict__ in, long long n,
                                                       const int *__restrict__ boff, int *__restrict__ out,
                                                       int inclusive) {
    __shared__ int buf[SCAN_B + SCAN_B / 32];          // one pad word per 32: fewer bank conflicts
    __shared__ int ws[32];
    const long long b0 = (long long)blockIdx.x * SCAN_B;
    auto at = [](int k) { return k + (k >> 5); };
    for (int k = threadIdx.x; k < SCAN_B; k += SCAN_T) buf[at(k)] = b0 + k < n ? in[b0 + k] : 0;
    __syncthreads();
    int loc[SCAN_I], s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_I; ++i) {
        loc[i] = buf[at(threadIdx.x * SCAN_I + i)];
        s += loc[i];
    }
    int tot;
    int run = boff[blockIdx.x] + block_exclusive(s, ws, tot);
#pragma unroll
    for (int i = 0; i < SCAN_I; ++i) {
        const int v = loc[i];
        buf[at(threadIdx.x * SCAN_I + i)] = inclusive ? run + v : run;
        run += v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < SCAN_B; k += SCAN_T)
        if (b0 + k < n) out[b0 + k] = buf[at(k)];
}

// Records in sorted order: the visibilities of each bin (tmp, from
// k_bin_scatter) are placed at their final position inside the bin's
// segment, by residue: position = a rank claimed on the cursor of their key
// (kcur = the exclusive scan of the key counts).  Per position: fractional
// offsets + packed start cell, the w-shift phase e^{i o_c w} (cuft.cu:19-39,
// FP64) and the input index.
template <typename T>
__global__ void k_records(DevGeom g, const double *__restrict__ uu, const double *__restrict__ vv,
                          const double *__restrict__ ww, const double *__restrict__ foc,
                          const int *__restrict__ tmp, long long M, int *__restrict__ kcur, R<T> *__restrict__ rec,
                          C<T> *__restrict__ ph, int *__restrict__ idx) {
    // two positions per thread and step, their random coordinate reads issued
    // together (the pass is bound by their latency)
    constexpr int U = 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; i0 < M; i0 += U * stride) {
        int j[U];
        bool ok[U];
        double u[U], v[U], w[U], f[U];
        long long row[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const long long i = i0 + k * stride;
            ok[k] = i < M;
            j[k] = ok[k] ? tmp[i] : 0;
            ok[k] = ok[k] && IN_BOUNDS(j[k] >= 0 && j[k] < M, g.dbg);
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
            row[k] = j[k] / g.nchan;
            const int ch = (int)(j[k] - row[k] * g.nchan);
            const long long o = row[k] * g.uvw_stride;
            u[k] = ok[k] ? uu[o] : 0.0;
            v[k] = ok[k] ? vv[o] : 0.0;
            w[k] = ok[k] ? ww[o] : 0.0;
            f[k] = ok[k] ? foc[ch] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
            if (!ok[k]) continue;
            double gx, gy, gz;
            VisLoc L;
            grid_coords(g, u[k], v[k], w[k], f[k], gx, gy, gz);
            locate(g, gx, gy, gz, L);
            const unsigned cell = (unsigned)((L.lz * g.ty + L.ly) * g.tpitch + L.lx) & ((1u << g.cbits) - 1u);
            const long long slab = g.nslab > 1 ? row[k] * g.nslab / g.nrow : 0;
            const unsigned key = ((unsigned)(slab * g.nbins_slab + L.bin) << g.cbits) | cell;
            if (!IN_BOUNDS((long long)key < (g.nbins << g.cbits), g.dbg)) continue;
            const int p = atomicAdd(kcur + key, 1);
            if (!IN_BOUNDS(p >= 0 && p < M, g.dbg)) continue;
            R<T> r;
            r.x = (T)L.ux;
            r.y = (T)L.uy;
            r.z = (T)L.uz;
            if constexpr (sizeof(T) == 4) r.w = pack_cell_f(L.lx, L.ly, L.lz);
            else r.w = pack_cell_d(L.lx, L.ly, L.lz);
            rec[p] = r;
            double sn, cs;
            sincos(g.o_center * w_eff_v(g, w[k], f[k]), &sn, &cs);
            ph[p] = C<T>{(T)cs, (T)sn};
            idx[p] = j[k];
        }
    }
}

// vw = vis * wgt in input order (coalesced): the gather below then reads one
// random 8- or 16-byte element per visibility instead of two (vis and wgt
// live in different arrays, each random read costing a whole DRAM burst).
template <typename T>
__global__ void k_vis_weight(long long n, const C<T> *__restrict__ vis, const T *__restrict__ wgt,
                             C<T> *__restrict__ vw) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const C<T> v = vis[k];
        const T wt = wgt[k];
        vw[k] = C<T>{v.x * wt, v.y * wt};
    }
}

// vis *= wgt in input order (coalesced), after the interpolator's scatter has
// written vis[j] = value e^{-i o_c w}: the scatter then reads no weight at
// random.  (value e^{-i o_c w}) wgt is the product the scatter formed itself.
template <typename T>
__global__ void k_vis_scale(long long n, C<T> *__restrict__ vis, const T *__restrict__ wgt) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const C<T> v = vis[k];
        const T wt = wgt[k];
        vis[k] = C<T>{v.x * wt, v.y * wt};
    }
}

// c = vis * wgt * e^{i o_c w} gathered into bin order (ra_exec.cu:98-104).
template <typename T>
__global__ void k_vis_prep(long long M, const int *__restrict__ idx, const C<T> *__restrict__ ph,
                           const C<T> *__restrict__ vis, const T *__restrict__ wgt, C<T> *__restrict__ cs) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x) {
        int j = idx[i];
        C<T> v = vis[j], e = ph[i];
        T wt = wgt ? wgt[j] : (T)1;
        cs[i] = C<T>{(v.x * e.x - v.y * e.y) * wt, (v.x * e.y + v.y * e.x) * wt};
    }
}

// vis = interp * wgt * e^{-i o_c w} scattered back to input order
// (ra_exec.cu:56-89; the reference's weight "divide" invoker multiplies, utils.cu:189).
template <typename T>
__global__ void k_vis_out(long long M, const int *__restrict__ idx, const C<T> *__restrict__ ph,
                          const C<T> *__restrict__ os, const T *__restrict__ wgt, C<T> *__restrict__ vis) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x) {
        int j = idx[i];
        C<T> v = os[i], e = ph[i];
        T wt = wgt ? wgt[j] : (T)1;
        vis[j] = C<T>{(v.x * e.x + v.y * e.y) * wt, (v.y * e.x - v.x * e.y) * wt};
    }
}

// ------------------------------------------------------------------ window
template <typename T>
__device__ __forceinline__ T win_eval(const DevGeom &g, const T *__restrict__ coef, T u, int d) {
    if (g.wkind == 0) {
        T t = u + (T)d - (T)0.5 * (T)g.kw;
        T a = (T)1 - (T)g.c * t * t;
        if (!(a > (T)0)) return (T)0;
        // sqrt(a)-1 written as (a-1)/(sqrt(a)+1): no cancellation near t = 0
        T e = ((T)g.c * t * t) / (sqrt(a) + (T)1);
        return exp(-(T)g.beta * e);
    }
    const T *c = coef + d * (g.wdeg + 1);
    T s = (T)2 * u - (T)1;
    T v = c[0];
    for (int i = 1; i <= g.wdeg; ++i) v = fma(v, s, c[i]);
    return v;
}

template <typename T>
__device__ __forceinline__ void warp_kernel_values(const DevGeom &g, const T *coef, T *ks, T ux, T uy,
                                                   T uz, int kw, int lane) {
    for (int q = lane; q < 3 * kw; q += 32) {
        int ax = q >= 2 * kw ? 2 : (q >= kw ? 1 : 0);
        int d = q - ax * kw;
        T u = ax == 0 ? ux : (ax == 1 ? uy : uz);
        ks[ax * KSTR + d] = win_eval<T>(g, coef, u, d);
    }
}

__device__ __forceinline__ long long find_bin(const int *__restrict__ sub_end, long long nb, int s) {
    long long lo = 0, hi = nb - 1;      // first b with sub_end[b] > s
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (sub_end[mid] > s) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ void atomic_add_c(float2 *p, float2 v) { atomicAdd(p, v); }
// 16-byte vector reduction into global memory (address 16-byte aligned).
__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}
// 8-byte vector reduction into global memory (address 8-byte aligned).
__device__ __forceinline__ void red_add_v2(float *p, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b) : "memory");
}
__device__ __forceinline__ void atomic_add_c(double2 *p, double2 v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}

// ------------------------------------------------------------------ spreader
// One CTA per sub-problem (a bin and up to `sub` of its visibilities, persistent
// grid-stride over sub-problems); the bin's tile (bin + kw halo, all w-planes or
// a z-slab) is accumulated in shared memory with one warp per visibility (lanes
// over the kw^3 taps: no intra-warp address collisions) and flushed once with
// vector atomics.  KW > 0 fixes the width at compile time (0: runtime width).
template <typename T, int KW>
__global__ void __launch_bounds__(NTHREADS)
k_spread(DevGeom g, const int *__restrict__ bin_start, const int *__restrict__ bin_count,
         const int *__restrict__ sub_end, const R<T> *__restrict__ rec, const C<T> *__restrict__ cs,
         C<T> *__restrict__ grid, const double *__restrict__ wcoef) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int kw = KW > 0 ? KW : g.kw;
    const int ntile = g.tx * g.ty * g.tz;
    C<T> *tile = reinterpret_cast<C<T> *>(smem);
    T *ksall = reinterpret_cast<T *>(tile + ntile);
    T *coef = ksall + NWARPS * 3 * KSTR;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T *ks = ksall + warp * 3 * KSTR;
    if (g.wkind == 1)
        for (int i = threadIdx.x; i < kw * (g.wdeg + 1); i += NTHREADS) coef[i] = (T)wcoef[i];
    const int total = g.sub_hi ? g.sub_hi : sub_end[g.nbins - 1];   // sub-problem window [sub_lo, total)
    const int kk = kw * kw, k3 = kk * kw;
    const int txy = g.tx * g.ty;
    for (int s = g.sub_lo + blockIdx.x; s < total; s += gridDim.x) {
        long long b = g.cbin ? g.cbin[s] : find_bin(sub_end, g.nbins, s);
        int cnt = bin_count[b];
        int nsb = (cnt + g.sub - 1) / g.sub;
        int chunk = s - (sub_end[b] - nsb);
        int first = bin_start[b] + chunk * g.sub;
        int last = min(first + g.sub, bin_start[b] + cnt);
        for (int e = threadIdx.x; e < ntile; e += NTHREADS) tile[e] = C<T>{0, 0};
        __syncthreads();
        for (int i = first + warp; i < last; i += NWARPS) {
            R<T> r = rec[i];
            C<T> c = cs[i];
            warp_kernel_values<T>(g, coef, ks, r.x, r.y, r.z, kw, lane);
            __syncwarp();
            int cb = cell_bits(r.w);
            int base = ((cb >> 20) & 0xfff) * txy + ((cb >> 10) & 0x3ff) * g.tx + (cb & 0x3ff);
            for (int t = lane; t < k3; t += 32) {
                int dz = t / kk;
                int rm = t - dz * kk;
                int dy = rm / kw;
                int dx = rm - dy * kw;
                T wt = ks[dx] * ks[KSTR + dy] * ks[2 * KSTR + dz];
                C<T> *p = tile + base + dz * txy + dy * g.tx + dx;
                atomicAdd(&p->x, c.x * wt);
                atomicAdd(&p->y, c.y * wt);
            }
            __syncwarp();
        }
        __syncthreads();
        const long long bl = b % g.nbins_slab;
        long long bxi = bl % g.nbx, byi = (bl / g.nbx) % g.nby, bzi = bl / ((long long)g.nbx * g.nby);
        int ox = (int)bxi * g.bx - g.hkw, oy = (int)byi * g.by - g.hkw;
        int oz = g.zpad ? (int)bzi * g.bz - g.hkw : 0;
        for (int row = warp; row < g.ty * g.tz; row += NWARPS) {
            int y = row % g.ty, z = row / g.ty;
            int gy = wrap3(oy + y, g.nf2);
            int gz = g.zpad ? wrap3(oz + z, g.nf3) : z;
            C<T> *grow = grid + ((long long)gz * g.nf2 + gy) * g.nf1;
            const C<T> *trow = tile + row * g.tx;
            for (int x = lane; x < g.tx; x += 32) {
                C<T> v = trow[x];
                if (v.x != (T)0 || v.y != (T)0) atomic_add_c(grow + wrap3(ox + x, g.nf1), v);
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ interpolator
// One CTA per sub-problem: the bin's tile (with halo, wrapped) is staged in
// shared memory with coalesced row loads; one warp per visibility gathers the
// kw^3 taps and reduces with shuffles; results are written in bin order.
template <typename T, int KW>
__global__ void __launch_bounds__(NTHREADS)
k_interp(DevGeom g, const int *__restrict__ bin_start, const int *__restrict__ bin_count,
         const int *__restrict__ sub_end, const R<T> *__restrict__ rec, const C<T> *__restrict__ grid,
         C<T> *__restrict__ os, const double *__restrict__ wcoef) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int kw = KW > 0 ? KW : g.kw;
    const int ntile = g.tx * g.ty * g.tz;
    C<T> *tile = reinterpret_cast<C<T> *>(smem);
    T *ksall = reinterpret_cast<T *>(tile + ntile);
    T *coef = ksall + NWARPS * 3 * KSTR;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T *ks = ksall + warp * 3 * KSTR;
    if (g.wkind == 1)
        for (int i = threadIdx.x; i < kw * (g.wdeg + 1); i += NTHREADS) coef[i] = (T)wcoef[i];
    const int total = g.sub_hi ? g.sub_hi : sub_end[g.nbins - 1];   // sub-problem window [sub_lo, total)
    const int kk = kw * kw, k3 = kk * kw;
    const int txy = g.tx * g.ty;
    for (int s = g.sub_lo + blockIdx.x; s < total; s += gridDim.x) {
        long long b = g.cbin ? g.cbin[s] : find_bin(sub_end, g.nbins, s);
        int cnt = bin_count[b];
        int nsb = (cnt + g.sub - 1) / g.sub;
        int chunk = s - (sub_end[b] - nsb);
        int first = bin_start[b] + chunk * g.sub;
        int last = min(first + g.sub, bin_start[b] + cnt);
        const long long bl = b % g.nbins_slab;
        long long bxi = bl % g.nbx, byi = (bl / g.nbx) % g.nby, bzi = bl / ((long long)g.nbx * g.nby);
        int ox = (int)bxi * g.bx - g.hkw, oy = (int)byi * g.by - g.hkw;
        int oz = g.zpad ? (int)bzi * g.bz - g.hkw : 0;
        for (int row = warp; row < g.ty * g.tz; row += NWARPS) {
            int y = row % g.ty, z = row / g.ty;
            int gy = wrap3(oy + y, g.nf2);
            int gz = g.zpad ? wrap3(oz + z, g.nf3) : z;
            const C<T> *grow = grid + ((long long)gz * g.nf2 + gy) * g.nf1;
            C<T> *trow = tile + row * g.tx;
            for (int x = lane; x < g.tx; x += 32) trow[x] = grow[wrap3(ox + x, g.nf1)];
        }
        __syncthreads();
        for (int i = first + warp; i < last; i += NWARPS) {
            R<T> r = rec[i];
            warp_kernel_values<T>(g, coef, ks, r.x, r.y, r.z, kw, lane);
            __syncwarp();
            int cb = cell_bits(r.w);
            int base = ((cb >> 20) & 0xfff) * txy + ((cb >> 10) & 0x3ff) * g.tx + (cb & 0x3ff);
            T ar = 0, ai = 0;
            for (int t = lane; t < k3; t += 32) {
                int dz = t / kk;
                int rm = t - dz * kk;
                int dy = rm / kw;
                int dx = rm - dy * kw;
                T wt = ks[dx] * ks[KSTR + dy] * ks[2 * KSTR + dz];
                C<T> v = tile[base + dz * txy + dy * g.tx + dx];
                ar = fma(v.x, wt, ar);
                ai = fma(v.y, wt, ai);
            }
            for (int o = 16; o > 0; o >>= 1) {
                ar += __shfl_xor_sync(0xffffffffu, ar, o);
                ai += __shfl_xor_sync(0xffffffffu, ai, o);
            }
            if (lane == 0) os[i] = C<T>{ar, ai};
            __syncwarp();
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ thread-per-visibility
// Same sub-problem / tile structure, one thread per visibility: the kernel
// values along x and y live in registers (compile-time width), the taps are
// unrolled along x and y with immediate offsets and the w-axis value is
// evaluated per plane.  Visibilities are sorted by the bank residue of their
// start cell inside a bin, so the 32 lanes of a warp touch distinct banks.

// Window value for tap d: ES (direct) or the Horner table in parameter space.
template <typename T>
__device__ __forceinline__ T win_tap(const DevGeom &g, const WinTab<T> &tab, T u, int d) {
    if (g.wkind == 0) return win_eval<T>(g, nullptr, u, d);
    T s = (T)2 * u - (T)1;
    T v = tab.c[d][0];
#pragma unroll
    for (int i = 1; i < TAB_DEG; ++i) v = fma(v, s, tab.c[d][i]);
    return v;
}

// Sub-problem s is chunk j of the nsb chunks of bin b: the bin's sorted
// positions start + m * stride, m < n.  Chunks interleave, so each one samples
// every start-cell residue of the bin.
__device__ __forceinline__ void sub_range(const DevGeom &g, const int *bin_start, const int *bin_count,
                                          const int *sub_end, int s, long long &b, int &start, int &stride,
                                          int &n) {
    b = g.cbin ? g.cbin[s] : find_bin(sub_end, g.nbins, s);
    if (!IN_BOUNDS(b >= 0 && b < g.nbins, g.dbg)) {
        b = 0; start = 0; stride = 1; n = 0;
        return;
    }
    int cnt = bin_count[b];
    int nsb = sub_end[b] - (b ? sub_end[b - 1] : 0);   // the binning's chunk count (cnt / sub or more)
    int j = s - (sub_end[b] - nsb);
    if (!IN_BOUNDS(nsb >= 1 && j >= 0 && j < nsb, g.dbg)) {
        start = 0; stride = 1; n = 0;
        return;
    }
    start = bin_start[b] + j;
    stride = nsb;
    n = (cnt - j + nsb - 1) / nsb;
    if (!IN_BOUNDS(start >= 0 && n >= 0 && (n == 0 || start + (long long)(n - 1) * stride < g.nrow * g.nchan),
                   g.dbg))
        n = 0;
}

// Exact fixed-point accumulation of the FP32 spreader.  Shared-memory float
// atomics are a compare-and-swap loop on this part (about 9 updates / clock /
// SM without conflicts), native 32-bit integer atomics run at about 28.  Each
// term x (scaled by q = 2^(35 - e), 2^(e-1) <= max|c| < 2^e, so |x| < 2^35 for
// window products <= 2) is split exactly as h * 2^18 + l with |l| <= 2^17
// (rounding l to an integer: error <= 0.5 of 2^-35 max|c|), and h, l go to two
// int32 accumulators per component.  With at most 4096 terms per cell
// (sub <= 4096): |sum h| <= 2^12 * 2^18 = 2^30 and |sum l| <= 2^12 * 2^17 =
// 2^29, so nothing overflows; the sums are exact and order-independent.
constexpr int FIX_BITS = 35;   // the split point 2^18 is built into split_fix

__device__ __forceinline__ void split_fix(float x, int &h, int &l) {
    const float M = 12582912.0f;                       // 1.5 * 2^23: rounds to integers below 2^22
    float t = fmaf(x, 3.814697265625e-06f, M);         // x * 2^-18, rounded to an integer
    h = __float_as_int(t) - 0x4B400000;
    float hf = t - M;
    float lf = fmaf(hf, -262144.0f, x);                // x - h * 2^18, exact
    l = __float_as_int(lf + M) - 0x4B400000;
}

// One-word fixed point: each term x * q is rounded to an integer by one FMA
// against 1.5 * 2^23 (valid for |x q| <= 2^22) and added with one int32 atomic
// per component.  A cell (x, y, z) receives only from visibilities whose start
// column lies in the kw x kw box ending at (x, y), a visibility starting at
// (x - dx, y - dy) with a term of at most max(|re c|, |im c|) wenv[dx]
// wenv[dy] wzmax (wenv[d]: bound on tap d's window value over all offsets, a
// few percent of the peak at the edge taps); B = max over cells of the sum of
// max(|re c|, |im c|) wenv[dx] wenv[dy] over that box bounds every cell sum by
// B wzmax.  The chunk's scale q = 2^k takes the largest k with max|c| wmax3 q
// <= 2^22 and B wzmax q <= 2^30, so no cell sum (at most B wzmax q + n/2 <
// 2^31) overflows; a term's rounding error is at most 2^-23 of max|c| wmax3,
// unless the box bound binds (for the ES window of width 6, more than about
// 1000 visibilities of the largest magnitude in one box).
__device__ __forceinline__ int round_fix(float a, float k) {
    return __float_as_int(fmaf(a, k, 12582912.0f)) - 0x4B400000;
}

// FP64 tiles (shared-memory double atomics are compare-and-swap loops, and
// 64-bit integer atomics run at about a quarter of the 32-bit rate on this
// part): each scaled term x is split exactly as h * 2^36 + m * 2^18 + l with
// three int32 planes.  Adding 1.5 * 2^70 rounds x to a multiple of 2^18 whose
// quotient X = round(x / 2^18) is the bit-pattern difference (same binade for
// |x| <= 2^54); h = X >> 18 and m = X & (2^18 - 1) split it further (m >= 0),
// and the remainder x - X 2^18 (exact, |.| <= 2^17) is rounded to the integer
// l by adding 1.5 * 2^52.  Four FP64 additions per term.  The chunk scale
// q = 2^k takes the largest k with max|c| wmax3 q <= 2^54, so |h| <= 2^18,
// 0 <= m < 2^18, |l| <= 2^17 and, with at most 4096 terms per cell (sub <=
// 4096), no plane's sum leaves int32: cell sums are exact and order-
// independent, and a term's rounding is at most 2^-55 of max|c| wmax3, below
// the FP64 rounding of the product itself (2^-53 of the product).
constexpr int FIX64_BITS = 54;
__device__ __forceinline__ void split_fix3(double x, int &h, int &m, int &l) {
    const double M18 = 1770887431076116955136.0;          // 1.5 * 2^70: ulp 2^18
    const double M0 = 6755399441055744.0;                 // 1.5 * 2^52: ulp 1
    const double t1 = x + M18;                            // x rounded to a multiple of 2^18
    const double t2 = (x - (t1 - M18)) + M0;              // remainder (exact), rounded to an integer
    const long long X = __double_as_longlong(t1) - __double_as_longlong(M18);
    h = (int)(X >> 18);
    m = (int)(X & 0x3FFFF);
    l = (int)(__double_as_longlong(t2) - __double_as_longlong(M0));
}

template <typename T, int KW>
__global__ void __launch_bounds__(TTHREADS, sizeof(T) == 4 ? 2 : 1)
k_spread_t(DevGeom g, const int *__restrict__ bin_start, const int *__restrict__ bin_count,
           const int *__restrict__ sub_end, const R<T> *__restrict__ rec, const C<T> *__restrict__ cs,
           C<T> *__restrict__ grid, const WinTab<T> tab) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ T redbuf[TWARPS];
    const int ntile = g.tpitch * g.ty * g.tz;            // tile [tz][ty][tpitch], columns >= tx stay 0
    const bool fix = sizeof(T) == 4 && g.smode == 0;    // FP32: exact two-word int32 fixed point
    const bool fix1 = sizeof(T) == 4 && g.smode == 2;   // FP32: one-word int32 fixed point
    const bool fix64 = sizeof(T) == 8 && g.smode != 1;  // FP64: three-word int32 fixed point (exact)
    const int csz = fix ? 16 : fix64 ? 24 : (int)sizeof(C<T>);   // bytes per complex cell
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = g.sub_hi ? g.sub_hi : sub_end[g.nbins - 1];   // sub-problem window [sub_lo, total)
    const int tx = g.tpitch, txy = g.tpitch * g.ty;
    const int nvec = (ntile * csz) / 16;
    int *fhr = reinterpret_cast<int *>(smem);          // two-word planes: re-high, re-low, im-high, im-low
    int *flr = fhr + ntile, *fhi = flr + ntile, *fli = fhi + ntile;
    int *fre = fhr, *fim = flr;                        // one-word planes: re, im
    float *colsum = reinterpret_cast<float *>(fhr + 2 * ntile);   // one-word: per start column sum|c|
    // FP64 planes: re-high, im-high (int64, units of 2^18), re-low, im-low (int32)
    // FP64 planes: re high / mid / low, im high / mid / low (int32 each)
    int *hre = reinterpret_cast<int *>(smem), *mre = hre + ntile, *lre = mre + ntile;
    int *him = lre + ntile, *mim = him + ntile, *lim = mim + ntile;
    for (int s = g.sub_lo + blockIdx.x; s < total; s += gridDim.x) {
        long long b;
        int start, stride, n;
        sub_range(g, bin_start, bin_count, sub_end, s, b, start, stride, n);
        // tile origin; columns are stored from x_al = ox rounded down to even
        // (column lx + shift), the layout of the interpolator's tiles
        const long long bl = b % g.nbins_slab;     // bin within its row slab
        const long long bxi = bl % g.nbx, byi = (bl / g.nbx) % g.nby, bzi = bl / ((long long)g.nbx * g.nby);
        const int ox = (int)bxi * g.bx - g.hkw, oy = (int)byi * g.by - g.hkw;
        const int oz = g.zpad ? (int)bzi * g.bz - g.hkw : 0;
        const int shift = ox & 1, x_al = ox - shift;
        if (sizeof(T) == 8 && n < g.sparse_n) {
            // A sparse FP64 chunk: one warp per visibility adds its taps
            // straight to the grid with double atomics (the lanes hold the kx,
            // ky, kz tap values, a shuffle apart; item t of the kz x ky x kx
            // block is one cell, so a warp instruction covers whole rows).
            // Uniform across the CTA; no shared memory is touched.
            constexpr int NT = 3 * KW;
            const int KZ = g.no_w ? 1 : KW, items = KZ * KW * KW;
            for (int v = warp; v < n; v += TWARPS) {
                const int i = start + v * stride;
                const R<T> r = rec[i];
                const C<T> c = cs[i];
                auto tapval = [&](int t) {        // t < NT: axis t / KW, tap t % KW
                    const int ax = t / KW, d = t - ax * KW;
                    if (ax == 2 && g.no_w) return d == 0 ? (T)1 : (T)0;
                    return win_tap<T>(g, tab, ax == 0 ? r.x : ax == 1 ? r.y : r.z, d);
                };
                const T tv0 = lane < NT ? tapval(lane) : (T)0;
                T tv1 = 0;
                if constexpr (NT > 32) tv1 = lane + 32 < NT ? tapval(lane + 32) : (T)0;
                auto tap = [&](int t) {           // uniform call: every lane shuffles
                    const T a0 = __shfl_sync(0xffffffffu, tv0, t & 31);
                    if constexpr (NT > 32) {
                        const T a1 = __shfl_sync(0xffffffffu, tv1, t & 31);
                        return t < 32 ? a0 : a1;
                    }
                    return a0;
                };
                const int cb = cell_bits(r.w);
                const int gx0 = ox + (cb & 0x3ff), gy0 = oy + ((cb >> 10) & 0x3ff), gz0 = oz + ((cb >> 20) & 0xfff);
                for (int t0 = 0; t0 < items; t0 += 32) {
                    const int t = t0 + lane, tt = min(t, items - 1);
                    const int dz = tt / (KW * KW), rem = tt - dz * (KW * KW), dy = rem / KW, dx = rem - dy * KW;
                    const T kx = tap(dx), ky = tap(KW + dy), kz = tap(2 * KW + dz);
                    const int gz = g.zpad ? wrap3(gz0 + dz, g.nf3) : gz0 + dz;
                    const int gy = wrap3(gy0 + dy, g.nf2), gx = wrap3(gx0 + dx, g.nf1);
                    if (t < items && IN_BOUNDS(gx >= 0 && gx < g.nf1 && gy >= 0 && gy < g.nf2 && gz >= 0 &&
                                                   gz < g.nf3, g.dbg)) {
                        C<T> *cell = grid + ((long long)gz * g.nf2 + gy) * g.nf1 + gx;
                        const T ar = c.x * kz * ky, ai = c.y * kz * ky;
                        atomicAdd(&cell->x, ar * kx);
                        atomicAdd(&cell->y, ai * kx);
                    }
                }
            }
            continue;
        }
        float4 *tv = reinterpret_cast<float4 *>(smem);
        for (int e = threadIdx.x; e < nvec; e += TTHREADS) tv[e] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!fix && !fix64)                              // (ntile is even: 24-byte cells fill whole float4s)
            for (int e = nvec * 16 / csz + threadIdx.x; e < ntile; e += TTHREADS)
                reinterpret_cast<C<T> *>(smem)[e] = C<T>{0, 0};
        if (fix1)
            for (int e = threadIdx.x; e < txy; e += TTHREADS) colsum[e] = 0.f;
        __syncthreads();
        // Scale statistics of the chunk: largest component of c (gathered into
        // bin order by k_vis_prep); one word: start-column histogram of it.
        T m = 0;
        if (fix || fix1 || fix64)
            for (int k = threadIdx.x; k < n; k += TTHREADS) {
                const int i = start + k * stride;
                const C<T> c = cs[i];
                const T mc = fmax(fabs(c.x), fabs(c.y));
                m = fmax(m, mc);
                if (fix1) {
                    const int cb = cell_bits(rec[i].w);
                    atomicAdd(colsum + ((cb >> 10) & 0x3ff) * tx + (cb & 0x3ff), (float)mc);
                }
            }
        T q = 1;
        double qinv = 1;
        if (fix || fix1 || fix64) {
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) redbuf[warp] = m;
            __syncthreads();
            m = 0;
#pragma unroll
            for (int w = 0; w < TWARPS; ++w) m = fmax(m, redbuf[w]);
            int k;
            if (fix) {
                int e = m > (T)0 ? ilogb(m) + 1 : 0;       // 2^(e-1) <= m < 2^e
                k = FIX_BITS - e;
            } else if (fix64) {
                k = FIX64_BITS - (m > (T)0 ? ilogb(m * g.wmax3) + 1 : 0);
            } else {
                // largest kw x kw box sum of the start-column histogram
                float bmax = 0.f;
                for (int e = threadIdx.x; e < txy; e += TTHREADS) {
                    const int x = e % tx, y = e / tx;
                    float a = 0.f;
                    for (int yy = max(0, y - KW + 1); yy <= y; ++yy)
                        for (int xx = max(0, x - KW + 1); xx <= x; ++xx) a += colsum[yy * tx + xx];
                    bmax = fmaxf(bmax, a);
                }
                for (int o = 16; o > 0; o >>= 1) bmax = fmaxf(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
                __syncthreads();                                  // every thread has read redbuf
                if (lane == 0) redbuf[warp] = (T)bmax;
                __syncthreads();
                T bb = 0;
#pragma unroll
                for (int w = 0; w < TWARPS; ++w) bb = fmax(bb, redbuf[w]);
                // float sums of <= 4096 terms: relative error < 2^-12, inside the bound's factor-2 margin
                int em = m > (T)0 ? ilogb(m * g.wmax3) + 1 : 0;
                int es = bb > (T)0 ? ilogb(bb * g.wmax3) + 1 : 0;
                k = min(22 - em, 30 - es);
            }
            k = min(k, 120);                             // chunks of near-zero values
            q = (T)ldexp(1.0, k);
            qinv = ldexp(1.0, -k);
        }
        __syncthreads();
        // Lane l of a warp takes row l of the 32 x L matrix of the chunk's
        // positions (sorted by start-cell residue mod 32), warps walk its
        // columns: the lanes' cells are distinct mod 32 wherever the residues
        // are balanced, and every tap then hits 32 distinct banks.  A chunk of
        // fewer than TWARPS columns splits each visibility's w-planes into S
        // parts (one warp per column and part) so that all warps have work.
        const int L = (n + 31) >> 5;
        const int KZ = g.no_w ? 1 : KW;                   // z taps (2-D: one, weight 1)
        const int S = max(1, min(KZ, TWARPS / max(L, 1)));
        for (int u = warp; u < L * S; u += TWARPS) {
            const int k = u / S, part = u - k * S;
            const int m = lane * L + k;
            if (m >= n) continue;
            const int i = start + m * stride;
            const int dz0 = part * KZ / S, dz1 = (part + 1) * KZ / S;
            R<T> r = rec[i];
            C<T> c = cs[i];
            T kx[KW], ky[KW];
#pragma unroll
            for (int d = 0; d < KW; ++d) {
                kx[d] = win_tap<T>(g, tab, r.x, d);
                ky[d] = win_tap<T>(g, tab, r.y, d);
            }
            int cb = cell_bits(r.w);
            int cell = ((cb >> 20) & 0xfff) * txy + ((cb >> 10) & 0x3ff) * tx + (cb & 0x3ff) + shift;
            if (!IN_BOUNDS(cell >= 0 && cell + (KZ - 1) * txy + (KW - 1) * (tx + 1) < ntile, g.dbg)) continue;
            c.x *= q;
            c.y *= q;
#pragma unroll 1
            for (int dz = dz0; dz < dz1; ++dz) {
                T kz = g.no_w ? (T)1 : win_tap<T>(g, tab, r.z, dz);
                T cr = c.x * kz, ci = c.y * kz;
                int pz = cell + dz * txy;
#pragma unroll
                for (int dy = 0; dy < KW; ++dy) {
                    T ar = cr * ky[dy], ai = ci * ky[dy];
                    int prow = pz + dy * tx;
                    if constexpr (sizeof(T) == 4) {
                        if (fix1) {
#pragma unroll
                            for (int dx = 0; dx < KW; ++dx) {
                                atomicAdd(fre + prow + dx, round_fix(ar, kx[dx]));
                                atomicAdd(fim + prow + dx, round_fix(ai, kx[dx]));
                            }
                            continue;
                        }
                        if (fix) {
#pragma unroll
                            for (int dx = 0; dx < KW; ++dx) {
                                int h, l;
                                split_fix(ar * kx[dx], h, l);
                                atomicAdd(fhr + prow + dx, h);
                                atomicAdd(flr + prow + dx, l);
                                split_fix(ai * kx[dx], h, l);
                                atomicAdd(fhi + prow + dx, h);
                                atomicAdd(fli + prow + dx, l);
                            }
                            continue;
                        }
                    } else {
                        if (fix64) {
#pragma unroll
                            for (int dx = 0; dx < KW; ++dx) {
                                int h, mm, l;
                                split_fix3(ar * kx[dx], h, mm, l);
                                atomicAdd(hre + prow + dx, h);
                                atomicAdd(mre + prow + dx, mm);
                                atomicAdd(lre + prow + dx, l);
                                split_fix3(ai * kx[dx], h, mm, l);
                                atomicAdd(him + prow + dx, h);
                                atomicAdd(mim + prow + dx, mm);
                                atomicAdd(lim + prow + dx, l);
                            }
                            continue;
                        }
                    }
                    T *row = reinterpret_cast<T *>(smem) + 2 * prow;
#pragma unroll
                    for (int dx = 0; dx < KW; ++dx) {
                        atomicAdd(row + 2 * dx, ar * kx[dx]);
                        atomicAdd(row + 2 * dx + 1, ai * kx[dx]);
                    }
                }
            }
        }
        __syncthreads();
        // Flush: thread t walks the cell pairs (2p, 2p + 1) of the tile in memory
        // order ((x, y, z) of the pair advanced incrementally; the pitch is even,
        // so a pair never straddles rows); fixed-point cells convert in FP32 (one
        // rounding of each word, then one FMA).  Tiles that do not wrap the
        // periodic grid in x add a pair with one 16-byte vector reduction (the
        // pair's grid column x_al + 2k is even); the rest add cell by cell.
        {
            const float qf = (float)qinv, qf18 = (float)(qinv * 262144.0);
            const bool xin = x_al >= 0 && x_al + tx <= g.nf1;
            const int ty = g.ty, npair = ntile >> 1, hp = tx >> 1;      // pairs per row: hp
            const int q0 = TTHREADS / hp;
            const int sx = TTHREADS - q0 * hp, sy = q0 % ty, sz = q0 / ty;
            int xp = threadIdx.x % hp, yz = threadIdx.x / hp;
            int y = yz % ty, z = yz / ty;
            auto cellv = [&](int e) {
                C<T> v;
                if (fix) {
                    v.x = (T)fmaf(__int2float_rn(fhr[e]), qf18, __int2float_rn(flr[e]) * qf);
                    v.y = (T)fmaf(__int2float_rn(fhi[e]), qf18, __int2float_rn(fli[e]) * qf);
                } else if (fix1) {
                    v.x = (T)(__int2float_rn(fre[e]) * qf);
                    v.y = (T)(__int2float_rn(fim[e]) * qf);
                } else if (fix64) {
                    const double q36 = qinv * 0x1p36, q18 = qinv * 0x1p18;
                    v.x = (T)fma((double)hre[e], q36, fma((double)mre[e], q18, (double)lre[e] * qinv));
                    v.y = (T)fma((double)him[e], q36, fma((double)mim[e], q18, (double)lim[e] * qinv));
                } else {
                    v = reinterpret_cast<const C<T> *>(smem)[e];
                }
                return v;
            };
            for (int pr = threadIdx.x; pr < npair; pr += TTHREADS) {
                const C<T> v0 = cellv(2 * pr), v1 = cellv(2 * pr + 1);
                const bool nz0 = v0.x != (T)0 || v0.y != (T)0, nz1 = v1.x != (T)0 || v1.y != (T)0;
                if (nz0 || nz1) {
                    const int gy = wrap3(oy + y, g.nf2);
                    const int gz = g.zpad ? wrap3(oz + z, g.nf3) : z;
                    C<T> *grow = grid + ((long long)gz * g.nf2 + gy) * g.nf1;
                    const int c0 = 2 * xp;
                    bool vec = !IN_BOUNDS(gy >= 0 && gy < g.nf2 && gz >= 0 && gz < g.nf3 && z < g.tz, g.dbg);
                    if constexpr (sizeof(T) == 4) {
                        if (xin) {
                            red_add_v4(reinterpret_cast<float *>(grow + x_al + c0), v0.x, v0.y, v1.x, v1.y);
                            vec = true;
                        }
                    }
                    if (!vec) {
                        if (nz0) atomic_add_c(grow + wrap3(x_al + c0, g.nf1), v0);
                        if (nz1) atomic_add_c(grow + wrap3(x_al + c0 + 1, g.nf1), v1);
                    }
                }
                xp += sx;
                if (xp >= hp) { xp -= hp; ++y; }
                y += sy;
                z += sz;
                if (y >= ty) { y -= ty; ++z; }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ FP32 spreader
// The FP32 tile kernels order each bin by the residue mod 16 of its start
// cells (NCLS classes; the sort key's residue) and give every class two lanes
// of a warp, one in each half-warp: lane k + 16 f takes elements f, f + 2,
// f + 4, ... of class k (8-byte shared loads are served half a warp at a
// time, so the two lanes of a class must not share a half).  A
// tile cell's two words (re, im, or the high and low word of one component)
// are adjacent, so cell c covers banks 2c and 2c + 1 (mod 32): cells of
// different classes never share a bank, and the two lanes of one class write
// their cells' words in opposite order (lane f = 0: first word, then second;
// f = 1: second, then first), so they never meet in one instruction either.
// Every atomic instruction is one shared-memory wavefront; a warp step idles
// the lanes of classes that have run out (steps = the largest class / 2).
constexpr int NCLS = 16;

// Class boundaries of chunk j of bin b (positions first + j + k * nsb, k < n,
// first = the bin's first position): cls[q] = the first k of class q,
// cls[NCLS] = n.  The bin is in class order and g.ccls holds the end of every
// class run, so class q starts at position ccls[16 b + q - 1] (q > 0) and the
// chunk's elements before it number ceil((start_q - first - j) / nsb).
// Threads 0..NCLS write one entry each; the caller synchronises before reading.
__device__ __forceinline__ void chunk_classes(const DevGeom &g, long long b, int first, int j, int nsb, int n,
                                              int *cls) {
    const int q = threadIdx.x;
    if (q > NCLS) return;
    int v = n;
    if (q < NCLS) {
        const int s0 = q ? g.ccls[(b << 4) + q - 1] : first;
        const int d = s0 - first - j;
        v = d <= 0 ? 0 : min((d + nsb - 1) / nsb, n);
    }
    cls[q] = v;
}

// Warp steps of the class schedule: the largest class, halved (rounded up).
__device__ __forceinline__ int class_steps(const int *cls, int n) {
    int t = 0;
#pragma unroll
    for (int q = 0; q < NCLS; ++q) t = max(t, (min(max(cls[q + 1] - cls[q], 0), n) + 1) >> 1);
    return t;
}

// First position and size of class q, clamped to the chunk [0, n) (memory
// safety only: the sort makes the boundaries monotonic).
__device__ __forceinline__ void class_range(const int *cls, int q, int n, int &c0, int &nk) {
    c0 = min(max(cls[q], 0), n);
    nk = min(max(cls[q + 1] - c0, 0), n - c0);
}

// One chunk's warp steps of the class schedule (see k_spread_f32), for one
// accumulation mode (MODE: 2 one-word int32, 0 two-word int32, 1 float).  A
// lane's two words of a cell are its first word (word f) and second word
// (word 1 - f); the amplitude components are ordered to match once per
// visibility.  The next step's record and amplitude are loaded before this
// step's taps, so their latency overlaps the shared-memory atomics.
struct TapRun {
    int start, stride, c0, nk, T, S, KZ, txy, tx, shift, warp, f, ntile;
    float q;
};

template <int KW, int MODE>
__device__ __forceinline__ void spread_steps(const DevGeom &g, const WinTab<float> &tab,
                                             const float4 *__restrict__ rec, const float2 *__restrict__ cs, int *wA,
                                             int *wB, const TapRun &t) {
    const int steps = t.T * t.S;
    auto fetch = [&](int u, float4 &r, float2 &c, int &part) {
        if (u >= steps) return false;
        const int k = u / t.S;
        const int e = 2 * k + t.f;
        if (e >= t.nk) return false;
        part = u - k * t.S;
        const int i = t.start + (t.c0 + e) * t.stride;
        r = rec[i];
        c = cs[i];
        return true;
    };
    float4 rn = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 cn = make_float2(0.f, 0.f);
    int pn = 0;
    bool hn = fetch(t.warp, rn, cn, pn);
    for (int u = t.warp; u < steps; u += TWARPS) {
        const float4 r = rn;
        const float2 c = cn;
        const int part = pn;
        const bool have = hn;
        hn = fetch(u + TWARPS, rn, cn, pn);
        if (!have) continue;
        const int dz0 = part * t.KZ / t.S, dz1 = (part + 1) * t.KZ / t.S;
        float kx[KW], ky[KW];
#pragma unroll
        for (int d = 0; d < KW; ++d) {
            kx[d] = win_tap<float>(g, tab, r.x, d);
            ky[d] = win_tap<float>(g, tab, r.y, d);
        }
        const int cb = cell_bits(r.w);
        const int cell = ((cb >> 20) & 0xfff) * t.txy + ((cb >> 10) & 0x3ff) * t.tx + (cb & 0x3ff) + t.shift;
        const int p0 = 2 * cell + t.f, d1 = 1 - 2 * t.f;     // first word; second word = first + d1
        // the visibility's cells: cell .. cell + (KZ - 1) txy + (KW - 1) (tx + 1)
        if (!IN_BOUNDS(cell >= 0 && cell + (t.KZ - 1) * t.txy + (KW - 1) * (t.tx + 1) < t.ntile, g.dbg)) continue;
        if constexpr (MODE == 0) {
            const float cr = c.x * t.q, ci = c.y * t.q;
#pragma unroll 1
            for (int dz = dz0; dz < dz1; ++dz) {
                const float kz = g.no_w ? 1.f : win_tap<float>(g, tab, r.z, dz);
                const float zr = cr * kz, zi = ci * kz;
#pragma unroll
                for (int dy = 0; dy < KW; ++dy) {
                    const float ar = zr * ky[dy], ai = zi * ky[dy];
                    const int o = p0 + 2 * (dz * t.txy + dy * t.tx);
                    int *a0 = wA + o, *a1 = a0 + d1, *b0 = wB + o, *b1 = b0 + d1;
#pragma unroll
                    for (int dx = 0; dx < KW; ++dx) {
                        int hr, lr, hi, li;
                        split_fix(ar * kx[dx], hr, lr);
                        split_fix(ai * kx[dx], hi, li);
                        atomicAdd(a0 + 2 * dx, t.f ? lr : hr);
                        atomicAdd(a1 + 2 * dx, t.f ? hr : lr);
                        atomicAdd(b0 + 2 * dx, t.f ? li : hi);
                        atomicAdd(b1 + 2 * dx, t.f ? hi : li);
                    }
                }
            }
        } else {
            // this lane's first word holds component f, its second word the other
            const float c1 = (t.f ? c.y : c.x) * t.q, c2 = (t.f ? c.x : c.y) * t.q;
#pragma unroll 1
            for (int dz = dz0; dz < dz1; ++dz) {
                const float kz = g.no_w ? 1.f : win_tap<float>(g, tab, r.z, dz);
                const float z1 = c1 * kz, z2 = c2 * kz;
#pragma unroll
                for (int dy = 0; dy < KW; ++dy) {
                    const float a1 = z1 * ky[dy], a2 = z2 * ky[dy];
                    int *w1 = wA + p0 + 2 * (dz * t.txy + dy * t.tx), *w2 = w1 + d1;
#pragma unroll
                    for (int dx = 0; dx < KW; ++dx) {
                        if constexpr (MODE == 2) {
                            atomicAdd(w1 + 2 * dx, round_fix(a1, kx[dx]));
                            atomicAdd(w2 + 2 * dx, round_fix(a2, kx[dx]));
                        } else {
                            atomicAdd(reinterpret_cast<float *>(w1) + 2 * dx, a1 * kx[dx]);
                            atomicAdd(reinterpret_cast<float *>(w2) + 2 * dx, a2 * kx[dx]);
                        }
                    }
                }
            }
        }
    }
}

// FP32 tile accumulation (g.smode): 2 one-word int32 fixed point [re, im] per
// cell; 0 exact two-word int32 fixed point, plane A [re high, re low] and plane
// B [im high, im low] per cell; 1 float atomics [re, im] per cell.  Scale,
// overflow bound and chunk statistics as in k_spread_t.
template <int KW>
__global__ void __launch_bounds__(TTHREADS, 2)
k_spread_f32(DevGeom g, const int *__restrict__ bin_start, const int *__restrict__ bin_count,
             const int *__restrict__ sub_end, const float4 *__restrict__ rec, const float2 *__restrict__ cs,
             float2 *__restrict__ grid, const WinTab<float> tab) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ float redbuf[TWARPS];
    __shared__ int cls[NCLS + 1];
    const int ntile = g.tpitch * g.ty * g.tz;           // cells; tile [tz][ty][tpitch], columns >= tx stay 0
    const int mode = g.smode;
    const bool two = mode == 0, one = mode == 2, fixed = mode != 1;
    int *wA = reinterpret_cast<int *>(smem);            // [ntile][2]
    int *wB = wA + 2 * ntile;                           // two-word: [ntile][2]
    const int nwords = (two ? 4 : 2) * ntile;
    float *colsum = reinterpret_cast<float *>(wA + nwords);   // one word: per start column sum|c|
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = g.sub_hi ? g.sub_hi : sub_end[g.nbins - 1];
    const int tx = g.tpitch, txy = g.tpitch * g.ty;
    const int klass = lane & 15, f = lane >> 4;
    for (int s = g.sub_lo + blockIdx.x; s < total; s += gridDim.x) {
        long long b;
        int start, stride, n;
        sub_range(g, bin_start, bin_count, sub_end, s, b, start, stride, n);
        const long long bl = b % g.nbins_slab;
        const long long bxi = bl % g.nbx, byi = (bl / g.nbx) % g.nby, bzi = bl / ((long long)g.nbx * g.nby);
        const int ox = (int)bxi * g.bx - g.hkw, oy = (int)byi * g.by - g.hkw;
        const int oz = g.zpad ? (int)bzi * g.bz - g.hkw : 0;
        const int shift = ox & 1, x_al = ox - shift;
        if (n < g.sparse_n) {
            // A sparse chunk: its cells receive about one tap each, so the
            // tile would only add its fixed cost (zeroing, statistics, flush).
            // One warp per visibility adds its taps straight to the grid:
            // the lanes hold the kx, ky, kz tap values (a shuffle apart), and
            // item t of a plane (row dy = t / P, cell pair p = t % P of the P
            // pairs from the even column at or below the first x) is one
            // 16-byte vector reduction (FP32 sums, as the flush's); the
            // periodic wrap keeps a pair whole (nf1 is even).
            // Uniform across the CTA; no shared memory is touched.
            constexpr int P = (KW + 2) / 2, NT = 3 * KW;
            const int KZ = g.no_w ? 1 : KW;
            for (int v = warp; v < n; v += TWARPS) {
                const int i = start + v * stride;
                const float4 r = rec[i];
                const float2 c = cs[i];
                auto tapval = [&](int t) {       // t < NT: axis t / KW, tap t % KW
                    const int ax = t / KW, d = t - ax * KW;
                    if (ax == 2 && g.no_w) return d == 0 ? 1.f : 0.f;
                    return win_tap<float>(g, tab, ax == 0 ? r.x : ax == 1 ? r.y : r.z, d);
                };
                const float tv0 = lane < NT ? tapval(lane) : 0.f;
                float tv1 = 0.f;
                if constexpr (NT > 32) tv1 = lane + 32 < NT ? tapval(lane + 32) : 0.f;
                auto tap = [&](int t) {          // uniform call: every lane shuffles
                    const float a0 = __shfl_sync(0xffffffffu, tv0, t & 31);
                    if constexpr (NT > 32) {
                        const float a1 = __shfl_sync(0xffffffffu, tv1, t & 31);
                        return t < 32 ? a0 : a1;
                    }
                    return a0;
                };
                const int cb = cell_bits(r.w);
                const int gx0 = ox + (cb & 0x3ff), gy0 = oy + ((cb >> 10) & 0x3ff), gz0 = oz + ((cb >> 20) & 0xfff);
                const int sh = gx0 & 1;
                for (int t0 = 0; t0 < KW * P; t0 += 32) {
                    const int t = t0 + lane;
                    const int dy = min(t / P, KW - 1), pp = t - (t / P) * P;
                    const int d0 = 2 * pp - sh, d1 = d0 + 1;
                    const float x0 = tap(d0 >= 0 && d0 < KW ? d0 : 0);
                    const float x1 = tap(d1 < KW ? d1 : 0);
                    const float ky = tap(KW + dy);
                    const float k0 = d0 >= 0 && d0 < KW ? x0 : 0.f, k1 = d1 < KW ? x1 : 0.f;
                    const bool act = t < KW * P && d0 < KW;
                    const int gx = wrap3(gx0 - sh + 2 * pp, g.nf1), gy = wrap3(gy0 + dy, g.nf2);
#pragma unroll 1
                    for (int dz = 0; dz < KZ; ++dz) {
                        const float kz = tap(2 * KW + dz);
                        if (!act) continue;
                        const int gz = g.zpad ? wrap3(gz0 + dz, g.nf3) : gz0 + dz;
                        const float cr = c.x * kz * ky, ci = c.y * kz * ky;
                        if (IN_BOUNDS(gx >= 0 && (gx & 1) == 0 && gx + 1 < g.nf1 && gy >= 0 && gy < g.nf2 &&
                                          gz >= 0 && gz < g.nf3, g.dbg))
                            red_add_v4(reinterpret_cast<float *>(grid + ((long long)gz * g.nf2 + gy) * g.nf1 + gx),
                                       cr * k0, ci * k0, cr * k1, ci * k1);
                    }
                }
            }
            continue;
        }
        float4 *tv = reinterpret_cast<float4 *>(smem);
        for (int e = threadIdx.x; e < nwords / 4; e += TTHREADS) tv[e] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (one)
            for (int e = threadIdx.x; e < txy; e += TTHREADS) colsum[e] = 0.f;
        __syncthreads();
        // chunk statistics: largest component of c, one word: start-column sums
        // (four elements per thread in flight: the loads are issued first)
        float m = 0.f;
        if (fixed)
            for (int k0 = threadIdx.x; k0 < n; k0 += 4 * TTHREADS) {
                float2 cc[4];
                int cb[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = k0 + u * TTHREADS;
                    cc[u] = make_float2(0.f, 0.f);
                    cb[u] = 0;
                    if (k < n) {
                        const int i = start + k * stride;
                        cc[u] = cs[i];
                        if (one) cb[u] = cell_bits(rec[i].w);
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float mc = fmaxf(fabsf(cc[u].x), fabsf(cc[u].y));
                    m = fmaxf(m, mc);
                    if (one && k0 + u * TTHREADS < n &&
                        IN_BOUNDS(((cb[u] >> 10) & 0x3ff) < g.ty && (cb[u] & 0x3ff) < tx, g.dbg))
                        atomicAdd(colsum + ((cb[u] >> 10) & 0x3ff) * tx + (cb[u] & 0x3ff), mc);
                }
            }
        chunk_classes(g, b, bin_start[b], start - bin_start[b], stride, n, cls);
        float q = 1.f;
        double qinv = 1.0;
        if (fixed) {
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) redbuf[warp] = m;
            __syncthreads();
            m = 0.f;
#pragma unroll
            for (int w = 0; w < TWARPS; ++w) m = fmaxf(m, redbuf[w]);
            int k;
            if (two) {
                int e = m > 0.f ? ilogb(m) + 1 : 0;       // 2^(e-1) <= m < 2^e
                k = FIX_BITS - e;
            } else {
                // largest kw x kw box sum of the start-column sums, each
                // start column weighted by the bound on the taps it gives the
                // cell (wenv[dy] wenv[dx]): weighted sums of kw rows of each
                // column into the first txy words of the zeroed tile, then of
                // kw of those along each row (every thread a few cells); the
                // borrowed words are zeroed again
                float *vs = reinterpret_cast<float *>(wA);
                for (int e = threadIdx.x; e < txy; e += TTHREADS) {
                    const int y = e / tx, x = e - y * tx;
                    float a = 0.f;
#pragma unroll
                    for (int d = 0; d < KW; ++d)
                        if (y - d >= 0) a = fmaf(g.wenv[d], colsum[(y - d) * tx + x], a);
                    vs[e] = a;
                }
                __syncthreads();
                float bmax = 0.f;
                for (int e = threadIdx.x; e < txy; e += TTHREADS) {
                    const int y = e / tx, x = e - y * tx;
                    float a = 0.f;
#pragma unroll
                    for (int d = 0; d < KW; ++d)
                        if (x - d >= 0) a = fmaf(g.wenv[d], vs[y * tx + x - d], a);
                    bmax = fmaxf(bmax, a);
                }
                __syncthreads();                          // every read of vs is done
                for (int e = threadIdx.x; e < txy; e += TTHREADS) vs[e] = 0.f;
                for (int o = 16; o > 0; o >>= 1) bmax = fmaxf(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
                __syncthreads();                          // every thread has read redbuf
                if (lane == 0) redbuf[warp] = bmax;
                __syncthreads();
                float bb = 0.f;
#pragma unroll
                for (int w = 0; w < TWARPS; ++w) bb = fmaxf(bb, redbuf[w]);
                const int em = m > 0.f ? ilogb(m * g.wmax3) + 1 : 0;
                const int es = bb > 0.f ? ilogb(bb * g.wzmax) + 1 : 0;
                k = min(22 - em, 30 - es);
            }
            k = min(k, 120);
            q = (float)ldexp(1.0, k);
            qinv = ldexp(1.0, -k);
        }
        __syncthreads();
        // class schedule: lane k + 16 f, element 2t + f of class k at step t;
        // chunks of few steps split each visibility's w-planes into S parts
        {
            const int T = class_steps(cls, n);
            int c0, nk;
            class_range(cls, klass, n, c0, nk);
            const int KZ = g.no_w ? 1 : KW;
            const int S = max(1, min(KZ, TWARPS / max(T, 1)));
            const TapRun run{start, stride, c0, nk, T, S, KZ, txy, tx, shift, warp, f, ntile, q};
            if (one) spread_steps<KW, 2>(g, tab, rec, cs, wA, wB, run);
            else if (two) spread_steps<KW, 0>(g, tab, rec, cs, wA, wB, run);
            else spread_steps<KW, 1>(g, tab, rec, cs, wA, wB, run);
        }
        __syncthreads();
        // Flush: cell pairs in memory order (one 16-byte shared load per pair
        // and plane); non-wrapping tiles add a pair with one 16-byte vector
        // reduction (grid column x_al + 2k is even), wrapping tiles cell by cell.
        {
            const float qf = (float)qinv, qf18 = (float)(qinv * 262144.0);
            const bool xin = x_al >= 0 && x_al + tx <= g.nf1;
            const int ty = g.ty, npair = ntile >> 1, hp = tx >> 1;
            const int q0 = TTHREADS / hp;
            const int sx = TTHREADS - q0 * hp, sy = q0 % ty, sz = q0 / ty;
            int xp = threadIdx.x % hp, yz = threadIdx.x / hp;
            int y = yz % ty, z = yz / ty;
            for (int pr = threadIdx.x; pr < npair; pr += TTHREADS) {
                float2 v0, v1;
                if (one) {
                    const int4 a = reinterpret_cast<const int4 *>(wA)[pr];
                    v0 = make_float2(__int2float_rn(a.x) * qf, __int2float_rn(a.y) * qf);
                    v1 = make_float2(__int2float_rn(a.z) * qf, __int2float_rn(a.w) * qf);
                } else if (two) {
                    const int4 a = reinterpret_cast<const int4 *>(wA)[pr], bq = reinterpret_cast<const int4 *>(wB)[pr];
                    v0 = make_float2(fmaf(__int2float_rn(a.x), qf18, __int2float_rn(a.y) * qf),
                                     fmaf(__int2float_rn(bq.x), qf18, __int2float_rn(bq.y) * qf));
                    v1 = make_float2(fmaf(__int2float_rn(a.z), qf18, __int2float_rn(a.w) * qf),
                                     fmaf(__int2float_rn(bq.z), qf18, __int2float_rn(bq.w) * qf));
                } else {
                    const float4 a = reinterpret_cast<const float4 *>(wA)[pr];
                    v0 = make_float2(a.x, a.y);
                    v1 = make_float2(a.z, a.w);
                }
                const bool nz0 = v0.x != 0.f || v0.y != 0.f, nz1 = v1.x != 0.f || v1.y != 0.f;
                if (nz0 || nz1) {
                    const int gy = wrap3(oy + y, g.nf2);
                    const int gz = g.zpad ? wrap3(oz + z, g.nf3) : z;
                    float2 *grow = grid + ((long long)gz * g.nf2 + gy) * g.nf1;
                    const int col = 2 * xp;
                    if (!IN_BOUNDS(gy >= 0 && gy < g.nf2 && gz >= 0 && gz < g.nf3 && z < g.tz &&
                                       (!xin || (x_al + col >= 0 && x_al + col + 1 < g.nf1)), g.dbg)) {
                    } else if (xin) {
                        red_add_v4(reinterpret_cast<float *>(grow + x_al + col), v0.x, v0.y, v1.x, v1.y);
                    } else {
                        if (nz0) atomic_add_c(grow + wrap3(x_al + col, g.nf1), v0);
                        if (nz1) atomic_add_c(grow + wrap3(x_al + col + 1, g.nf1), v1);
                    }
                }
                xp += sx;
                if (xp >= hp) { xp -= hp; ++y; }
                y += sy;
                z += sz;
                if (y >= ty) { y -= ty; ++z; }
            }
        }
        __syncthreads();
    }
}

// vis[idx[i]] = value * wgt * e^{-i o_c w} (ra_exec.cu:56-89; the weight
// multiplies, utils.cu:189): the scatter of dirty2ms back to input order.
template <typename T>
__device__ __forceinline__ void vis_store(const VisIO &io, int i, C<T> v, long long m, int *dbg) {
    const int j = io.idx[i];
    if (!IN_BOUNDS(j >= 0 && j < m, dbg)) return;
    const C<T> e = static_cast<const C<T> *>(io.ph)[i];
    const T wt = io.wgt ? static_cast<const T *>(io.wgt)[j] : (T)1;
    static_cast<C<T> *>(io.vis)[j] = C<T>{(v.x * e.x + v.y * e.y) * wt, (v.y * e.x - v.x * e.y) * wt};
}

// The same scatter in two halves: the loads (index, phase, weight) issued
// before the gather so that their latency overlaps the shared-memory work.
template <typename T> struct VisDst {
    int j;
    C<T> e;
    T wt;
};
template <typename T>
__device__ __forceinline__ VisDst<T> vis_dst(const VisIO &io, int i, long long m, int *dbg) {
    VisDst<T> d;
    d.j = io.idx[i];
    d.e = static_cast<const C<T> *>(io.ph)[i];
    if (!IN_BOUNDS(d.j >= 0 && d.j < m, dbg)) {
        d.j = -1;                                    // (bounds-checked build only) no scatter
        d.wt = (T)0;
        return d;
    }
    d.wt = io.wgt ? static_cast<const T *>(io.wgt)[d.j] : (T)1;
    return d;
}
template <typename T>
__device__ __forceinline__ void vis_put(const VisIO &io, const VisDst<T> &d, C<T> v) {
#ifdef CURIG_BOUNDS_CHECK
    if (d.j < 0) return;
#endif
    static_cast<C<T> *>(io.vis)[d.j] =
        C<T>{(v.x * d.e.x + v.y * d.e.y) * d.wt, (v.y * d.e.x - v.x * d.e.y) * d.wt};
}

// Interpolator tile layout: [tz][ty][tpitch], column c holding grid x =
// x_al + c with x_al = ox rounded down to even (so a TMA box may start there),
// i.e. tile cell lx of the bin at column lx + (ox & 1).
//
// Stage the tile (wrapped rows of all its planes) with plain loads: rows are
// walked without divisions and eight rows are in flight per warp before the
// shared stores.
template <typename T, int NW>
__device__ __forceinline__ void load_tile(const DevGeom &g, const C<T> *__restrict__ grid, C<T> *tile, int x_al,
                                          int oy, int oz, int warp, int lane) {
    const int nrows = g.ty * g.tz, W = g.tpitch;
    constexpr int RB = 8;
    for (int x0 = 0; x0 < W; x0 += 32) {
        const int x = x0 + lane;
        const bool xin = x < W;
        const int gx = wrap3(x_al + x, g.nf1);
        int row = warp, y = warp % g.ty, z = warp / g.ty;
        while (row < nrows) {
            C<T> v[RB];
            int rr[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                rr[k] = row;
                if (xin && row < nrows) {
                    int gy = wrap3(oy + y, g.nf2);
                    int gz = g.zpad ? wrap3(oz + z, g.nf3) : z;
                    v[k] = IN_BOUNDS(gx >= 0 && gx < g.nf1 && gy >= 0 && gy < g.nf2 && gz >= 0 && gz < g.nf3, g.dbg)
                               ? grid[((long long)gz * g.nf2 + gy) * g.nf1 + gx] : C<T>{0, 0};
                }
                row += NW;
                y += NW;
                while (y >= g.ty) { y -= g.ty; ++z; }
            }
#pragma unroll
            for (int k = 0; k < RB; ++k)
                if (xin && rr[k] < nrows) tile[rr[k] * W + x] = v[k];
        }
    }
}

// mbarrier / TMA helpers (PTX): one-shot barrier per tile, byte-count completion.
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// 3-D tiled box load (no multicast) of {x, y, z} (x in 8-byte elements, x * 8
// a multiple of 16) into dst.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, unsigned long long *bar, int x, int y,
                                            int z) {
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
                 ::"r"(smem_addr(dst)), "l"(map), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

template <typename T, int KW>
__global__ void __launch_bounds__(interp_threads<T>(), sizeof(T) == 4 ? 3 : 2)
k_interp_t(DevGeom g, const int *__restrict__ bin_start, const int *__restrict__ bin_count,
           const int *__restrict__ sub_end, const R<T> *__restrict__ rec, const C<T> *__restrict__ grid,
           const WinTab<T> tab, const VisIO io, const __grid_constant__ CUtensorMap tmap, int *err) {
    constexpr int IT = interp_threads<T>(), IW = IT / 32;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ C<T> partial[IT];      // per (column, part, lane) sums of split visibilities
    __shared__ unsigned long long bar;      // TMA completion barrier
    __shared__ int cls[NCLS + 1];           // FP32: class boundaries of the chunk
    C<T> *tile = reinterpret_cast<C<T> *>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = g.sub_hi ? g.sub_hi : sub_end[g.nbins - 1];   // sub-problem window [sub_lo, total)
    const int tx = g.tpitch, txy = g.tpitch * g.ty;
    const unsigned tile_bytes = (unsigned)(g.tpitch * g.ty * g.tz * sizeof(C<T>));
    unsigned parity = 0;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    for (int s = g.sub_lo + blockIdx.x; s < total; s += gridDim.x) {
        long long b;
        int start, stride, n;
        sub_range(g, bin_start, bin_count, sub_end, s, b, start, stride, n);
        const long long bl = b % g.nbins_slab;     // bin within its row slab
        const long long bxi = bl % g.nbx, byi = (bl / g.nbx) % g.nby, bzi = bl / ((long long)g.nbx * g.nby);
        const int ox = (int)bxi * g.bx - g.hkw, oy = (int)byi * g.by - g.hkw;
        const int oz = g.zpad ? (int)bzi * g.bz - g.hkw : 0;
        const int shift = ox & 1, x_al = ox - shift;
        // interior tiles (no periodic wrap) in one TMA box; the rest with plain loads
        const bool inner = g.use_tma && x_al >= 0 && x_al + g.tpitch <= g.nf1 && oy >= 0 &&
                           oy + g.ty <= g.nf2 && (!g.zpad || (oz >= 0 && oz + g.tz <= g.nf3));
        // FP32 class schedule (the classes are read while the tile loads)
        if constexpr (sizeof(T) == 4) chunk_classes(g, b, bin_start[b], start - bin_start[b], stride, n, cls);
        if (inner) {
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier reads of the tile
                mbar_expect_tx(&bar, tile_bytes);
                // x in 8-byte elements: the cell in FP32, its real part in FP64 (16-byte aligned)
                if (!g.tma_test_noissue) tma_load_3d(tile, &tmap, &bar, sizeof(T) == 4 ? x_al : 2 * x_al, oy, oz);
            }
            long long polls = 0;
            bool done = false;
            while (!(done = mbar_try_wait(&bar, parity)) && ++polls < g.tma_polls) {
            }
            parity ^= 1u;
            if (__syncthreads_or(!done)) {          // the load never completed: flag it and stop
                if (threadIdx.x == 0) atomicOr(err, EF_TIMEOUT);
                return;
            }
        } else {
            load_tile<T, IW>(g, grid, tile, x_al, oy, oz, warp, lane);
            __syncthreads();
        }
        // lane / position map and w-plane split of the spreader: FP32 the class
        // schedule (two lanes per class: a warp's 8-byte loads take the minimum
        // two wavefronts), FP64 the 32 x L matrix of residue-sorted positions
        const int KZ = g.no_w ? 1 : KW;
        int L, c0 = 0, nk = 0;
        if constexpr (sizeof(T) == 4) {
            L = class_steps(cls, n);
            class_range(cls, lane & 15, n, c0, nk);
        } else {
            L = (n + 31) >> 5;
        }
        const int S = max(1, min(KZ, IW / max(L, 1)));
        for (int u = warp; u < L * S; u += IW) {
            const int k = u / S, part = u - k * S;
            int m;
            if constexpr (sizeof(T) == 4) {
                const int e = 2 * k + (lane >> 4);
                if (e >= nk) continue;
                m = c0 + e;
            } else {
                m = lane * L + k;
                if (m >= n) continue;
            }
            const int i = start + m * stride;
            const int dz0 = part * KZ / S, dz1 = (part + 1) * KZ / S;
            R<T> r = rec[i];
            VisDst<T> dst;
            if (S == 1) dst = vis_dst<T>(io, i, g.nrow * g.nchan, g.dbg);
            T kx[KW], ky[KW];
#pragma unroll
            for (int d = 0; d < KW; ++d) {
                kx[d] = win_tap<T>(g, tab, r.x, d);
                ky[d] = win_tap<T>(g, tab, r.y, d);
            }
            int cb = cell_bits(r.w);
            const int c0i = ((cb >> 20) & 0xfff) * txy + ((cb >> 10) & 0x3ff) * tx + (cb & 0x3ff) + shift;
            if (!IN_BOUNDS(c0i >= 0 && c0i + (KZ - 1) * txy + (KW - 1) * (tx + 1) < txy * g.tz, g.dbg)) continue;
            const C<T> *base = tile + c0i;
            T ar = 0, ai = 0;
#pragma unroll 1
            for (int dz = dz0; dz < dz1; ++dz) {
                T kz = g.no_w ? (T)1 : win_tap<T>(g, tab, r.z, dz);
                const C<T> *pz = base + dz * txy;
                T sr = 0, si = 0;
#pragma unroll
                for (int dy = 0; dy < KW; ++dy) {
                    const C<T> *row = pz + dy * tx;
                    T rr = 0, ri = 0;
#pragma unroll
                    for (int dx = 0; dx < KW; ++dx) {
                        C<T> v = row[dx];
                        rr = fma(v.x, kx[dx], rr);
                        ri = fma(v.y, kx[dx], ri);
                    }
                    sr = fma(rr, ky[dy], sr);
                    si = fma(ri, ky[dy], si);
                }
                ar = fma(sr, kz, ar);
                ai = fma(si, kz, ai);
            }
            if (S == 1) vis_put<T>(io, dst, C<T>{ar, ai});
            else partial[u * 32 + lane] = C<T>{ar, ai};
        }
        if (S > 1) {                                   // L * S <= IW: one pass
            __syncthreads();
            for (int m = threadIdx.x; m < n; m += IT) {
                int ln, k;
                if constexpr (sizeof(T) == 4) {          // the lane and step that held position m
                    int q = 0;
                    while (q < NCLS - 1 && cls[q + 1] <= m) ++q;
                    const int e = m - cls[q];
                    if (e < 0 || (e >> 1) >= L) continue;   // (unreachable for sorted chunks)
                    ln = q + 16 * (e & 1);
                    k = e >> 1;
                } else {
                    ln = m / L;
                    k = m - ln * L;
                }
                C<T> v = partial[(k * S) * 32 + ln];
                for (int p = 1; p < S; ++p) {
                    C<T> w = partial[(k * S + p) * 32 + ln];
                    v.x += w.x;
                    v.y += w.y;
                }
                vis_store<T>(io, start + m * stride, v, g.nrow * g.nchan, g.dbg);
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ correction
// Shared per-quarter-pixel factors: n, k' and psi3 depend on |l|, |m| only.
struct QuarterPix {
    double n, kp, psi3, ph;
};

__device__ __forceinline__ QuarterPix quarter(const DevCorr &cc, int r, int s) {
    QuarterPix q;
    if (cc.no_w) {                                    // 2-D: no n, no w screen, no psi3
        q.n = 1.0;
        q.kp = 0.0;
        q.psi3 = 1.0;
        q.ph = 0.0;
        return q;
    }
    double a = (double)r * cc.psx, b = (double)s * cc.psy;
    q.n = sqrt(1.0 - a * a - b * b);                  // ra_exec.cu:31, precomp.cu:220
    double k = q.n - 1;
    q.kp = (k - cc.o_center) * cc.gamma * cc.h;       // cuft.cu:73
    double ps = 0.0;
    for (int i = 0; i < cc.nquad; ++i) ps += cc.qg[i] * cos(cc.qx[i] * q.kp);
    q.psi3 = 2.0 * ps;                                // deconv.cu:45-57
    q.ph = (k - cc.o_center) * cc.i_center;           // deconv.cu:390
    return q;
}

// The transformed planes are read and written in the column-transposed
// layout T[z][x'][y] (x' over the ny image columns in FFT order: grid column
// x' for x' < ny - ny/2, nf1 - ny + x' above; y over nf2, contiguous), so the
// y transforms are contiguous rows for cuFFT.  Thread index: r (the y side)
// fastest, so a warp's plane accesses are contiguous.

// ms2dirty epilogue: w-screen sum over planes + all corrections, one pass.
template <typename T>
__global__ void k_correct_m2d(DevCorr cc, const C<T> *__restrict__ grid, C<T> *__restrict__ dirty) {
    const int hx = cc.nx / 2, hy = cc.ny / 2;
    const long long nq = (long long)(hx + 1) * (hy + 1);
    const long long plane = (long long)cc.ny * cc.nf2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
         q += (long long)gridDim.x * blockDim.x) {
        int s = (int)(q / (hx + 1)), r = (int)(q - (long long)s * (hx + 1));
        QuarterPix Q = quarter(cc, r, s);
        double sc, cs;
        sincos(Q.ph, &sc, &cs);
        double den = cc.psi1[s] * cc.psi2[r] * Q.psi3 * Q.n;
        double fr = cs / den, fi = sc / den;
        // the four mirrored pixels (hx +- r, hy +- s), slot t = 2 sx + sy, in
        // fixed register slots with a validity flag
        bool val[4];
        long long off[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int sx = t >> 1, sy = t & 1;
            const int ix = sx ? hx - r : hx + r, iy = sy ? hy - s : hy + s;
            val[t] = ix >= 0 && ix < cc.nx && !(sx && r == 0) && iy >= 0 && iy < cc.ny && !(sy && s == 0);
            const int w2 = sx ? cc.nf2 - r : r;
            const int xp = sy ? cc.ny - s : s;               // image column of grid column nf1 - s / s
            if (val[t] && !IN_BOUNDS(w2 >= 0 && w2 < cc.nf2 && xp >= 0 && xp < cc.ny, cc.dbg)) val[t] = false;
            off[t] = val[t] ? (long long)xp * cc.nf2 + w2 : 0;
        }
        double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
        double es, ec, ss, scs;
        sincos(Q.kp, &ss, &scs);                                   // step e^{i k'}
        sincos(-Q.kp * (double)(cc.nf3 / 2), &es, &ec);            // e^{i k'(0 - nf3/2)}
        for (int p = 0; p < cc.nf3; ++p) {
            const C<T> *gp = grid + p * plane;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (val[t]) {
                    C<T> v = gp[off[t]];
                    ar[t] += (double)v.x * ec - (double)v.y * es;
                    ai[t] += (double)v.x * es + (double)v.y * ec;
                }
            }
            double nr = ec * scs - es * ss, ni = ec * ss + es * scs;
            ec = nr;
            es = ni;
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if (!val[t]) continue;
            const int ix = (t >> 1) ? hx - r : hx + r, iy = (t & 1) ? hy - s : hy + s;
            C<T> o;
            o.x = (T)(ar[t] * fr - ai[t] * fi);
            o.y = (T)(ar[t] * fi + ai[t] * fr);
            dirty[(long long)ix * cc.ny + iy] = o;
        }
    }
}

// dirty2ms prologue: corrections + per-plane screen, written at the image cells
// of every plane of T (its other rows are zeroed by k_zero_tpad).
template <typename T>
__global__ void k_correct_d2m(DevCorr cc, const C<T> *__restrict__ dirty, C<T> *__restrict__ grid) {
    const int hx = cc.nx / 2, hy = cc.ny / 2;
    const long long nq = (long long)(hx + 1) * (hy + 1);
    const long long plane = (long long)cc.ny * cc.nf2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
         q += (long long)gridDim.x * blockDim.x) {
        int s = (int)(q / (hx + 1)), r = (int)(q - (long long)s * (hx + 1));
        QuarterPix Q = quarter(cc, r, s);
        double sc, cs;
        sincos(-Q.ph, &sc, &cs);
        double den = cc.psi1[s] * cc.psi2[r] * Q.psi3 * Q.n;
        double fr = cs / den, fi = sc / den;
        // the four mirrored pixels in fixed register slots (t = 2 sx + sy)
        bool val[4];
        double vr[4], vi[4];
        long long off[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int sx = t >> 1, sy = t & 1;
            const int ix = sx ? hx - r : hx + r, iy = sy ? hy - s : hy + s;
            val[t] = ix >= 0 && ix < cc.nx && !(sx && r == 0) && iy >= 0 && iy < cc.ny && !(sy && s == 0);
            const int w2 = sx ? cc.nf2 - r : r;
            const int xp = sy ? cc.ny - s : s;
            if (val[t] && !IN_BOUNDS(w2 >= 0 && w2 < cc.nf2 && xp >= 0 && xp < cc.ny, cc.dbg)) val[t] = false;
            off[t] = val[t] ? (long long)xp * cc.nf2 + w2 : 0;
            vr[t] = vi[t] = 0;
            if (val[t]) {
                C<T> d = dirty[(long long)ix * cc.ny + iy];
                vr[t] = (double)d.x * fr - (double)d.y * fi;
                vi[t] = (double)d.x * fi + (double)d.y * fr;
            }
        }
        double es, ec, ss, scs;
        sincos(-Q.kp, &ss, &scs);                                  // step e^{-i k'}
        sincos(Q.kp * (double)(cc.nf3 / 2), &es, &ec);             // e^{-i k'(0 - nf3/2)}
        for (int p = 0; p < cc.nf3; ++p) {
            C<T> *gp = grid + p * plane;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (val[t]) {
                    C<T> o;
                    o.x = (T)(vr[t] * ec - vi[t] * es);
                    o.y = (T)(vr[t] * es + vi[t] * ec);
                    gp[off[t]] = o;
                }
            }
            double nr = ec * scs - es * ss, ni = ec * ss + es * scs;
            ec = nr;
            es = ni;
        }
    }
}

// Generic 3-D NUFFT (types 1 and 2): the third axis is a periodic grid of nf3
// planes like the first two, so after the planes' 2-D transforms (the image
// columns in T[z][x'][y]) the modes k3 = iz - n3/2 are the planes' series
// sum_p T[p] e^{+2 pi i k3 p / nf3}, divided by psi1 psi2 psi3 (the grid tables
// with the half-grid sign, as the first two axes).  Modes fk [nx][ny][n3],
// n3 fastest; pixel (ix, iy) maps to T's column as in k_correct_m2d.  The
// phase is advanced by one rotation per term and taken afresh every 64 terms.
__device__ __forceinline__ void col3(const DevCorr &cc, int ix, int iy, int &r, int &s, long long &off) {
    const int hx = cc.nx / 2, hy = cc.ny / 2;
    int w2, xp;
    if (ix >= hx) { r = ix - hx; w2 = r; } else { r = hx - ix; w2 = cc.nf2 - r; }
    if (iy >= hy) { s = iy - hy; xp = s; } else { s = hy - iy; xp = cc.ny - s; }
    off = (long long)xp * cc.nf2 + w2;
}

template <typename T>
__global__ void k_correct3_m2d(DevCorr cc, const C<T> *__restrict__ tg, C<T> *__restrict__ fk) {
    const long long total = (long long)cc.nx * cc.ny * cc.n3;
    const long long plane = (long long)cc.ny * cc.nf2;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(o % cc.n3);
        const long long pix = o / cc.n3;
        const int iy = (int)(pix % cc.ny), ix = (int)(pix / cc.ny);
        int r, s;
        long long off;
        col3(cc, ix, iy, r, s, off);
        const int k3 = iz - cc.n3 / 2;
        const double th = 2.0 * PI_D * (double)k3 / (double)cc.nf3;
        double sr, cr, er = 1.0, ei = 0.0, ar = 0.0, ai = 0.0;
        sincos(th, &sr, &cr);
        for (int p = 0; p < cc.nf3; ++p) {
            if ((p & 63) == 0) sincos(th * (double)p, &ei, &er);
            const C<T> v = tg[p * plane + off];
            ar += (double)v.x * er - (double)v.y * ei;
            ai += (double)v.x * ei + (double)v.y * er;
            const double nr = er * cr - ei * sr;
            ei = er * sr + ei * cr;
            er = nr;
        }
        const double den = cc.psi1[s] * cc.psi2[r] * cc.psi3[k3 < 0 ? -k3 : k3];
        fk[o] = C<T>{(T)(ar / den), (T)(ai / den)};
    }
}

// Type 2: plane p at pixel (ix, iy) = sum_k3 fk[ix][iy][k3] / (psi1 psi2 psi3)
// e^{-2 pi i k3 p / nf3}, written where k_correct_d2m writes (the other rows of
// T are zeroed by k_zero_tpad).  Thread per (plane, pixel), pixel x fastest.
template <typename T>
__global__ void k_correct3_d2m(DevCorr cc, const C<T> *__restrict__ fk, C<T> *__restrict__ tg) {
    const long long total = (long long)cc.nx * cc.ny * cc.nf3;
    const long long plane = (long long)cc.ny * cc.nf2;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(o % cc.nx);
        const long long t = o / cc.nx;
        const int iy = (int)(t % cc.ny), p = (int)(t / cc.ny);
        int r, s;
        long long off;
        col3(cc, ix, iy, r, s, off);
        const C<T> *f = fk + ((long long)ix * cc.ny + iy) * cc.n3;
        const double th = -2.0 * PI_D * (double)p / (double)cc.nf3;    // phase step per k3
        double sr, cr, er = 1.0, ei = 0.0, ar = 0.0, ai = 0.0;
        sincos(th, &sr, &cr);
        for (int iz = 0; iz < cc.n3; ++iz) {
            const int k3 = iz - cc.n3 / 2;
            if ((iz & 63) == 0) sincos(th * (double)k3, &ei, &er);
            const double w = 1.0 / cc.psi3[k3 < 0 ? -k3 : k3];
            const double vr = (double)f[iz].x * w, vi = (double)f[iz].y * w;
            ar += vr * er - vi * ei;
            ai += vr * ei + vi * er;
            const double nr = er * cr - ei * sr;
            ei = er * sr + ei * cr;
            er = nr;
        }
        const double den = cc.psi1[s] * cc.psi2[r];
        tg[p * plane + off] = C<T>{(T)(ar / den), (T)(ai / den)};
    }
}

// psi-hat of the window on the grid (deconv.cu:60-103): out[k] =
// 2 sum_i g_i cos((x_i - N + 1) / (N - 1) pi k), N = nf/2 + 1, the same
// arithmetic as the host psi_hat_grid.
__global__ void k_psi_grid(int n, int nq, const double *__restrict__ qx, const double *__restrict__ qg,
                           double *__restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < nq; ++i) s += qg[i] * cos((qx[i] - n + 1) / (double)(n - 1) * PI_D * k);
        out[k] = 2 * s;
    }
}

// Grid column of image column x' (FFT order: the two corners of the x axis).
__device__ __forceinline__ int grid_col(int xp, int ny, int nf1) { return xp < ny - ny / 2 ? xp : xp + nf1 - ny; }
// Image column of grid column x, or -1 outside the image's columns.
__device__ __forceinline__ int image_col(int x, int ny, int nf1) {
    return x < ny - ny / 2 ? x : (x >= nf1 - ny / 2 ? x - nf1 + ny : -1);
}

// Transposes between the grid and T through shared memory: tiles of 32
// columns x tt_y rows, 256 threads, each thread tt_y / 8 loads in flight before
// the tile's barrier; reads and writes along the contiguous axis (coalesced).
// 64 rows for 8-byte elements (17 KB tiles); 32 for 16-byte ones, whose 64-row
// tiles (34 KB) measured slower (fewer CTAs per SM).
template <typename T> constexpr int tt_y() { return sizeof(T) == 4 ? 64 : 32; }

// T[z][x'][y] = grid[z][y][grid_col(x')].  Grid: (ny/32, nf2/tt_y, nf3).
template <typename T>
__global__ void __launch_bounds__(256) k_cols_to_t(int ny, int nf1, int nf2, const C<T> *__restrict__ grid,
                                                   C<T> *__restrict__ t) {
    constexpr int TT_Y = tt_y<T>();
    __shared__ C<T> tile[TT_Y][33];
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TT_Y;
    const C<T> *gp = grid + (long long)blockIdx.z * nf1 * nf2;
    C<T> *tp = t + (long long)blockIdx.z * ny * nf2;
    const int xp = x0 + threadIdx.x;
    const int gx = xp < ny ? grid_col(xp, ny, nf1) : 0;
#pragma unroll
    for (int j = threadIdx.y; j < TT_Y; j += 8) {
        const int y = y0 + j;
        if (xp < ny && y < nf2) tile[j][threadIdx.x] = gp[(long long)y * nf1 + gx];
    }
    __syncthreads();
#pragma unroll
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int xq = x0 + j;
#pragma unroll
        for (int h = 0; h < TT_Y; h += 32) {
            const int y = y0 + h + threadIdx.x;
            if (xq < ny && y < nf2) tp[(long long)xq * nf2 + y] = tile[h + threadIdx.x][j];
        }
    }
}

// grid[z][y][x] = T[z][image_col(x)][y] for the image's columns, 0 elsewhere
// (tiles of columns outside the image are written as zeros directly).
// Grid: (nf1/32, nf2/tt_y, nf3).
template <typename T>
__global__ void __launch_bounds__(256) k_t_to_grid(int ny, int nf1, int nf2, const C<T> *__restrict__ t,
                                                   C<T> *__restrict__ grid) {
    constexpr int TT_Y = tt_y<T>();
    __shared__ C<T> tile[32][TT_Y + 1];
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TT_Y;
    C<T> *gp = grid + (long long)blockIdx.z * nf1 * nf2;
    const C<T> *tp = t + (long long)blockIdx.z * ny * nf2;
    const int x = x0 + threadIdx.x;
    // no image column in [x0, x0 + 32): image columns are x < ny - ny/2 and x >= nf1 - ny/2
    if (x0 >= ny - ny / 2 && x0 + 32 <= nf1 - ny / 2) {
#pragma unroll
        for (int j = threadIdx.y; j < TT_Y; j += 8) {
            const int yy = y0 + j;
            if (x < nf1 && yy < nf2) gp[(long long)yy * nf1 + x] = C<T>{0, 0};
        }
        return;
    }
#pragma unroll
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int xj = x0 + j;
        const int xp = xj < nf1 ? image_col(xj, ny, nf1) : -1;
#pragma unroll
        for (int h = 0; h < TT_Y; h += 32) {
            const int y = y0 + h + threadIdx.x;
            tile[j][h + threadIdx.x] = (xp >= 0 && y < nf2) ? tp[(long long)xp * nf2 + y] : C<T>{0, 0};
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = threadIdx.y; j < TT_Y; j += 8) {
        const int yy = y0 + j;
        if (x < nf1 && yy < nf2) gp[(long long)yy * nf1 + x] = tile[threadIdx.x][j];
    }
}

// Zero the rows of T that are not image rows (y in [nx - nx/2, nf2 - nx/2)),
// which k_correct_d2m does not write.
template <typename T>
__global__ void k_zero_tpad(int nx, int nf2, long long nrows, C<T> *__restrict__ t) {
    const int y0 = nx - nx / 2, y1 = nf2 - nx / 2;
    for (long long rr = blockIdx.x; rr < nrows; rr += gridDim.x) {
        C<T> *row = t + rr * nf2;
        for (int y = y0 + threadIdx.x; y < y1; y += blockDim.x) row[y] = C<T>{0, 0};
    }
}

// ------------------------------------------------------------------ launchers
static int grid_for(long long n, int per = NTHREADS) {
    long long b = (n + per - 1) / per;
    if (b > 148LL * 32) b = 148LL * 32;
    if (b < 1) b = 1;
    return (int)b;
}

void launch_wrange(const double *w, int stride, long long nrow, unsigned long long *keys, int *err,
                   cudaStream_t st) {
    count_launch();
    k_wrange<<<grid_for(nrow), NTHREADS, 0, st>>>(w, stride, nrow, keys, err);
}

void launch_bin_count(const DevGeom &g, const double *u, const double *v, const double *w, const double *foc,
                      unsigned *keys, int *count, int *err, cudaStream_t st) {
    count_launch();
    k_bin_count<<<grid_for(g.nrow * g.nchan), NTHREADS, 0, st>>>(g, u, v, w, foc, keys, count, err);
}

void launch_bin_scatter(long long M, const unsigned *keys, int cbits, int *bcur, int *tmp, cudaStream_t st) {
    count_launch();
    k_bin_scatter<<<grid_for(M), NTHREADS, 0, st>>>(M, keys, cbits, bcur, tmp);
}

void launch_bins_from_keys(const int *kstart, const int *total, long long nb, int cbits, int sub, int *bin_start,
                           int *bin_count, int *nsub, int *bcur, cudaStream_t st) {
    count_launch();
    k_bins_from_keys<<<grid_for(nb), NTHREADS, 0, st>>>(kstart, total, nb, cbits, sub, bin_start, bin_count, nsub,
                                                        bcur);
}

void launch_chunk_bins(long long nb, const int *sub_end, int *cbin, cudaStream_t st) {
    count_launch();
    k_chunk_bins<<<grid_for(nb), NTHREADS, 0, st>>>(nb, sub_end, cbin);
}

long long scan_temp_ints(long long n) { return (n + SCAN_B - 1) / SCAN_B + 1; }

void scan_ints(const int *in, int *out, long long n, bool inclusive, int *tmp, cudaStream_t st) {
    const long long nblk = (n + SCAN_B - 1) / SCAN_B;
    if (nblk == 0) {
        cudaMemsetAsync(tmp + 1, 0, sizeof(int), st);
        return;
    }
    count_launch(3);
    k_scan_sums<<<(unsigned)nblk, SCAN_T, 0, st>>>(in, n, tmp + 1);
    k_scan_top<<<1, SCAN_T, 0, st>>>(tmp + 1, nblk, tmp);
    k_scan_apply<<<(unsigned)nblk, SCAN_T, 0, st>>>(in, n, tmp + 1, out, inclusive ? 1 : 0);
}

template <typename T>
void launch_records(const DevGeom &g, const double *u, const double *v, const double *w, const double *foc,
                    const int *tmp, long long M, int *kcur, void *rec, void *ph, int *idx, cudaStream_t st) {
    count_launch();
    k_records<T><<<grid_for(M), NTHREADS, 0, st>>>(g, u, v, w, foc, tmp, M, kcur, reinterpret_cast<R<T> *>(rec),
                                                   reinterpret_cast<C<T> *>(ph), idx);
}

template <typename T>
void launch_vis_scale(long long i0, long long n, void *vis, const void *wgt, cudaStream_t st) {
    if (n <= 0 || !wgt) return;
    count_launch();
    k_vis_scale<T><<<grid_for(n), NTHREADS, 0, st>>>(n, reinterpret_cast<C<T> *>(vis) + i0,
                                                     reinterpret_cast<const T *>(wgt) + i0);
}

template <typename T>
void launch_vis_prep(long long i0, long long n, const int *idx, const void *ph, const void *vis, const void *wgt,
                     void *vw, void *cs, cudaStream_t st) {
    if (n <= 0) return;
    const C<T> *src = reinterpret_cast<const C<T> *>(vis);
    const T *w = reinterpret_cast<const T *>(wgt);
    if (w && vw) {                 // weights applied in input order first
        count_launch();
        k_vis_weight<T><<<grid_for(n), NTHREADS, 0, st>>>(n, src + i0, w + i0, reinterpret_cast<C<T> *>(vw) + i0);
        src = reinterpret_cast<const C<T> *>(vw);
        w = nullptr;
    }
    count_launch();
    k_vis_prep<T><<<grid_for(n), NTHREADS, 0, st>>>(n, idx + i0, reinterpret_cast<const C<T> *>(ph) + i0, src, w,
                                                    reinterpret_cast<C<T> *>(cs) + i0);
}

template <typename T>
void launch_vis_out(long long M, const int *idx, const void *ph, const void *os, const void *wgt, void *vis,
                    cudaStream_t st) {
    count_launch();
    k_vis_out<T><<<grid_for(M), NTHREADS, 0, st>>>(M, idx, reinterpret_cast<const C<T> *>(ph),
                                                   reinterpret_cast<const C<T> *>(os),
                                                   reinterpret_cast<const T *>(wgt), reinterpret_cast<C<T> *>(vis));
}

size_t tile_smem_bytes(const TileGeom &tg, int esize, int kw, int wdeg) {
    // rows padded to an even pitch (tx + 1 rounded up): the same cell index in
    // the spreader's and the interpolator's tiles (bank order of the sort key)
    const size_t pitch = (size_t)((tg.tx + 2) & ~1);
    // cell bytes: FP32 two-word 4 int32, FP64 2 int64 + 2 int32, else two words of esize
    size_t s = pitch * tg.ty * tg.tz * (tg.fix == 1 ? 16 : tg.fix == 3 ? 24 : 2 * esize);
    if (tg.fix == 2) s += pitch * tg.ty * 4;                           // one-word: column load histogram
    s += (size_t)NWARPS * 3 * KSTR * esize;
    s += (size_t)kw * (wdeg + 1) * esize;
    return (s + 15) & ~(size_t)15;
}

template <typename K>
static int launch_persistent(K kern, size_t smem, int nsm, int &blocks, int threads = NTHREADS) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return ERR_CUDA;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
    if (occ < 1) return ERR_UNSUPPORTED;
    blocks = nsm * occ;
    return OK;
}

template <typename T>
static WinTab<T> make_tab(const DevGeom &g, const double *ht) {
    WinTab<T> t{};
    if (g.wkind == 1 && ht)                         // host copy: [kw][TAB_DEG], highest power first
        for (int d = 0; d < g.kw && d < TAB_KW; ++d)
            for (int i = 0; i < TAB_DEG; ++i) t.c[d][i] = (T)ht[d * TAB_DEG + i];
    return t;
}

template <typename T, int KW>
static int launch_spread_kw(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                            const void *rec, void *cs, void *grid, const double *wc, const double *ht,
                            const VisIO &io, long long M, int nsm, cudaStream_t st) {
    int blocks = 0, s;
    if constexpr (KW > 0 && sizeof(T) == 4) {
        auto kern = k_spread_f32<KW>;
        if ((s = launch_persistent(kern, smem, nsm, blocks, TTHREADS))) return s;
        count_launch();
        kern<<<blocks, TTHREADS, smem, st>>>(g, bs, bc, se, reinterpret_cast<const float4 *>(rec),
                                             reinterpret_cast<const float2 *>(cs), reinterpret_cast<float2 *>(grid),
                                             make_tab<float>(g, ht));
    } else if constexpr (KW > 0) {
        auto kern = k_spread_t<T, KW>;
        if ((s = launch_persistent(kern, smem, nsm, blocks, TTHREADS))) return s;
        count_launch();
        kern<<<blocks, TTHREADS, smem, st>>>(g, bs, bc, se, reinterpret_cast<const R<T> *>(rec),
                                             reinterpret_cast<const C<T> *>(cs), reinterpret_cast<C<T> *>(grid),
                                             make_tab<T>(g, ht));
    } else {
        auto kern = k_spread<T, 0>;
        if ((s = launch_persistent(kern, smem, nsm, blocks))) return s;
        count_launch();
        kern<<<blocks, NTHREADS, smem, st>>>(g, bs, bc, se, reinterpret_cast<const R<T> *>(rec),
                                             reinterpret_cast<const C<T> *>(cs), reinterpret_cast<C<T> *>(grid), wc);
    }
    return OK;
}

template <typename T, int KW>
static int launch_interp_kw(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                            const void *rec, const void *grid, void *os, const double *wc, const double *ht,
                            const VisIO &io, long long M, const CUtensorMap *tmap, int *err, int nsm,
                            cudaStream_t st) {
    int blocks = 0, s;
    if constexpr (KW > 0) {
        auto kern = k_interp_t<T, KW>;
        if ((s = launch_persistent(kern, smem, nsm, blocks, interp_threads<T>()))) return s;
        count_launch();
        kern<<<blocks, interp_threads<T>(), smem, st>>>(g, bs, bc, se, reinterpret_cast<const R<T> *>(rec),
                                             reinterpret_cast<const C<T> *>(grid), make_tab<T>(g, ht), io,
                                             *tmap, err);
    } else {
        auto kern = k_interp<T, 0>;
        if ((s = launch_persistent(kern, smem, nsm, blocks))) return s;
        count_launch();
        kern<<<blocks, NTHREADS, smem, st>>>(g, bs, bc, se, reinterpret_cast<const R<T> *>(rec),
                                             reinterpret_cast<const C<T> *>(grid), reinterpret_cast<C<T> *>(os), wc);
        launch_vis_out<T>(M, io.idx, io.ph, os, io.wgt, io.vis, st);
    }
    return OK;
}

#define CURIG_KW_SWITCH(F, ...)                                  \
    switch (g.kw) {                                              \
    case 2: return F<T, 2>(__VA_ARGS__);                         \
    case 3: return F<T, 3>(__VA_ARGS__);                         \
    case 4: return F<T, 4>(__VA_ARGS__);                         \
    case 5: return F<T, 5>(__VA_ARGS__);                         \
    case 6: return F<T, 6>(__VA_ARGS__);                         \
    case 7: return F<T, 7>(__VA_ARGS__);                         \
    case 8: return F<T, 8>(__VA_ARGS__);                         \
    case 9: return F<T, 9>(__VA_ARGS__);                         \
    case 10: return F<T, 10>(__VA_ARGS__);                       \
    case 11: return F<T, 11>(__VA_ARGS__);                       \
    case 12: return F<T, 12>(__VA_ARGS__);                       \
    default: return F<T, 0>(__VA_ARGS__);                        \
    }

template <typename T>
int launch_spread(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                  const void *rec, void *cs, void *grid, const double *wc, const double *ht, VisIO io,
                  long long M, int nsm, cudaStream_t st) {
    CURIG_KW_SWITCH(launch_spread_kw, g, smem, bs, bc, se, rec, cs, grid, wc, ht, io, M, nsm, st)
}

template <typename T>
int launch_interp(const DevGeom &g, size_t smem, const int *bs, const int *bc, const int *se,
                  const void *rec, const void *grid, void *os, const double *wc, const double *ht, VisIO io,
                  long long M, const CUtensorMap *tmap, int *err, int nsm, cudaStream_t st) {
    CURIG_KW_SWITCH(launch_interp_kw, g, smem, bs, bc, se, rec, grid, os, wc, ht, io, M, tmap, err, nsm, st)
}

template <typename T>
void launch_correct_m2d(const DevCorr &cc, const void *grid, void *dirty, cudaStream_t st) {
    long long nq = (long long)(cc.nx / 2 + 1) * (cc.ny / 2 + 1);
    count_launch();
    k_correct_m2d<T><<<grid_for(nq, 128), 128, 0, st>>>(cc, reinterpret_cast<const C<T> *>(grid),
                                                        reinterpret_cast<C<T> *>(dirty));
}

template <typename T>
void launch_correct_d2m(const DevCorr &cc, const void *dirty, void *grid, cudaStream_t st) {
    long long nq = (long long)(cc.nx / 2 + 1) * (cc.ny / 2 + 1);
    count_launch();
    k_correct_d2m<T><<<grid_for(nq, 128), 128, 0, st>>>(cc, reinterpret_cast<const C<T> *>(dirty),
                                                        reinterpret_cast<C<T> *>(grid));
}

template <typename T>
void launch_correct3_m2d(const DevCorr &cc, const void *tgrid, void *fk, cudaStream_t st) {
    const long long total = (long long)cc.nx * cc.ny * cc.n3;
    count_launch();
    k_correct3_m2d<T><<<grid_for(total, 128), 128, 0, st>>>(cc, reinterpret_cast<const C<T> *>(tgrid),
                                                            reinterpret_cast<C<T> *>(fk));
}

template <typename T>
void launch_correct3_d2m(const DevCorr &cc, const void *fk, void *tgrid, cudaStream_t st) {
    const long long total = (long long)cc.nx * cc.ny * cc.nf3;
    count_launch();
    k_correct3_d2m<T><<<grid_for(total, 128), 128, 0, st>>>(cc, reinterpret_cast<const C<T> *>(fk),
                                                            reinterpret_cast<C<T> *>(tgrid));
}

template <typename T>
void launch_cols_to_t(int ny, int nf1, int nf2, int nf3, const void *grid, void *t, cudaStream_t st) {
    count_launch();
    dim3 g((ny + 31) / 32, (nf2 + tt_y<T>() - 1) / tt_y<T>(), nf3);
    k_cols_to_t<T><<<g, dim3(32, 8), 0, st>>>(ny, nf1, nf2, reinterpret_cast<const C<T> *>(grid),
                                              reinterpret_cast<C<T> *>(t));
}

template <typename T>
void launch_t_to_grid(int ny, int nf1, int nf2, int nf3, const void *t, void *grid, cudaStream_t st) {
    count_launch();
    dim3 g((nf1 + 31) / 32, (nf2 + tt_y<T>() - 1) / tt_y<T>(), nf3);
    k_t_to_grid<T><<<g, dim3(32, 8), 0, st>>>(ny, nf1, nf2, reinterpret_cast<const C<T> *>(t),
                                              reinterpret_cast<C<T> *>(grid));
}

// Nonuniform points of the generic NUFFT as gridder rows: (s x / 2pi, s y / 2pi, 0)
// (with unit pixels and frequency c the gridder's phase is then +-k.x).
__global__ void k_nupts_uvw(long long m, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, double s, double *__restrict__ uvw) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < m;
         j += (long long)gridDim.x * blockDim.x) {
        uvw[3 * j] = s * x[j] * INV_2PI;
        uvw[3 * j + 1] = y ? s * y[j] * INV_2PI : 0.0;
        uvw[3 * j + 2] = z ? s * z[j] * INV_2PI : 0.0;
    }
}

void launch_nupts_uvw(long long m, const double *x, const double *y, const double *z, double s, double *uvw,
                      cudaStream_t st) {
    count_launch();
    k_nupts_uvw<<<grid_for(m), NTHREADS, 0, st>>>(m, x, y, z, s, uvw);
}

void launch_psi_grid(int n, int nq, const double *qx, const double *qg, double *out, cudaStream_t st) {
    count_launch();
    k_psi_grid<<<grid_for(n, 128), 128, 0, st>>>(n, nq, qx, qg, out);
}

template <typename T>
void launch_zero_tpad(int nx, int ny, int nf2, int nf3, void *t, cudaStream_t st) {
    const long long rows = (long long)nf3 * ny;
    count_launch();
    k_zero_tpad<T><<<grid_for(rows, 1), 256, 0, st>>>(nx, nf2, rows, reinterpret_cast<C<T> *>(t));
}

#define CURIG_INSTANTIATE(T)                                                                          \
    template void launch_records<T>(const DevGeom &, const double *, const double *, const double *,  \
                                    const double *, const int *, long long, int *, void *, void *,    \
                                    int *, cudaStream_t);                                             \
    template void launch_vis_prep<T>(long long, long long, const int *, const void *, const void *,    \
                                     const void *, void *, void *, cudaStream_t);                     \
    template void launch_vis_scale<T>(long long, long long, void *, const void *, cudaStream_t);      \
    template void launch_vis_out<T>(long long, const int *, const void *, const void *, const void *, \
                                    void *, cudaStream_t);                                            \
    template int launch_spread<T>(const DevGeom &, size_t, const int *, const int *, const int *,     \
                                  const void *, void *, void *, const double *, const double *,       \
                                  VisIO, long long, int, cudaStream_t);                               \
    template int launch_interp<T>(const DevGeom &, size_t, const int *, const int *, const int *,     \
                                  const void *, const void *, void *, const double *, const double *, \
                                  VisIO, long long, const CUtensorMap *, int *, int, cudaStream_t);   \
    template void launch_correct_m2d<T>(const DevCorr &, const void *, void *, cudaStream_t);         \
    template void launch_correct_d2m<T>(const DevCorr &, const void *, void *, cudaStream_t);         \
    template void launch_correct3_m2d<T>(const DevCorr &, const void *, void *, cudaStream_t);        \
    template void launch_correct3_d2m<T>(const DevCorr &, const void *, void *, cudaStream_t);        \
    template void launch_cols_to_t<T>(int, int, int, int, const void *, void *, cudaStream_t);         \
    template void launch_t_to_grid<T>(int, int, int, int, const void *, void *, cudaStream_t);         \
    template void launch_zero_tpad<T>(int, int, int, int, void *, cudaStream_t);

CURIG_INSTANTIATE(float)
CURIG_INSTANTIATE(double)

}  // namespace curig
