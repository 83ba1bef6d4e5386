/*
 * gexs_tiles.cuh — the tile kernel of the cross-section path and its launch
 * templates.  One translation unit per profile class instantiates them
 * (gexs_tiles_voigt.cu, gexs_tiles_erf.cu, gexs_tiles_gh16.cu,
 * gexs_tiles_gh32.cu), so the variants compile in parallel.
 *
 * Work decomposition (replaces the reference's one-CTA-per-grid-point scan
 * over every line of a chunk, compute/CUDA/cross_kernal_v2.cu:403-457):
 *  - a work item is one tile of W = 32*B*WARPS consecutive bins of one job,
 *    or one slice of consecutive lines of a tile that holds more than the
 *    launch's lines_per_slice (SliceTables, gexs_internal.h);
 *  - a persistent grid pulls items from a global counter;
 *  - the CTA finds the lines whose window can reach its tile with two
 *    warp-cooperative binary searches over the nu-sorted line list;
 *  - line records stream global -> shared memory through cp.async,
 *    double-buffered, WARPS*32 lines per stage;
 *  - each thread derives one line per stage in FP64: S(T) (Boltzmann and
 *    stimulated-emission factors), the Doppler width, gammaL, and the exact
 *    integer bin limits of the line's window and of its Humlicek regions
 *    inside the tile, computed with the same FP64 predicates as the
 *    reference CPU path, so FP32 evaluation never changes a window or a
 *    region decision;
 *  - lane l of warp w owns bins wb + l + 32k (k < B) in registers and loops
 *    over the stage's lines: no atomic accumulation, every bin sums its
 *    lines in ascending line order, a split tile's slices are added in
 *    slice order (deterministic, independent of other jobs);
 *  - FP32 form: FP32 partial sums of up to 128 lines merged into a
 *    Kahan-compensated (sum, compensation) pair per bin in shared memory;
 *    FP64 form: plain FP64 sums in registers.
 */
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>
#include "gexs_device.cuh"
#include "gexs_internal.h"

namespace gexs {

/* profile classes of the kernel template */
enum { PK_VOIGT = 0, PK_ERF = 1, PK_GH16 = 2, PK_GH32 = 3 };

/* --------------------------------------------------------------- records
 * One derived record per (line, tile), written by the thread that derived
 * the line and read by every warp as 16-byte broadcast loads. */
struct __align__(16) RecF32 {   /* 48 bytes; Doppler/Gaussian and GH */
    float icf;             /* tile-relative centre bin floor(tc), exact      */
    float dx;              /* dnu * invw: x per bin                          */
    float mfcdx;           /* -(tc - floor(tc)) * dx                         */
    float a1;              /* GH: amp*y/pi                                   */
    float p;               /* GH: y^2                                        */
    float y;               /* GH: y ; Doppler: half bin in x units           */
    float amp;             /* GH: S*invw*out_scale ; Doppler: S*out_scale    */
    float fc;              /* tc - floor(tc) in [0, 1)                       */
    int   win;             /* a | b << 16 : bins [a, b) of the tile          */
    int   c1;              /* Doppler: bins whose xm <= the zero threshold   */
    int   mask;            /* per warp w: bit w touches, bit 8+w fast tier,
                              bit 16+w mid tier; bit 24: |x| may exceed 1e8
                              in this tile (overflow-free forms); bit 25 (GH):
                              y < 1/8, x as a float pair (gh_sum_f32_pair)   */
    int   pad;
};
/* GH records reuse two fields: y holds the low part of dx and amp the low
 * part of mfcdx (their high parts are dx and mfcdx), see make_rec */
constexpr int GH_PAIR_BIT = 1 << 25;

struct __align__(16) RecF64 {   /* 64 bytes */
    double nu;             /* centre after the nu==0 rule                   */
    double invw;
    double y;              /* Voigt/GH: y ; Doppler: unused                 */
    double amp;            /* Voigt/GH: S*invw ; Doppler: S                 */
    int    win, c1, c2, c3;
    int    mask, pad0, pad1, pad2;
};

/* FP32 Voigt record (64 bytes): the main-loop constants of a line in a
 * tile, each stored twice so that one 16-byte shared load fills two f32x2
 * register pairs; read by every warp as broadcast loads. */
struct __align__(16) RecV {
    int    win;            /* a | b << 16 : bins [a, b) of the tile          */
    int    c1;             /* bins not in Humlicek region I (the core)       */
    int    tiers;          /* 2 bits per warp: 0 skip, 1 full, 2 partial,
                              3 wide (|x| may exceed 1e8 in the tile)        */
    int    pad;
    float2 dx;             /* dnu * invw: x per bin                          */
    float2 mf;             /* -(tc - floor(tc)) * dx                         */
    float2 c;              /* y^2 - 1/2                                      */
    float2 y2;             /* 2 y^2                                          */
    float2 a;              /* amp * 0.5641896 * y                            */
    float2 nb;             /* {-floor(tc), 32 - floor(tc)}: bin offset of a
                              lane's bins k = 0, 1 after adding wb + lane    */
};


/* record type of a (profile class, precision) */
template <int PK, int PREC> struct RecOf;
template <int PK> struct RecOf<PK, GEXS_FP32> { typedef RecF32 T; };
template <int PK> struct RecOf<PK, GEXS_FP64> { typedef RecF64 T; };

__device__ __forceinline__ int pack2(int a, int b) { return a | (b << 16); }
__device__ __forceinline__ int lo16(int v) { return v & 0xffff; }
__device__ __forceinline__ int hi16(int v) { return (int)((unsigned)v >> 16); }


/* lines derived per thread between two CTA barriers */
constexpr int PH = 2;

/* ------------------------------------------------------- cp.async helpers */
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" :: "r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" :: "r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

/* ------------------------------------------------- warp binary searches */
/* first index in [0, n) with a[i] >= v (LE=false) or a[i] > v (LE=true) */
template <bool LE>
__device__ int64_t warp_bound(const double* __restrict__ a, int64_t n, double v, int lane)
{
    int64_t lo = 0, hi = n;
    while (hi - lo > 32) {
        int64_t step = (hi - lo) / 33;
        int64_t idx = lo + step * (lane + 1);
        double av = __ldg(a + idx);
        bool below = LE ? (av <= v) : (av < v);
        int c = __popc(__ballot_sync(0xffffffffu, below));
        int64_t nlo = (c == 0) ? lo : lo + step * c + 1;
        int64_t nhi = (c == 32) ? hi : lo + step * (c + 1);
        lo = nlo; hi = nhi;
    }
    int64_t idx = lo + lane;
    bool below = false;
    if (idx < hi) { double av = __ldg(a + idx); below = LE ? (av <= v) : (av < v); }
    return lo + __popc(__ballot_sync(0xffffffffu, below));
}

/* ---------------------------------------------------------- tile geometry */
struct Tile {
    const gexs_job* J;
    int64_t j0;          /* absolute first bin                       */
    int     jn;          /* bins in this tile                        */
    double  f0, fl;      /* frequencies of first / last bin          */
    double  inv_dnu;     /* 1 / dnu: tile-relative centres (search
                            guesses and FP32 offsets; every window and
                            region decision uses exact predicates)   */
};

/* window of a line inside the tile as [a, b) (tile-relative) */
__device__ __forceinline__ void tile_window(const Tile& T, double nu, double tc,
                                            int* pa, int* pb)
{
    const gexs_job& J = *T.J;
    if (J.window_rule == GEXS_WINDOW_ROUNDED) {
        double ib = round(ddiv(dsub(dsub(nu, J.cutoff), J.nu_start), J.dnu));
        double ie = round(ddiv(dsub(dadd(nu, J.cutoff), J.nu_start), J.dnu));
        double s0 = (double)J.start_idx, s1 = (double)(J.start_idx + J.n_points);
        ib = fmax(ib, s0); ie = fmin(ie, s1);
        double a = ib - (double)T.j0, b = ie - (double)T.j0;
        a = fmin(fmax(a, 0.0), (double)T.jn);
        b = fmin(fmax(b, 0.0), (double)T.jn);
        if (b < a) b = a;
        *pa = (int)a; *pb = (int)b;
        return;
    }
    /* inclusive rule: {t : |f_t - nu| <= cut} */
    const double cut = J.cutoff;
    auto in = [&](int t) {
        return fabs(dsub(grid_f(J.nu_start, J.dnu, T.j0 + t), nu)) <= cut;
    };
    double dmin = nu < T.f0 ? T.f0 - nu : (nu > T.fl ? nu - T.fl : 0.0);
    if (dmin > cut * (1.0 + 1e-12) + 1e-300) { *pa = *pb = 0; return; }
    if (in(0) && in(T.jn - 1)) { *pa = 0; *pb = T.jn; return; }
    int tcen = (int)fmin(fmax(rint(tc), 0.0), (double)(T.jn - 1));
    int anchor = -1;
    if (in(tcen)) anchor = tcen;
    else if (tcen > 0 && in(tcen - 1)) anchor = tcen - 1;
    else if (tcen + 1 < T.jn && in(tcen + 1)) anchor = tcen + 1;
    if (anchor < 0) { *pa = *pb = 0; return; }
    double w = cut * T.inv_dnu;   /* guesses only: first_true finds the ends */
    int gl = (int)fmin(fmax(ceil(tc - w), 0.0), (double)anchor);
    int gr = (int)fmin(fmax(floor(tc + w) + 1.0, (double)anchor), (double)T.jn);
    *pa = first_true(0, anchor, gl, [&](int t) { return in(t); });
    *pb = first_true(anchor, T.jn, gr, [&](int t) { return !in(t); });
}

/* bins of [wa, wb) (a sub-range of the tile) where dist-predicate `in`
 * holds; `in` must be true on one contiguous interval around the line
 * centre.  The predicate can only hold where (dist - off) * invw <= xthr;
 * the nearest bin's distance decides that without a division (a
 * conservative test: `in` takes the exact decisions), and the guesses for
 * the interval's ends come from the same limit. */
template <typename P>
__device__ __forceinline__ int centered(const Tile& T, int wa, int wb, double nu, double tc,
                                        double xthr, double invw, double off, const P& in)
{
    if (wa >= wb || !(xthr >= 0.0)) return 0;
    double fa = grid_f(T.J->nu_start, T.J->dnu, T.j0 + wa);
    double fb = grid_f(T.J->nu_start, T.J->dnu, T.j0 + wb - 1);
    double dmin = nu < fa ? fa - nu : (nu > fb ? nu - fb : 0.0);
    if ((dmin - off) * invw > xthr * (1.0 + 1e-9) + 1e-300) return 0;
    const double d_thr = xthr / invw + off;
    int tcen = (int)fmin(fmax(rint(tc), (double)wa), (double)(wb - 1));
    int anchor = -1;
    if (in(tcen)) anchor = tcen;
    else if (tcen > wa && in(tcen - 1)) anchor = tcen - 1;
    else if (tcen + 1 < wb && in(tcen + 1)) anchor = tcen + 1;
    if (anchor < 0) return 0;
    double w = d_thr / T.J->dnu;
    int gl = (int)fmin(fmax(ceil(tc - w), (double)wa), (double)anchor);
    int gr = (int)fmin(fmax(floor(tc + w) + 1.0, (double)anchor), (double)wb);
    int a = first_true(wa, anchor, gl, [&](int t) { return in(t); });
    int b = first_true(anchor, wb, gr, [&](int t) { return !in(t); });
    return pack2(a, b);
}

/* ------------------------------------------------------------ derive one line */
struct RawLine { double nu, elow, aif, gam, nexp; int g; };

/* FP64 per-line quantities of a job: centre (after the nu==0 rule), S(T),
 * 1/width and y = gammaL/width.  Either computed on load or read from the
 * job's prep arrays (prep_kernel). */
struct LineQ { double nu, S, invw, y; };

template <int PK>
struct Derived {
    double nu, S, invw, y, tc;
    int win, c1, c2, c3;
};

/* S(T) (Managers/CPU/OpenMPManager.cpp:394-396 operation order), the width
 * and y (:398,404) */
template <bool PRESS>
__device__ __forceinline__ LineQ line_quantities(const gexs_job& J, const RawLine& L)
{
    LineQ q;
    double nu = L.nu == 0.0 ? 1e-6 : L.nu;
    double t = dmul(J.s_scale, L.aif);
    t = dmul(t, (double)L.g);
    t = dmul(t, J.s_scale2);
    t = dmul(t, exp(dmul(-J.beta, L.elow)));
    t = dmul(t, dsub(1.0, exp(dmul(-J.beta, nu))));
    double den = dmul(dmul(nu, nu), J.partition);
    q.nu = nu;
    q.S = ddiv(t, den);
    q.invw = (J.profile == GEXS_GAUSSIAN) ? J.inv_width : ddiv(1.0, dmul(nu, J.dop_coef));
    if constexpr (PRESS) {
        double gl = dmul(L.gam, pow(J.t_ratio, L.nexp));
        gl = dmul(gl, J.gamma_scale);
        q.y = dmul(gl, q.invw);
    } else {
        q.y = 0.0;
    }
    return q;
}

/* tile-dependent part: centre in bins, window and Humlicek region limits
 * (inlined into the warp-specialised producers; derive_line below is the
 * out-of-line form for kernels that interleave it with their FP32 loops) */
template <int PK>
__device__ __forceinline__ Derived<PK> derive_line_body(const Tile& T, const LineQ& q, double zthr)
{
    const gexs_job& J = *T.J;
    Derived<PK> d;
    const double nu = q.nu;
    d.nu = nu; d.S = q.S; d.invw = q.invw; d.y = q.y;
    d.tc = dmul(dsub(nu, T.f0), T.inv_dnu);
    int a, b;
    tile_window(T, nu, d.tc, &a, &b);
    d.win = pack2(a, b);
    d.c1 = d.c2 = d.c3 = 0;
    if (a >= b || d.S == 0.0) { d.win = 0; return d; }
    const double invw = d.invw, y = d.y, nu_s = J.nu_start, dnu = J.dnu;
    const int64_t j0 = T.j0;
    auto xof = [&](int tt) { return dmul(fabs(dsub(grid_f(nu_s, dnu, j0 + tt), nu)), invw); };
    if constexpr (PK == PK_VOIGT) {
        /* region tests of compute/CPU/profiles.cpp:17,24,31 */
        d.c1 = centered(T, a, b, nu, d.tc, 15.0 - y, invw, 0.0,
                        [&](int tt) { return dadd(xof(tt), y) < 15.0; });
        if (lo16(d.c1) < hi16(d.c1)) {
            d.c2 = centered(T, lo16(d.c1), hi16(d.c1), nu, d.tc, 5.5 - y, invw, 0.0,
                            [&](int tt) { return dadd(xof(tt), y) < 5.5; });
            if (lo16(d.c2) < hi16(d.c2))
                d.c3 = centered(T, lo16(d.c2), hi16(d.c2), nu, d.tc, (y + 0.176) / 0.195, invw, 0.0,
                                [&](int tt) { return y >= dsub(dmul(0.195, xof(tt)), 0.176); });
        }
    } else if constexpr (PK == PK_ERF) {
        /* bins whose lower erf argument is <= zthr; beyond it both erfc
         * terms underflow to exactly zero */
        const double h = 0.5 * dnu;
        d.c1 = centered(T, a, b, nu, d.tc, zthr, invw, h,
                        [&](int tt) {
                            double dist = fabs(dsub(grid_f(nu_s, dnu, j0 + tt), nu));
                            return dmul(invw, dsub(dist, h)) <= zthr;
                        });
    }
    return d;
}

template <int PK>
__device__ __noinline__ Derived<PK> derive_line(const Tile& T, const LineQ& q, double zthr)
{
    return derive_line_body<PK>(T, q, zthr);
}

/* ------------------------------------------------------------ kernel args */
struct KArgs {
    const gexs_job* jobs;
    const int*      prefix;    /* njobs+1 tile prefix sums               */
    int             njobs;
    int             nitems;
    int*            counter;   /* work counter (zeroed before launch)    */
    int*            err;       /* sticky error word                      */
    double* const*  prep;      /* per job S|invw|y arrays, or NULL       */
    int             tile_w;    /* bins per work item (core kernel)       */
    SliceTables     sl;        /* line slices (sl.prefix NULL: none)     */
    SliceTables     csl;       /* FP32 Voigt core kernel's slices        */
    int             spin;      /* try_wait attempts of every bounded wait */
    const int*      order;     /* tile-major order tables F|R|P, or NULL
                                  for job-major items (gexs_capi.cu
                                  tile_order)                           */
};

/* flat tile index ti (the index the slice tables use) -> job, and the
 * tile of that job in *tile.  Job-major: the last job whose prefix is
 * <= ti.  Tile-major: the segment s of ti (last F[s] <= ti) has its first
 * nj - s ranked jobs active, one tile of each per row.  ORDER = false
 * compiles the job-major search alone (for builds that never see a.order). */
template <bool ORDER = true>
__device__ __forceinline__ int tile_job(const KArgs& a, int ti, int* tile)
{
    const int nj = a.njobs;
    if (ORDER && a.order) {
        const int* F = a.order;
        const int* R = F + nj + 1;
        const int* P = R + nj;
        int lo = 0, hi = nj;
        while (hi - lo > 1) { int m = (lo + hi) >> 1; if (__ldg(F + m) <= ti) lo = m; else hi = m; }
        const int act = nj - lo, d = ti - __ldg(F + lo);
        *tile = __ldg(R + lo) + d / act;
        return __ldg(P + d % act);
    }
    int jl = 0, jh = nj;
    while (jh - jl > 1) { int m = (jl + jh) >> 1; if (__ldg(a.prefix + m) <= ti) jl = m; else jh = m; }
    *tile = ti - __ldg(a.prefix + jl);
    return jl;
}

/* slice_plan_kernel + slice_scan_kernel (gexs_kernels.cu): every tile's
 * line range and slice count, then the item prefix and count */
cudaError_t launch_slice_plan(const KArgs& a, cudaStream_t st);
cudaError_t launch_core_slice_plan(const KArgs& a, cudaStream_t st);

__device__ __forceinline__ void kahan_add(float& s, float& c, float v)
{
    float yv = v - c;
    float t = s + yv;
    c = (t - s) - yv;
    s = t;
}

/* per-warp tiers of a line (bits of RecF*.mask).  Warp w owns bins
 * [32*B*w, 32*B*(w+1)) of the tile. */
template <int PK, int B, int WARPS>
__device__ __forceinline__ int warp_mask(const Derived<PK>& d, int wide)
{
    const int a = lo16(d.win), b = hi16(d.win);
    const int c1a = lo16(d.c1), c1b = hi16(d.c1);
    const int ic = (int)fmin(fmax(floor(d.tc), -1e6), 1e6);
    int m = 0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
        const int r0 = 32 * B * w, r1 = r0 + 32 * B;
        bool touch = a < r1 && b > r0;
        if (PK == PK_ERF) touch = touch && c1a < r1 && c1b > r0 && c1a < c1b;
        if (!touch) continue;
        m |= 1 << w;
        if (PK == PK_ERF || wide) continue;
        if (!(a <= r0 && b >= r1)) continue;
        /* GH: the single-FMA x of its fast tier keeps ~1e-7 relative
         * accuracy only when the centre is at least a warp span away */
        const bool far = ic < r0 - 32 * B || ic > r1 + 32 * B;
        m |= 1 << (far ? 8 + w : 16 + w);
    }
    return m | (wide << 24);
}

/* --------------------------------------------------------- record builders */
template <int PK, int B, int WARPS>
__device__ __forceinline__ void make_rec(RecF32& q, const Derived<PK>& d, const gexs_job& J,
                                         const Tile& T)
{
    double ic = floor(d.tc);
    ic = fmin(fmax(ic, -8388608.0), 8388607.0);
    double dx = dmul(J.dnu, d.invw);
    float fc = (float)(d.tc - ic);
    q.icf = (float)ic;
    q.dx = (float)dx;
    q.mfcdx = -fc * q.dx;
    double ampd = (PK == PK_ERF) ? dmul(d.S, J.out_scale) : dmul(dmul(d.S, d.invw), J.out_scale);
    q.amp = (float)ampd;
    bool pair = false;
    if constexpr (PK == PK_ERF) {
        q.a1 = 0.f; q.p = 0.f;
        q.y = (float)(0.5 * dx);
    } else {
        q.a1 = (float)(ampd * d.y * GEXS_INV_PI);
        q.p = (float)(d.y * d.y);
        /* dx and mf = -(tc - ic) dx as (high, low) float pairs from FP64 */
        const double mf = -(d.tc - ic) * dx;
        q.mfcdx = (float)mf;
        q.y = (float)(dx - (double)q.dx);
        q.amp = (float)(mf - (double)q.mfcdx);
        pair = d.y < 0.125;
    }
    q.fc = fc;
    q.win = d.win; q.c1 = d.c1;
    /* largest |x| the line reaches in this tile */
    double dfar = fmax(fabs(d.nu - T.f0), fabs(d.nu - T.fl));
    const int wide = (dfar * d.invw > 1e8) ? 1 : 0;
    q.mask = (d.win == 0) ? 0 : (warp_mask<PK, B, WARPS>(d, wide) | (pair && !wide ? GH_PAIR_BIT : 0));
    q.pad = 0;
}

/* per-warp tier codes of an FP32 Voigt record: 0 the line does not reach
 * the warp's bins, 1 full (all of them inside the window and outside the
 * core), 2 partial, 3 wide (overflow-free form) */
template <int B, int WARPS>
__device__ __forceinline__ int voigt_tiers(const Derived<PK_VOIGT>& d, int wide)
{
    const int a = lo16(d.win), b = hi16(d.win);
    const int c1a = lo16(d.c1), c1b = hi16(d.c1);
    int m = 0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
        const int r0 = 32 * B * w, r1 = r0 + 32 * B;
        if (!(a < r1 && b > r0)) continue;
        int t = 3;
        if (!wide) {
            const bool full = a <= r0 && b >= r1;
            const bool coredisj = c1a >= c1b || c1b <= r0 || c1a >= r1;
            t = (full && coredisj) ? 1 : 2;
        }
        m |= t << (2 * w);
    }
    return m;
}

template <int PK, int B, int WARPS>
__device__ __forceinline__ void make_rec(RecV& q, const Derived<PK>& d, const gexs_job& J,
                                         const Tile& T)
{
    double ic = floor(d.tc);
    ic = fmin(fmax(ic, -8388608.0), 8388607.0);
    const float fc = (float)(d.tc - ic);
    const float dx = (float)dmul(J.dnu, d.invw);
    const float mf = -fc * dx;
    const double ampd = dmul(dmul(d.S, d.invw), J.out_scale);
    /* region I as c y (m + 1) / (m^2 + 2 y^2), m = x^2 + y^2 - 1/2: the
     * same rational as c y (p + x^2) / ((p + x^2)^2 - 2 x^2), p = 1/2 +
     * y^2, with three FMAs and no cancellation in the denominator */
    const float a = (float)(ampd * 0.5641896 * d.y);
    const float c = (float)(d.y * d.y - 0.5);
    const float y2 = (float)(2.0 * d.y * d.y);
    const float icf = (float)ic;
    q.win = d.win; q.c1 = d.c1;
    /* largest |x| the line reaches in this tile */
    const double dfar = fmax(fabs(d.nu - T.f0), fabs(d.nu - T.fl));
    const int wide = (dfar * d.invw > 1e8) ? 1 : 0;
    q.tiers = (d.win == 0) ? 0 : voigt_tiers<B, WARPS>(d, wide);
    q.pad = __float_as_int(fc);
    q.dx = make_float2(dx, dx);
    q.mf = make_float2(mf, mf);
    q.c = make_float2(c, c);
    q.y2 = make_float2(y2, y2);
    q.a = make_float2(a, a);
    q.nb = make_float2(-icf, 32.f - icf);
}

template <int PK, int B, int WARPS>
__device__ __forceinline__ void make_rec(RecF64& q, const Derived<PK>& d, const gexs_job&,
                                         const Tile&)
{
    q.nu = d.nu; q.invw = d.invw; q.y = d.y;
    q.amp = (PK == PK_ERF) ? d.S : dmul(d.S, d.invw);
    q.win = d.win; q.c1 = d.c1; q.c2 = d.c2; q.c3 = d.c3;
    q.mask = (d.win == 0) ? 0 : warp_mask<PK, B, WARPS>(d, 1);
    q.pad0 = q.pad1 = q.pad2 = 0;
}


/* accumulator of bin k of a lane: pairs (2j, 2j+1) share one float2 so the
 * Voigt loop runs on packed f32x2 instructions; k is a compile-time
 * constant after unrolling */
template <int B>
__device__ __forceinline__ float& bin_acc(float2 (&part)[B / 2], int k)
{
    return (k & 1) ? part[k >> 1].y : part[k >> 1].x;
}

/* ------------------------------------------------- per-warp line loops
 * FP32 form of the Doppler/Gaussian and Gauss-Hermite profiles (the Voigt
 * form has its own loop, lines_voigt_f32).  Lane l of warp w owns bins
 * t_k = wb + l + 32k (k < B).
 * GH fast tier: whole warp in the window, centre >= one warp span away:
 *   x_k = fma(32k, dx, fma(l, dx, q)); otherwise per-bin window tests and
 *   x = ((l+32k + wb-ic) - fc)*dx exactly. */
template <int PK, int B>
__device__ __forceinline__ void lines_f32(const RecF32* __restrict__ rec, int nrec, int warp,
                                          int lane, float2 (&part)[B / 2])
{
    const int wb = warp * 32 * B;
    const float wbf = (float)wb, lanef = (float)lane;
    const int bit = 1 << warp;
    for (int i = 0; i < nrec; ++i) {
        const int4 qi = *reinterpret_cast<const int4*>(&rec[i].win);   /* win c1 mask pad */
        const int mask = qi.z;
        if (!(mask & bit)) continue;
        const float4 q0 = *reinterpret_cast<const float4*>(&rec[i].icf);   /* icf dx mfcdx a1 */
        const float4 q1 = *reinterpret_cast<const float4*>(&rec[i].p);     /* p y amp fc */
        const float ncf = wbf - q0.x;
        if constexpr (PK == PK_ERF) {
            const int a = lo16(qi.x), b = hi16(qi.x);
            const int c1a = lo16(qi.y), c1b = hi16(qi.y);
            const float t0 = lanef + ncf;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = wb + lane + 32 * k;
                if (t < a || t >= b || t < c1a || t >= c1b) continue;
                const float xd = fabsf(((t0 + (float)(32 * k)) - q1.w) * q0.y);
                /* FP32 always takes the cancellation-free form: the literal
                 * erf difference loses ~1e-7 absolute in FP32 far wings */
                float& acc = bin_acc<B>(part, k);
                acc = fmaf(q1.z, erf_bin_f32(xd - q1.y, xd + q1.y, GEXS_ERF_STABLE), acc);
            }
        } else {
            constexpr int NODES = (PK == PK_GH16) ? 16 : 32;
            if (mask & GH_PAIR_BIT) {
                /* narrow line: x as a float pair, per-bin window test */
                const int a = lo16(qi.x), b = hi16(qi.x);
                const float t0 = lanef + ncf;
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = wb + lane + 32 * k;
                    if (t < a || t >= b) continue;
                    float xs, xl;
                    x_pair(t0 + (float)(32 * k), q0.y, q1.y, q0.z, q1.z, xs, xl);
                    float& acc = bin_acc<B>(part, k);
                    acc = fmaf(q0.w, gh_sum_f32_pair<NODES>(xs, xl, q1.x), acc);
                }
                continue;
            }
            if (mask & (bit << 8)) {
                const float x0 = fmaf(lanef, q0.y, fmaf(ncf, q0.y, q0.z));
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    float& acc = bin_acc<B>(part, k);
                    acc = fmaf(q0.w, gh_sum_f32<NODES>(fabsf(fmaf((float)(32 * k), q0.y, x0)), q1.x),
                               acc);
                }
                continue;
            }
            const int a = lo16(qi.x), b = hi16(qi.x);
            const bool wide = (mask >> 24) & 1;
            const float t0 = lanef + ncf;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = wb + lane + 32 * k;
                if (t < a || t >= b) continue;
                const float x = fabsf(((t0 + (float)(32 * k)) - q1.w) * q0.y);
                const float g = wide ? gh_sum_f32_wide<NODES>(x, q1.x) : gh_sum_f32<NODES>(x, q1.x);
                float& acc = bin_acc<B>(part, k);
                acc = fmaf(q0.w, g, acc);
            }
        }
    }
}

/* FP32 Voigt main loop over RecV records.  Lane l of warp w owns bins
 * t_k = wb + l + 32k (k < B) as pairs (t_2j, t_2j+1); n = t - floor(tc) is
 * an exact integer, x = (n - fc) dx keeps full relative accuracy at every
 * distance from the centre.  Region I: x (FFMA2), m = x^2 + y^2 - 1/2
 * (FFMA2), d = m^2 + 2 y^2 (FFMA2), two MUFU reciprocals, t = (m + 1)/d
 * (FFMA2), accumulate a t (FFMA2), n += 64 (FADD2): 6 packed FP32 issues and
 * 2 MUFU per pair of bins.  Records are taken four (else two) at a time, all
 * their constants loaded first, so loads and arithmetic of several lines
 * overlap; a bin still sums its lines in ascending order. */
template <int B>
__device__ __forceinline__ void voigt_full2(const RecV& p, const RecV& q, float2 lw2,
                                            float2 (&part)[B / 2])
{
    const float2 step = make_float2(64.f, 64.f);
    const float2 pdx = p.dx, pmf = p.mf, pc = p.c, py2 = p.y2, pa = p.a;
    const float2 qdx = q.dx, qmf = q.mf, qc = q.c, qy2 = q.y2, qa = q.a;
    float2 np = __fadd2_rn(p.nb, lw2), nq = __fadd2_rn(q.nb, lw2);
#pragma unroll
    for (int j = 0; j < B / 2; ++j) {
        const float2 xp = __ffma2_rn(np, pdx, pmf), xq = __ffma2_rn(nq, qdx, qmf);
        const float2 mp = __ffma2_rn(xp, xp, pc), mq = __ffma2_rn(xq, xq, qc);
        const float2 dp = __ffma2_rn(mp, mp, py2), dq = __ffma2_rn(mq, mq, qy2);
        float2 rp, rq;
        rp.x = rcp_approx(dp.x); rp.y = rcp_approx(dp.y);
        rq.x = rcp_approx(dq.x); rq.y = rcp_approx(dq.y);
        const float2 tp = __ffma2_rn(mp, rp, rp), tq = __ffma2_rn(mq, rq, rq);
        part[j] = __ffma2_rn(tq, qa, __ffma2_rn(tp, pa, part[j]));
        np = __fadd2_rn(np, step); nq = __fadd2_rn(nq, step);
    }
}

template <int B>
__device__ __forceinline__ void voigt_one(const RecV& q, int tier, int wb, int lane, float2 lw2,
                                          float2 (&part)[B / 2])
{
    const float2 step = make_float2(64.f, 64.f);
    const float2 dx = q.dx, mf = q.mf, c = q.c, y2 = q.y2, a2 = q.a;
    float2 n2 = __fadd2_rn(q.nb, lw2);
    if (tier == 1) {
#pragma unroll
        for (int j = 0; j < B / 2; ++j) {
            const float2 x = __ffma2_rn(n2, dx, mf);
            const float2 m = __ffma2_rn(x, x, c);
            const float2 d = __ffma2_rn(m, m, y2);
            float2 r;
            r.x = rcp_approx(d.x); r.y = rcp_approx(d.y);
            part[j] = __ffma2_rn(__ffma2_rn(m, r, r), a2, part[j]);
            n2 = __fadd2_rn(n2, step);
        }
        return;
    }
    const int a = lo16(q.win), b = hi16(q.win);
    const int c1a = lo16(q.c1), c1b = hi16(q.c1);
    if (tier == 2) {
        /* partial: bins outside [a, b) or inside the core [c1a, c1b) are
         * evaluated but not accumulated (a core bin with y ~ 0 may give
         * inf/NaN here; it is discarded) */
        const unsigned wn = (unsigned)(b - a);
        const unsigned cn = c1b > c1a ? (unsigned)(c1b - c1a) : 0u;
        const int tl = wb + lane;
#pragma unroll
        for (int j = 0; j < B / 2; ++j) {
            const float2 x = __ffma2_rn(n2, dx, mf);
            const float2 m = __ffma2_rn(x, x, c);
            const float2 d = __ffma2_rn(m, m, y2);
            float2 r;
            r.x = rcp_approx(d.x); r.y = rcp_approx(d.y);
            const float2 v = __fmul2_rn(__ffma2_rn(m, r, r), a2);
            const int t0 = tl + 64 * j, t1 = t0 + 32;
            const bool in0 = (unsigned)(t0 - a) < wn && !((unsigned)(t0 - c1a) < cn);
            const bool in1 = (unsigned)(t1 - a) < wn && !((unsigned)(t1 - c1a) < cn);
            part[j].x += in0 ? v.x : 0.f;
            part[j].y += in1 ? v.y : 0.f;
            n2 = __fadd2_rn(n2, step);
        }
        return;
    }
    /* wide: |x| may exceed 1e8, num/den = 1/(num - 2 x^2/num) without num^2 */
    const float fc = __int_as_float(q.pad), p = c.x + 1.f;   /* 1/2 + y^2 */
#pragma unroll
    for (int k = 0; k < B; ++k) {
        const int t = wb + lane + 32 * k;
        if (t < a || t >= b || (t >= c1a && t < c1b)) continue;
        const float x = fabsf(((n2.x + (float)(32 * k)) - fc) * dx.x);
        const float x2 = x * x;
        const float num = x2 + p;
        bin_acc<B>(part, k) += (x < 1e18f) ? a2.x / (num - 2.f * (x2 / num)) : 0.f;
    }
}

/* four full-tier records: every constant loaded first, then two pairs */
template <int B>
__device__ __forceinline__ void voigt_full4(const RecV* __restrict__ r, float2 lw2,
                                            float2 (&part)[B / 2])
{
    RecV q[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        q[k].dx = r[k].dx; q[k].mf = r[k].mf; q[k].c = r[k].c;
        q[k].y2 = r[k].y2; q[k].a = r[k].a; q[k].nb = r[k].nb;
    }
    voigt_full2<B>(q[0], q[1], lw2, part);
    voigt_full2<B>(q[2], q[3], lw2, part);
}

/* Record-split form of the FP32 Voigt loop: every consumer warp covers
 * the whole tile (lane l owns bins l + 32k, k < B*CONS) and takes every
 * CONS-th record of a stage.  A record's constants are loaded once per
 * tile instead of once per warp, and its B*CONS/2 bin pairs are
 * independent chains.  Tier bits stay per quarter of 32*B bins (quarter q
 * = the bins a warp owns in the bins-split form): quarter q of a lane is
 * pairs q*B/2 .. q*B/2 + B/2 - 1. */
template <int B, int Q, int NPAIR>
__device__ __forceinline__ void voigt_quarter(const RecV& q, int tier, int lane, float2 n2,
                                              float2 (&part)[NPAIR])
{
    const float2 step = make_float2(64.f, 64.f);
    const float2 dx = q.dx, mf = q.mf, c = q.c, y2 = q.y2, a2 = q.a;
    constexpr int J0 = Q * (B / 2);
    if (tier == 1) {
#pragma unroll
        for (int j = 0; j < B / 2; ++j) {
            const float2 x = __ffma2_rn(n2, dx, mf);
            const float2 m = __ffma2_rn(x, x, c);
            const float2 d = __ffma2_rn(m, m, y2);
            float2 r;
            r.x = rcp_approx(d.x); r.y = rcp_approx(d.y);
            part[J0 + j] = __ffma2_rn(__ffma2_rn(m, r, r), a2, part[J0 + j]);
            n2 = __fadd2_rn(n2, step);
        }
        return;
    }
    const int a = lo16(q.win), b = hi16(q.win);
    const int c1a = lo16(q.c1), c1b = hi16(q.c1);
    const int tl = 32 * B * Q + lane;
    if (tier == 2) {
        const unsigned wn = (unsigned)(b - a);
        const unsigned cn = c1b > c1a ? (unsigned)(c1b - c1a) : 0u;
#pragma unroll
        for (int j = 0; j < B / 2; ++j) {
            const float2 x = __ffma2_rn(n2, dx, mf);
            const float2 m = __ffma2_rn(x, x, c);
            const float2 d = __ffma2_rn(m, m, y2);
            float2 r;
            r.x = rcp_approx(d.x); r.y = rcp_approx(d.y);
            const float2 v = __fmul2_rn(__ffma2_rn(m, r, r), a2);
            const int t0 = tl + 64 * j, t1 = t0 + 32;
            const bool in0 = (unsigned)(t0 - a) < wn && !((unsigned)(t0 - c1a) < cn);
            const bool in1 = (unsigned)(t1 - a) < wn && !((unsigned)(t1 - c1a) < cn);
            part[J0 + j].x += in0 ? v.x : 0.f;
            part[J0 + j].y += in1 ? v.y : 0.f;
            n2 = __fadd2_rn(n2, step);
        }
        return;
    }
    /* wide: |x| may exceed 1e8 */
    const float fc = __int_as_float(q.pad), p = c.x + 1.f;
#pragma unroll
    for (int k = 0; k < B; ++k) {
        const int t = tl + 32 * k;
        if (t < a || t >= b || (t >= c1a && t < c1b)) continue;
        const float x = fabsf(((n2.x + (float)(32 * k)) - fc) * dx.x);
        const float x2 = x * x;
        const float num = x2 + p;
        float& acc = (k & 1) ? part[J0 + (k >> 1)].y : part[J0 + (k >> 1)].x;
        acc += (x < 1e18f) ? a2.x / (num - 2.f * (x2 / num)) : 0.f;
    }
}

/* quarters Q .. CONS-1 of a record that is not full everywhere */
template <int B, int Q, int CONS>
struct RsQuarters {
    static __device__ __forceinline__ void run(const RecV& r, int tiers, int lane, float2 n0,
                                               float2 (&part)[B * CONS / 2])
    {
        const int t = (tiers >> (2 * Q)) & 3;
        /* quarter Q starts 32 B Q bins further: exact in float */
        if (t) voigt_quarter<B, Q>(r, t, lane, __fadd2_rn(n0, make_float2(32.f * B * Q, 32.f * B * Q)),
                                   part);
        RsQuarters<B, Q + 1, CONS>::run(r, tiers, lane, n0, part);
    }
};
template <int B, int CONS>
struct RsQuarters<B, CONS, CONS> {
    static __device__ __forceinline__ void run(const RecV&, int, int, float2, float2 (&)[B * CONS / 2]) {}
};

template <int B, int CONS>
__device__ __forceinline__ void voigt_rs_record(const RecV& r, int lane, float2 lw2,
                                                float2 (&part)[B * CONS / 2])
{
    constexpr int kAll = 0x55555555 & ((1 << (2 * CONS)) - 1);
    const int tiers = r.tiers;
    const float2 n0 = __fadd2_rn(r.nb, lw2);
    if (tiers == kAll) {
        const float2 dx = r.dx, mf = r.mf, c = r.c, y2 = r.y2, a2 = r.a;
        /* n of pair j is n0 + 64 j, built as a tree: n_j = n_{j-2^h} +
         * 64 * 2^h with 2^h the highest power of two in j.  The values are
         * the exact small integers that stepping n += 64 gives, with a
         * dependency depth of log2(pairs) instead of pairs - 1 (measured:
         * 1.4 ms less per 1e8-line cross-section, the same sums). */
        float2 nn[B * CONS / 2];
        nn[0] = n0;
#pragma unroll
        for (int j = 1; j < B * CONS / 2; ++j) {
            const int h = 31 - __clz(j);
            const float sj = 64.f * (float)(1 << h);
            nn[j] = __fadd2_rn(nn[j - (1 << h)], make_float2(sj, sj));
        }
#pragma unroll
        for (int j = 0; j < B * CONS / 2; ++j) {
            const float2 x = __ffma2_rn(nn[j], dx, mf);
            const float2 m = __ffma2_rn(x, x, c);
            const float2 d = __ffma2_rn(m, m, y2);
            float2 rr;
            rr.x = rcp_approx(d.x); rr.y = rcp_approx(d.y);
            part[j] = __ffma2_rn(__ffma2_rn(m, rr, rr), a2, part[j]);
        }
        return;
    }
    RsQuarters<B, 0, CONS>::run(r, tiers, lane, n0, part);
}

template <int B>
__device__ __forceinline__ void lines_voigt_f32(const RecV* __restrict__ rec, int nrec, int warp,
                                                int lane, float2 (&part)[B / 2])
{
    const int wb = warp * 32 * B, sh = 2 * warp;
    const float lw = (float)(wb + lane);
    const float2 lw2 = make_float2(lw, lw);
    int i = 0;
    for (; i + 3 < nrec; i += 4) {
        const int t0 = (rec[i].tiers >> sh) & 3, t1 = (rec[i + 1].tiers >> sh) & 3;
        const int t2 = (rec[i + 2].tiers >> sh) & 3, t3 = (rec[i + 3].tiers >> sh) & 3;
        if (t0 == 1 && t1 == 1 && t2 == 1 && t3 == 1) { voigt_full4<B>(rec + i, lw2, part); continue; }
        if (t0 == 1 && t1 == 1) voigt_full2<B>(rec[i], rec[i + 1], lw2, part);
        else {
            if (t0) voigt_one<B>(rec[i], t0, wb, lane, lw2, part);
            if (t1) voigt_one<B>(rec[i + 1], t1, wb, lane, lw2, part);
        }
        if (t2 == 1 && t3 == 1) voigt_full2<B>(rec[i + 2], rec[i + 3], lw2, part);
        else {
            if (t2) voigt_one<B>(rec[i + 2], t2, wb, lane, lw2, part);
            if (t3) voigt_one<B>(rec[i + 3], t3, wb, lane, lw2, part);
        }
    }
    for (; i + 1 < nrec; i += 2) {
        const int tp = (rec[i].tiers >> sh) & 3, tq = (rec[i + 1].tiers >> sh) & 3;
        if (tp == 1 && tq == 1) { voigt_full2<B>(rec[i], rec[i + 1], lw2, part); continue; }
        if (tp) voigt_one<B>(rec[i], tp, wb, lane, lw2, part);
        if (tq) voigt_one<B>(rec[i + 1], tq, wb, lane, lw2, part);
    }
    if (i < nrec) {
        const int tp = (rec[i].tiers >> sh) & 3;
        if (tp) voigt_one<B>(rec[i], tp, wb, lane, lw2, part);
    }
}

/* FP64 form: per-bin window and region tests, FP64 arithmetic, bins sum
 * their lines in line order (the order of the FP64 oracle). */
template <int PK, int B>
__device__ __forceinline__ void lines_f64(const RecF64* __restrict__ rec, int nrec, int warp,
                                          int lane, const double (&fbin)[B], double (&acc)[B],
                                          const gexs_job& J)
{
    const int wb = warp * 32 * B;
    const int bit = 1 << warp;
    const double out_scale = J.out_scale;
    for (int i = 0; i < nrec; ++i) {
        const RecF64& q = rec[i];
        if (!(q.mask & bit)) continue;
        const int a = lo16(q.win), b = hi16(q.win);
        if constexpr (PK == PK_VOIGT) {
            const int c1 = q.c1, c2 = q.c2, c3 = q.c3;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = wb + lane + 32 * k;
                if (t < a || t >= b) continue;
                double x = dmul(fabs(dsub(fbin[k], q.nu)), q.invw);
                int reg;
                if (t < lo16(c1) || t >= hi16(c1)) reg = 1;
                else if (t < lo16(c2) || t >= hi16(c2)) reg = 2;
                else reg = (t >= lo16(c3) && t < hi16(c3)) ? 3 : 4;
                double kv = hum_by_region<double>(reg, x, q.y);
                acc[k] = dadd(acc[k], dmul(dmul(q.amp, kv), out_scale));
            }
        } else if constexpr (PK == PK_ERF) {
            const int c1a = lo16(q.c1), c1b = hi16(q.c1);
            const int form = J.erf_form;
            const double h = 0.5 * J.dnu;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = wb + lane + 32 * k;
                if (t < a || t >= b || t < c1a || t >= c1b) continue;
                double dist = fabs(dsub(fbin[k], q.nu));
                double xp = dmul(q.invw, dadd(dist, h));
                double xm = dmul(q.invw, dsub(dist, h));
                double de = erf_bin_f64(xm, xp, form);
                acc[k] = dadd(acc[k], dmul(dmul(q.amp, de), out_scale));
            }
        } else {
            constexpr int NODES = (PK == PK_GH16) ? 16 : 32;
            const double y2 = dmul(q.y, q.y), yk = dmul(q.y, GEXS_INV_PI);
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = wb + lane + 32 * k;
                if (t < a || t >= b) continue;
                double x = dmul(fabs(dsub(fbin[k], q.nu)), q.invw);
                double kv = dmul(gh_sum_f64<NODES>(x, y2), yk);
                acc[k] = dadd(acc[k], dmul(dmul(q.amp, kv), out_scale));
            }
        }
    }
}

/* shared-memory layout of one CTA (dynamic shared memory) */
template <int PK, int PREC, int B, int WARPS, bool PREP>
struct Smem {
    static constexpr int NT = WARPS * 32;
    static constexpr int W = 32 * B * WARPS;
    static constexpr int R = PH * NT;                       /* lines per phase */
    static constexpr bool PRESS = (PK != PK_ERF);
    static constexpr size_t raw_d = (size_t)2 * NT * sizeof(double);   /* one f64 array, 2 bufs */
    /* staged per line: PREP nu S invw y ; on-load nu elow aif [gamma n] gns */
    static constexpr int NF64 = PREP ? 4 : (PRESS ? 5 : 3);
    static constexpr size_t off_gn = NF64 * raw_d;
    static constexpr size_t off_rec = (off_gn + (PREP ? 0 : (size_t)2 * NT * sizeof(int)) + 15) & ~size_t(15);
    static constexpr size_t rec_sz = sizeof(typename RecOf<PK, PREC>::T);
    /* FP32: Kahan (sum, compensation) per bin; each lane owns its bins */
    static constexpr size_t off_kahan = (off_rec + (size_t)R * rec_sz + 15) & ~size_t(15);
    static constexpr size_t bytes = off_kahan + (PREC == GEXS_FP32 ? (size_t)2 * W * sizeof(float) : 0);
};

/* ---------------------------------------------------------------- kernel */
/* resident CTAs per SM the register budget is sized for */
template <int B, int WARPS, int PREC>
constexpr int min_ctas()
{
    (void)PREC;
    return WARPS == 8 ? (B >= 8 ? 2 : 3) : (B >= 8 ? 4 : 6);
}

template <int PK, int PREC, int B, int WARPS, bool PREP>
__global__ void __launch_bounds__(WARPS * 32, min_ctas<B, WARPS, PREC>())
tile_kernel(const KArgs args)
{
    typedef Smem<PK, PREC, B, WARPS, PREP> L;
    static_assert(!(PK == PK_VOIGT && PREC == GEXS_FP32), "the FP32 Voigt form runs in voigt_ws_kernel");
    constexpr int NT = L::NT;
    constexpr int R = L::R;
    constexpr int W = 32 * B * WARPS;
    typedef typename RecOf<PK, PREC>::T Rec;

    extern __shared__ __align__(16) unsigned char smem[];
    /* staging arrays f[k][2*NT] (k < NF64) and gns[2*NT] */
    double* s_f = reinterpret_cast<double*>(smem);
    int*    s_gn = reinterpret_cast<int*>(smem + L::off_gn);
    Rec*    s_rec = reinterpret_cast<Rec*>(smem + L::off_rec);
    float*  s_ks = reinterpret_cast<float*>(smem + L::off_kahan);
    float*  s_kc = s_ks + W;
    __shared__ int s_item;
    __shared__ long long s_lohi[2];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double zthr = (PREC == GEXS_FP32) ? 10.5 : 27.5;

    const bool sliced = args.sl.prefix != nullptr;
    const int nitems = sliced ? *(volatile const int*)args.sl.nitems : args.nitems;
    __shared__ int s_last;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(args.counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= nitems) break;
        /* item -> (tile, slice): one item per tile unless sliced */
        int ti = item, sidx = 0, ns = 1;
        if (sliced) {
            int tl = 0, th = args.nitems;
            while (th - tl > 1) { int m = (tl + th) >> 1; if (__ldg(args.sl.prefix + m) <= item) tl = m; else th = m; }
            ti = tl;
            sidx = item - __ldg(args.sl.prefix + tl);
            ns = __ldg(args.sl.prefix + tl + 1) - __ldg(args.sl.prefix + tl);
        }

        /* job of this tile: last prefix entry <= tile */
        int tj = 0;
        const int jl = tile_job(args, ti, &tj);
        const gexs_job* Jp = args.jobs + jl;
        const gexs_job& J = *Jp;
        Tile T;
        T.J = Jp;
        T.j0 = J.start_idx + (int64_t)tj * W;
        T.jn = (int)min((int64_t)W, J.start_idx + J.n_points - T.j0);
        T.f0 = grid_f(J.nu_start, J.dnu, T.j0);
        T.fl = grid_f(J.nu_start, J.dnu, T.j0 + T.jn - 1);
        T.inv_dnu = 1.0 / J.dnu;

        const int64_t nl = J.lines.count;
        const double margin = 2.0 * J.dnu + 1e-9 * (fabs(T.fl) + J.cutoff);
        if (sliced) {
            if (tid == 0) {
                const long long tlo = __ldg(args.sl.lohi + 2 * ti), thi = __ldg(args.sl.lohi + 2 * ti + 1);
                const long long per = (thi - tlo + ns - 1) / ns;
                const long long a0 = tlo + (long long)sidx * per;
                s_lohi[0] = min(a0, thi);
                s_lohi[1] = min(a0 + per, thi);
            }
        } else if (warp == 0) {
            int64_t v = warp_bound<false>(J.lines.nu, nl, T.f0 - J.cutoff - margin, lane);
            if (lane == 0) s_lohi[0] = v;
        } else if (warp == 1) {
            int64_t v = warp_bound<true>(J.lines.nu, nl, T.fl + J.cutoff + margin, lane);
            if (lane == 0) s_lohi[1] = v;
        }
        __syncthreads();
        const int64_t lo = s_lohi[0];
        const int64_t hi = max((int64_t)s_lohi[1], lo);
        const int nph = (int)((hi - lo + R - 1) / R);
        if constexpr (PREC == GEXS_FP32) {
            /* Kahan pairs: touched only by the lane that owns the bin */
            for (int z = tid; z < W; z += NT) { s_ks[z] = 0.f; s_kc[z] = 0.f; }
            __syncthreads();
        }

        float2 part[B / 2];
        double acc[B], fbin[B];
#pragma unroll
        for (int k = 0; k < B; ++k) {
            acc[k] = 0.0;
            if (PREC == GEXS_FP64) fbin[k] = grid_f(J.nu_start, J.dnu, T.j0 + warp * 32 * B + lane + 32 * k);
        }
#pragma unroll
        for (int j = 0; j < B / 2; ++j) part[j] = make_float2(0.f, 0.f);

        /* thread tid stages and derives lines lo + u*NT + tid, u = 0, 1, ...;
         * every thread only ever reads the staging slots it filled itself,
         * so the double-buffered cp.async pipeline needs no barrier */
        const int nsub = nph * PH;
        const double* pb = nullptr;
        if constexpr (PREP) pb = args.prep[jl];
        auto issue = [&](int u) {
            const int64_t i = lo + (int64_t)u * NT + tid;
            const int o = (u & 1) * NT + tid;
            if (u < nsub && i < hi) {
                cp_async8(s_f + o, J.lines.nu + i);
                if constexpr (PREP) {
                    cp_async8(s_f + 2 * NT + o, pb + i);
                    cp_async8(s_f + 4 * NT + o, pb + nl + i);
                    cp_async8(s_f + 6 * NT + o, pb + 2 * nl + i);
                } else {
                    cp_async8(s_f + 2 * NT + o, J.lines.elow + i);
                    cp_async8(s_f + 4 * NT + o, J.lines.aif + i);
                    cp_async4(s_gn + o, J.lines.gns + i);
                    if constexpr (L::PRESS) {
                        cp_async8(s_f + 6 * NT + o, J.lines.gamma + i);
                        cp_async8(s_f + 8 * NT + o, J.lines.n + i);
                    }
                }
            }
            cp_async_commit();
        };
        issue(0);
        issue(1);

        for (int ph = 0; ph < nph; ++ph) {
            const int64_t pbase = lo + (int64_t)ph * R;
            const int nrec = (int)min((int64_t)R, hi - pbase);
#pragma unroll
            for (int sub = 0; sub < PH; ++sub) {
                const int u = ph * PH + sub;
                const int o = (u & 1) * NT + tid;
                cp_async_wait<1>();
                const int r = sub * NT + tid;
                if (r < nrec) {
                    LineQ lq;
                    if constexpr (PREP) {
                        const double nu = s_f[o];
                        lq.nu = nu == 0.0 ? 1e-6 : nu;
                        lq.S = s_f[2 * NT + o]; lq.invw = s_f[4 * NT + o]; lq.y = s_f[6 * NT + o];
                    } else {
                        RawLine Lr;
                        Lr.nu = s_f[o]; Lr.elow = s_f[2 * NT + o]; Lr.aif = s_f[4 * NT + o];
                        Lr.g = s_gn[o];
                        if constexpr (L::PRESS) { Lr.gam = s_f[6 * NT + o]; Lr.nexp = s_f[8 * NT + o]; }
                        else { Lr.gam = 0.0; Lr.nexp = 0.0; }
                        lq = line_quantities<L::PRESS>(J, Lr);
                    }
                    Derived<PK> d = derive_line<PK>(T, lq, zthr);
                    Rec rr;
                    make_rec<PK, B, WARPS>(rr, d, J, T);
                    s_rec[r] = rr;
                }
                issue(u + 2);
            }
            __syncthreads();

            if constexpr (PREC == GEXS_FP32) {
                /* Kahan merge of FP32 partial sums every 128 lines */
                for (int c0 = 0; c0 < nrec; c0 += 128) {
                    const int cn = min(128, nrec - c0);
                    lines_f32<PK, B>(reinterpret_cast<const RecF32*>(s_rec) + c0, cn, warp,
                                     lane, part);
#pragma unroll
                    for (int k = 0; k < B; ++k) {
                        const int t = warp * 32 * B + lane + 32 * k;
                        float ks = s_ks[t], kc = s_kc[t];
                        kahan_add(ks, kc, bin_acc<B>(part, k));
                        s_ks[t] = ks; s_kc[t] = kc;
                    }
#pragma unroll
                    for (int j = 0; j < B / 2; ++j) part[j] = make_float2(0.f, 0.f);
                }
            } else {
                lines_f64<PK, B>(reinterpret_cast<const RecF64*>(s_rec), nrec, warp, lane, fbin,
                                 acc, J);
            }
            __syncthreads();
        }
        cp_async_wait<0>();

        /* ------------------------------------------------------- write out */
        double* out = J.out;
        const int acc_mode = J.accumulate;
        if (ns == 1) {
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = warp * 32 * B + lane + 32 * k;
                if (t < T.jn) {
                    const double v = (PREC == GEXS_FP32) ? ((double)s_ks[t] - (double)s_kc[t]) : acc[k];
                    int64_t j = T.j0 + t;
                    out[j] = acc_mode ? out[j] + v : v;
                }
            }
        } else {
            /* one slice of a split tile: its partial row, then a ticket; the
             * last slice to finish adds the rows in slice order */
            const int base = args.sl.prefix[ti];
            const int rb = args.sl.rowbase[ti];
            double* row = args.sl.rows + (size_t)(rb + sidx) * W;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = warp * 32 * B + lane + 32 * k;
                if (t < T.jn) row[t] = (PREC == GEXS_FP32) ? ((double)s_ks[t] - (double)s_kc[t]) : acc[k];
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = atomicAdd(args.sl.ticket + ti, 1) == ns - 1;
            __syncthreads();
            if (s_last) {
                __threadfence();
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = warp * 32 * B + lane + 32 * k;
                    if (t < T.jn) {
                        double v = 0.0;
                        for (int q = 0; q < ns; ++q) v += __ldcg(args.sl.rows + (size_t)(rb + q) * W + t);
                        int64_t j = T.j0 + t;
                        out[j] = acc_mode ? out[j] + v : v;
                    }
                }
            }
            (void)base;
        }
        __syncthreads();
    }
}

/* ------------------------------------------ FP32 Voigt: warp-specialised
 * The region-I loop of the FP32 Voigt form runs in CONS consumer warps that
 * never wait at a CTA-wide barrier; PROD producer warps find each tile's
 * lines, stage them (cp.async, double-buffered) and derive their records
 * (FP64 S(T), width, window, core limits, per-warp tiers) into a ring of
 * WS_STAGES shared-memory stages of WS_R records.  A stage is handed over
 * through two mbarriers: `full` (every producer thread arrives after writing
 * its records) and `empty` (lane 0 of every consumer warp arrives after the
 * warp has read the stage).  Every wait is bounded: on timeout the thread
 * sets bit GEXS_KERR_PIPELINE of the launch's error word and returns, so a
 * fault in the hand-over ends the kernel with an error instead of a hang.
 * Two consumer forms:
 *  - bins-split (every shape but the 512-bin tiles): warp w
 *    owns bins [32 B w, 32 B (w+1)) and reads every record; its FP32
 *    partial sums live in registers and its Kahan pairs in shared memory
 *    (lane-private), so a tile boundary needs no barrier: the first stage
 *    of a tile zeroes them, the last writes the bins out.  Each bin sums
 *    its lines in ascending order.
 *  - record-split (512-bin tiles: B = 4 with four consumer warps, the
 *    default, or B = 2 with eight): every warp covers the whole tile (16
 *    bins per lane) and takes every CONS-th record of a stage into Kahan
 *    pairs of its own; at the end of a tile the warps meet (bounded
 *    mbarrier) and warp w writes its 32 B bins as the sum of all warps'
 *    pairs in warp order.  A record is read from shared memory once instead
 *    of CONS times and gives eight independent bin-pair chains; measured
 *    200.6 ms against 236.6 ms per 1e8-line cross-section for the
 *    bins-split form of the 4 x 4 shape (229 against 348 ms for 2 x 8).
 * Either way a bin's sum depends only on its tile's records, so results
 * are bitwise independent of batching. */
constexpr int WS_RING = 512;             /* records in the ring: stages x records per stage */
constexpr int WS_SPIN = 1 << 21;          /* default try_wait attempts before giving up */

struct StageHdr {
    long long j0;          /* absolute first bin of the tile                */
    int jl;                /* job index                                     */
    int jn;                /* bins in the tile                              */
    int nrec;              /* records in this stage                         */
    int flags;             /* 1 first stage of the tile, 2 last, 4 end,
                              8 the item is one slice of a split tile       */
    int item, tile;        /* work item and its tile                        */
};

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(b)) : "memory");
}
/* bounded wait for the completion of the phase with parity `parity`; a
 * waiting warp backs off (nanosleep, doubling up to 256 ns) so that it does
 * not take issue slots from the warps that do the work */
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity, int limit)
{
    const unsigned a = smem_u32(b);
    unsigned ns = 16;
    for (int it = 0; it < limit; ++it) {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
    return false;
}

template <int B, int CONS, int PROD, bool PREP, int SR>
struct WsSmem {
    static constexpr int WS_R = SR, WS_STAGES = WS_RING / SR;
    static constexpr int NP = PROD * 32;
    static constexpr int W = 32 * B * CONS;
    static constexpr int NF64 = PREP ? 4 : 5;
    static constexpr size_t off_rec = 0;
    static constexpr size_t off_hdr = off_rec + (size_t)WS_STAGES * WS_R * sizeof(RecV);
    static constexpr size_t off_bar = off_hdr + (size_t)WS_STAGES * sizeof(StageHdr);
    /* mbarriers: full[WS_STAGES], empty[WS_STAGES], producers' own barrier,
     * consumers' own barrier */
    static constexpr size_t off_stg = off_bar + (size_t)(2 * WS_STAGES + 2) * sizeof(unsigned long long);
    static constexpr size_t off_gn = off_stg + (size_t)NF64 * 2 * NP * sizeof(double);
    static constexpr size_t off_kahan = (off_gn + (PREP ? 0 : (size_t)2 * NP * sizeof(int)) + 15) & ~size_t(15);
    /* record-split consumers (512-bin tiles: B = 4 with four consumer
     * warps, B = 2 with eight): one Kahan pair per bin and warp */
    static constexpr bool RS = (B * CONS == 16);
    static constexpr size_t bytes = off_kahan + (size_t)(RS ? CONS : 1) * 2 * W * sizeof(float);
};

template <int B, int CONS, int PROD, bool PREP, int SR>
__global__ void __launch_bounds__((CONS + PROD) * 32, CONS == 4 ? (B >= 8 ? 3 : 4) : 2)
voigt_ws_kernel(const KArgs args)
{
    typedef WsSmem<B, CONS, PROD, PREP, SR> L;
    constexpr int WS_R = SR, WS_STAGES = WS_RING / SR;
    constexpr int NP = L::NP, W = L::W;
    constexpr int SUB = WS_R / NP;               /* lines per producer thread per stage */
    static_assert(WS_R % NP == 0, "stage size must be a multiple of the producer threads");
    extern __shared__ __align__(16) unsigned char smem[];
    RecV* s_rec = reinterpret_cast<RecV*>(smem + L::off_rec);
    StageHdr* s_hdr = reinterpret_cast<StageHdr*>(smem + L::off_hdr);
    unsigned long long* s_full = reinterpret_cast<unsigned long long*>(smem + L::off_bar);
    unsigned long long* s_empty = s_full + WS_STAGES;
    unsigned long long* s_pbar = s_empty + WS_STAGES;
    double* s_f = reinterpret_cast<double*>(smem + L::off_stg);
    int* s_gn = reinterpret_cast<int*>(smem + L::off_gn);
    float* s_ks = reinterpret_cast<float*>(smem + L::off_kahan);
    float* s_kc = s_ks + W;
    __shared__ int s_item;
    __shared__ long long s_lohi[2];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool sliced = args.sl.prefix != nullptr;
    const int nitems = sliced ? *(volatile const int*)args.sl.nitems : args.nitems;
    if (tid == 0) {
        for (int st = 0; st < WS_STAGES; ++st) { mbar_init(s_full + st, NP); mbar_init(s_empty + st, CONS); }
        mbar_init(s_pbar, NP);
        mbar_init(s_pbar + 1, CONS);
    }
    __syncthreads();   /* the only CTA-wide barrier: before the roles split */

    if (warp >= CONS) {
        /* ------------------------------------------------------ producers */
        const int ptid = tid - CONS * 32, pw = warp - CONS;
        int st = 0;
        unsigned ph = 1;   /* a fresh `empty` barrier counts as released */
        unsigned pph = 0;
        /* on a timed-out wait: flag it, let this thread's copies land, return */
        auto fail = [&]() {
            atomicOr(args.err, GEXS_KERR_PIPELINE);
            cp_async_wait<0>();
        };
        /* barrier among the producer threads, bounded like every wait here */
        auto psync = [&]() -> bool {
            mbar_arrive(s_pbar);
            const bool ok = mbar_wait(s_pbar, pph, args.spin);
            pph ^= 1;
            return ok;
        };
        for (;;) {
            if (ptid == 0) s_item = atomicAdd(args.counter, 1);
            if (!psync()) { fail(); return; }
            const int item = s_item;
            if (item >= nitems) {
                if (!mbar_wait(s_empty + st, ph, args.spin)) { fail(); return; }
                if (ptid == 0) { s_hdr[st].flags = 4; s_hdr[st].nrec = 0; }
                mbar_arrive(s_full + st);
                return;
            }
            /* item -> (tile, slice): one item per tile unless sliced */
            int ti = item, sidx = 0, ns = 1;
            if (sliced) {
                int tl = 0, th = args.nitems;
                while (th - tl > 1) { int m = (tl + th) >> 1; if (__ldg(args.sl.prefix + m) <= item) tl = m; else th = m; }
                ti = tl;
                sidx = item - __ldg(args.sl.prefix + tl);
                ns = __ldg(args.sl.prefix + tl + 1) - __ldg(args.sl.prefix + tl);
            }
            int tj = 0;
            const int jl = tile_job(args, ti, &tj);
            const gexs_job* Jp = args.jobs + jl;
            const gexs_job& J = *Jp;
            Tile T;
            T.J = Jp;
            T.j0 = J.start_idx + (int64_t)tj * W;
            T.jn = (int)min((int64_t)W, J.start_idx + J.n_points - T.j0);
            T.f0 = grid_f(J.nu_start, J.dnu, T.j0);
            T.fl = grid_f(J.nu_start, J.dnu, T.j0 + T.jn - 1);
            T.inv_dnu = 1.0 / J.dnu;
            const int64_t nl = J.lines.count;
            const double margin = 2.0 * J.dnu + 1e-9 * (fabs(T.fl) + J.cutoff);
            if (sliced) {
                /* the tile's range from slice_plan_kernel, cut into ns equal parts */
                if (ptid == 0) {
                    const long long tlo = __ldg(args.sl.lohi + 2 * ti), thi = __ldg(args.sl.lohi + 2 * ti + 1);
                    const long long per = (thi - tlo + ns - 1) / ns;
                    const long long a0 = tlo + (long long)sidx * per;
                    s_lohi[0] = min(a0, thi);
                    s_lohi[1] = min(a0 + per, thi);
                }
            } else {
                if (pw == 0) {
                    int64_t v = warp_bound<false>(J.lines.nu, nl, T.f0 - J.cutoff - margin, lane);
                    if (lane == 0) s_lohi[0] = v;
                }
                if (pw == (PROD > 1 ? 1 : 0)) {
                    int64_t v = warp_bound<true>(J.lines.nu, nl, T.fl + J.cutoff + margin, lane);
                    if (lane == 0) s_lohi[1] = v;
                }
            }
            if (!psync()) { fail(); return; }
            const int64_t lo = s_lohi[0];
            const int64_t hi = max((int64_t)s_lohi[1], lo);
            const int nchunk = max(1, (int)((hi - lo + WS_R - 1) / WS_R));
            const int nsub = nchunk * SUB;
            const double* pb = nullptr;
            if constexpr (PREP) pb = args.prep[jl];
            /* producer thread ptid stages and derives lines lo + u*NP + ptid;
             * it reads only the staging slots it filled itself */
            auto issue = [&](int u) {
                const int64_t i = lo + (int64_t)u * NP + ptid;
                const int o = (u & 1) * NP + ptid;
                if (u < nsub && i < hi) {
                    cp_async8(s_f + o, J.lines.nu + i);
                    if constexpr (PREP) {
                        cp_async8(s_f + 2 * NP + o, pb + i);
                        cp_async8(s_f + 4 * NP + o, pb + nl + i);
                        cp_async8(s_f + 6 * NP + o, pb + 2 * nl + i);
                    } else {
                        cp_async8(s_f + 2 * NP + o, J.lines.elow + i);
                        cp_async8(s_f + 4 * NP + o, J.lines.aif + i);
                        cp_async4(s_gn + o, J.lines.gns + i);
                        cp_async8(s_f + 6 * NP + o, J.lines.gamma + i);
                        cp_async8(s_f + 8 * NP + o, J.lines.n + i);
                    }
                }
                cp_async_commit();
            };
            issue(0);
            issue(1);
            for (int c = 0; c < nchunk; ++c) {
                if (!mbar_wait(s_empty + st, ph, args.spin)) { fail(); return; }
                const int64_t pbase = lo + (int64_t)c * WS_R;
                const int nrec = (int)max((int64_t)0, min((int64_t)WS_R, hi - pbase));
                RecV* rec = s_rec + st * WS_R;
#pragma unroll
                for (int sub = 0; sub < SUB; ++sub) {
                    const int u = c * SUB + sub;
                    const int o = (u & 1) * NP + ptid;
                    cp_async_wait<1>();
                    const int r = sub * NP + ptid;
                    if (r < nrec) {
                        LineQ lq;
                        if constexpr (PREP) {
                            const double nu = s_f[o];
                            lq.nu = nu == 0.0 ? 1e-6 : nu;
                            lq.S = s_f[2 * NP + o]; lq.invw = s_f[4 * NP + o]; lq.y = s_f[6 * NP + o];
                        } else {
                            RawLine Lr;
                            Lr.nu = s_f[o]; Lr.elow = s_f[2 * NP + o]; Lr.aif = s_f[4 * NP + o];
                            Lr.g = s_gn[o]; Lr.gam = s_f[6 * NP + o]; Lr.nexp = s_f[8 * NP + o];
                            lq = line_quantities<true>(J, Lr);
                        }
                        Derived<PK_VOIGT> d = derive_line_body<PK_VOIGT>(T, lq, 10.5);
                        RecV rr;
                        make_rec<PK_VOIGT, B, CONS>(rr, d, J, T);
                        rec[r] = rr;
                    }
                    issue(u + 2);
                }
                if (ptid == 0) {
                    StageHdr h;
                    h.j0 = T.j0; h.jl = jl; h.jn = T.jn; h.nrec = nrec;
                    h.flags = (c == 0 ? 1 : 0) | (c == nchunk - 1 ? 2 : 0) | (ns > 1 ? 8 : 0);
                    h.item = item;
                    h.tile = ti;
                    s_hdr[st] = h;
                }
                mbar_arrive(s_full + st);
                if (++st == WS_STAGES) { st = 0; ph ^= 1; }
            }
            cp_async_wait<0>();
            /* every producer is past s_item and s_lohi */
            if (!psync()) { fail(); return; }
        }
    }

    /* ---------------------------------------------------------- consumers */
    int st = 0;
    unsigned ph = 0;
    /* barrier among the consumer warps (a split tile's merge), bounded */
    unsigned cph = 0;
    __shared__ int s_last;
    auto csync = [&]() -> bool {
        __syncwarp();
        if (lane == 0) mbar_arrive(s_pbar + 1);
        const bool ok = mbar_wait(s_pbar + 1, cph, args.spin);
        cph ^= 1;
        return ok;
    };
    if constexpr (L::RS) {
        /* record-split: warp w adds records w, w + CONS, ... of every stage
         * into its own Kahan pairs of all W bins; at the end of a tile the
         * warps meet, and warp w writes bins [32 B w, 32 B (w+1)) as the sum
         * of the CONS warps' pairs in warp order */
        constexpr int BL = B * CONS;
        float* my_ks = s_ks + (size_t)warp * 2 * W;
        float* my_kc = my_ks + W;
        float2 part[BL / 2];
#pragma unroll
        for (int j = 0; j < BL / 2; ++j) part[j] = make_float2(0.f, 0.f);
        const float2 lw2 = make_float2((float)lane, (float)lane);
        for (;;) {
            if (!mbar_wait(s_full + st, ph, args.spin)) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
            const StageHdr h = s_hdr[st];
            if (h.flags & 4) return;
            if (h.flags & 1) {
#pragma unroll
                for (int k = 0; k < BL; ++k) { my_ks[lane + 32 * k] = 0.f; my_kc[lane + 32 * k] = 0.f; }
            }
            const RecV* rec = s_rec + st * WS_R;
            for (int i = warp; i < h.nrec; i += CONS) voigt_rs_record<B, CONS>(rec[i], lane, lw2, part);
#pragma unroll
            for (int k = 0; k < BL; ++k) {
                const int t = lane + 32 * k;
                float ks = my_ks[t], kc = my_kc[t];
                kahan_add(ks, kc, (k & 1) ? part[k >> 1].y : part[k >> 1].x);
                my_ks[t] = ks; my_kc[t] = kc;
            }
#pragma unroll
            for (int j = 0; j < BL / 2; ++j) part[j] = make_float2(0.f, 0.f);
            /* the stage's records are consumed: hand the slot back first */
            __syncwarp();
            if (lane == 0) mbar_arrive(s_empty + st);
            if (++st == WS_STAGES) { st = 0; ph ^= 1; }
            if (!(h.flags & 2)) continue;
            if (!csync()) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
            double v[B];
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = warp * 32 * B + lane + 32 * k;
                double acc = 0.0;
#pragma unroll
                for (int w = 0; w < CONS; ++w)
                    acc += (double)s_ks[(size_t)w * 2 * W + t] - (double)s_ks[(size_t)w * 2 * W + W + t];
                v[k] = acc;
            }
            const gexs_job& J = args.jobs[h.jl];
            double* out = J.out;
            if (!(h.flags & 8)) {
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = warp * 32 * B + lane + 32 * k;
                    if (t < h.jn) {
                        const int64_t j = h.j0 + t;
                        out[j] = J.accumulate ? out[j] + v[k] : v[k];
                    }
                }
            } else {
                const int base = args.sl.prefix[h.tile];
                const int ns = args.sl.prefix[h.tile + 1] - base;
                const int rb = args.sl.rowbase[h.tile];
                double* row = args.sl.rows + (size_t)(rb + (h.item - base)) * W;
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = warp * 32 * B + lane + 32 * k;
                    if (t < h.jn) row[t] = v[k];
                }
                __threadfence();
                if (!csync()) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
                if (tid == 0) s_last = atomicAdd(args.sl.ticket + h.tile, 1) == ns - 1;
                if (!csync()) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
                if (s_last) {
                    __threadfence();
#pragma unroll
                    for (int k = 0; k < B; ++k) {
                        const int t = warp * 32 * B + lane + 32 * k;
                        if (t < h.jn) {
                            double acc = 0.0;
                            for (int q = 0; q < ns; ++q) acc += __ldcg(args.sl.rows + (size_t)(rb + q) * W + t);
                            const int64_t j = h.j0 + t;
                            out[j] = J.accumulate ? out[j] + acc : acc;
                        }
                    }
                }
            }
            /* every warp has read the Kahan pairs before the next tile clears them */
            if (!csync()) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
        }
    }
    else {
        float2 part[B / 2];
#pragma unroll
        for (int j = 0; j < B / 2; ++j) part[j] = make_float2(0.f, 0.f);
        for (;;) {
            if (!mbar_wait(s_full + st, ph, args.spin)) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
            const StageHdr h = s_hdr[st];
            if (h.flags & 4) return;
            if (h.flags & 1) {
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = warp * 32 * B + lane + 32 * k;
                    s_ks[t] = 0.f; s_kc[t] = 0.f;
                }
            }
            const RecV* rec = s_rec + st * WS_R;
            lines_voigt_f32<B>(rec, h.nrec, warp, lane, part);
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const int t = warp * 32 * B + lane + 32 * k;
                float ks = s_ks[t], kc = s_kc[t];
                kahan_add(ks, kc, bin_acc<B>(part, k));
                s_ks[t] = ks; s_kc[t] = kc;
            }
#pragma unroll
            for (int j = 0; j < B / 2; ++j) part[j] = make_float2(0.f, 0.f);
            if ((h.flags & 2) && !(h.flags & 8)) {
                const gexs_job& J = args.jobs[h.jl];
                double* out = J.out;
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = warp * 32 * B + lane + 32 * k;
                    if (t < h.jn) {
                        const double v = (double)s_ks[t] - (double)s_kc[t];
                        const int64_t j = h.j0 + t;
                        out[j] = J.accumulate ? out[j] + v : v;
                    }
                }
            } else if (h.flags & 2) {
                /* one slice of a split tile: its partial row, then a ticket; the
                 * last slice to finish adds the rows in slice order */
                const gexs_job& J = args.jobs[h.jl];
                double* out = J.out;
                const int base = args.sl.prefix[h.tile];
                const int ns = args.sl.prefix[h.tile + 1] - base;
                const int rb = args.sl.rowbase[h.tile];
                double* row = args.sl.rows + (size_t)(rb + (h.item - base)) * W;
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = warp * 32 * B + lane + 32 * k;
                    if (t < h.jn) row[t] = (double)s_ks[t] - (double)s_kc[t];
                }
                __threadfence();
                if (!csync()) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
                if (tid == 0) s_last = atomicAdd(args.sl.ticket + h.tile, 1) == ns - 1;
                if (!csync()) { atomicOr(args.err, GEXS_KERR_PIPELINE); return; }
                if (s_last) {
                    __threadfence();
#pragma unroll
                    for (int k = 0; k < B; ++k) {
                        const int t = warp * 32 * B + lane + 32 * k;
                        if (t < h.jn) {
                            double v = 0.0;
                            for (int q = 0; q < ns; ++q) v += __ldcg(args.sl.rows + (size_t)(rb + q) * W + t);
                            const int64_t j = h.j0 + t;
                            out[j] = J.accumulate ? out[j] + v : v;
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(s_empty + st);
            if (++st == WS_STAGES) { st = 0; ph ^= 1; }
        }
    }
}

/* ------------------------------------------------- FP32 Voigt core kernel
 * The core of a line (its bins outside Humlicek region I: regions II, III,
 * IV) is evaluated here, after the region-I kernel, and added into the
 * output.  Kept out of that kernel so it carries no FP64 Humlicek code and
 * no core accumulator rows.
 *
 * Work items are the region-I kernel's tiles, each taken in sub-tiles of at
 * most CORE_W bins.  Per sub-tile, the lines whose core can reach it
 * (|f - nu| < 15 / invw = 15 nu dop_coef, inside the cutoff) are found by
 * two warp searches and taken 32 at a time by the warps in turn, one line
 * per lane, derived in FP64 with the region-I kernel's predicates.  A warp
 * then steps through the union of its 32 lines' cores bin by bin: at bin t
 * every lane evaluates its own line in the region t falls in (II in FP32,
 * III and the rational part of IV in FP64, IV's exp term in FP32), a
 * butterfly of shuffles sums the 32 terms in a fixed order, and lane 0
 * adds the sum into the warp's row of doubles.  Lines that
 * are neighbours in nu have overlapping cores, so most lanes work at every
 * step and no lane scans for work.  A bin receives its core terms in a
 * fixed order (groups of 32 lines in ascending order per warp, rows added
 * in warp order), so results are bitwise independent of batching. */
constexpr int CORE_W = 1024;
constexpr int CORE_WARPS = 4;

struct CoreSmem {
    static constexpr int NT = CORE_WARPS * 32;
    static constexpr size_t bytes = (size_t)CORE_WARPS * CORE_W * sizeof(double);
};

/* the core of a line as single-region bin ranges, c3 within c2 within c1
 * (an empty inner range collapses to a point):
 * II = [c1a, c2a) u [c2b, c1b), III = [c3a, c3b), IV = [c2a, c3a) u [c3b, c2b) */
__device__ __forceinline__ void core_ranges(int c1, int c2, int c3, int& c1a, int& c1b,
                                            int& c2a, int& c2b, int& c3a, int& c3b)
{
    c1a = lo16(c1); c1b = hi16(c1);
    c2a = lo16(c2); c2b = hi16(c2);
    if (c2a >= c2b) c2a = c2b = c1b;
    c3a = lo16(c3); c3b = hi16(c3);
    if (c3a >= c3b) c3a = c3b = c2b;
}

/* ORDER: the launch's items may be tile-major (its own instantiation: the
 * decode's divisions cost this kernel 8 registers when compiled in) */
template <bool PREP, bool ORDER>
__global__ void __launch_bounds__(CORE_WARPS * 32)
core_kernel(const KArgs args)
{
    constexpr int NT = CoreSmem::NT;
    extern __shared__ __align__(16) unsigned char smem[];
    double* s_rows = reinterpret_cast<double*>(smem);
    __shared__ int s_item;
    __shared__ long long s_lohi[2];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* row = s_rows + warp * CORE_W;
    /* sliced (host-enabled only when a tile is one sub-tile of CORE_W) */
    const bool sliced = args.csl.prefix != nullptr;
    const int nitems = sliced ? *(volatile const int*)args.csl.nitems : args.nitems;
    __shared__ int s_last;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(args.counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= nitems) break;
        int ti = item, sidx = 0, ns = 1;
        if (sliced) {
            int tl = 0, th = args.nitems;
            while (th - tl > 1) { int m = (tl + th) >> 1; if (__ldg(args.csl.prefix + m) <= item) tl = m; else th = m; }
            ti = tl;
            sidx = item - __ldg(args.csl.prefix + tl);
            ns = __ldg(args.csl.prefix + tl + 1) - __ldg(args.csl.prefix + tl);
        }
        int tj = 0;
        const int jl = tile_job<ORDER>(args, ti, &tj);
        const gexs_job* Jp = args.jobs + jl;
        const gexs_job& J = *Jp;
        /* the region-I kernel's tile of this item */
        const int64_t t0 = J.start_idx + (int64_t)tj * args.tile_w;
        const int64_t tend = min((int64_t)(t0 + args.tile_w), J.start_idx + J.n_points);
        const int64_t nl = J.lines.count;
        const double* pb = PREP ? args.prep[jl] : nullptr;
        const double k15 = 15.0 * J.dop_coef;
        for (int64_t s0 = t0; s0 < tend; s0 += CORE_W) {
            Tile T;
            T.J = Jp;
            T.j0 = s0;
            T.jn = (int)min((int64_t)CORE_W, tend - s0);
            T.f0 = grid_f(J.nu_start, J.dnu, T.j0);
            T.fl = grid_f(J.nu_start, J.dnu, T.j0 + T.jn - 1);
            T.inv_dnu = 1.0 / J.dnu;
            const double margin = 2.0 * J.dnu + 1e-9 * (fabs(T.fl) + J.cutoff);
            /* a core reaches f only if |f - nu| < 15 nu dop_coef */
            double vlo = T.f0 - J.cutoff, vhi = T.fl + J.cutoff;
            vlo = fmax(vlo, T.f0 / (1.0 + k15));
            if (k15 < 1.0) vhi = fmin(vhi, T.fl / (1.0 - k15));
            vlo -= margin; vhi += margin;
            if (vlo < 1e-6 + margin) vlo = -1.0;   /* nu == 0 lines count as 1e-6 */
            if (sliced) {
                /* the range from core_slice_plan_kernel, cut into ns parts */
                if (tid == 0) {
                    const long long tlo = __ldg(args.csl.lohi + 2 * ti), thi = __ldg(args.csl.lohi + 2 * ti + 1);
                    const long long per = (thi - tlo + ns - 1) / ns;
                    const long long a0 = tlo + (long long)sidx * per;
                    s_lohi[0] = min(a0, thi);
                    s_lohi[1] = min(a0 + per, thi);
                }
            } else if (warp == 0) {
                int64_t v = warp_bound<false>(J.lines.nu, nl, vlo, lane);
                if (lane == 0) s_lohi[0] = v;
            } else if (warp == 1) {
                int64_t v = warp_bound<true>(J.lines.nu, nl, vhi, lane);
                if (lane == 0) s_lohi[1] = v;
            }
            for (int z = tid; z < CORE_WARPS * CORE_W; z += NT) s_rows[z] = 0.0;
            __syncthreads();
            const int64_t lo = s_lohi[0], hi = max((int64_t)s_lohi[1], lo);
            for (int64_t g0 = lo + (int64_t)warp * 32; g0 < hi; g0 += NT) {
                const int64_t i = g0 + lane;
                bool has = false;
                int c1a = 0, c1b = 0, c2a = 0, c2b = 0, c3a = 0, c3b = 0;
                double nu = 0.0, invw = 0.0, y = 0.0, amp = 0.0;
                float icf = 0.f, fc = 0.f, dx = 0.f, yf = 0.f, ampf = 0.f;
                if (i < hi) {
                    LineQ lq;
                    if constexpr (PREP) {
                        const double v = __ldg(J.lines.nu + i);
                        lq.nu = v == 0.0 ? 1e-6 : v;
                        lq.S = __ldg(pb + i); lq.invw = __ldg(pb + nl + i); lq.y = __ldg(pb + 2 * nl + i);
                    } else {
                        RawLine Lr;
                        Lr.nu = __ldg(J.lines.nu + i); Lr.elow = __ldg(J.lines.elow + i);
                        Lr.aif = __ldg(J.lines.aif + i); Lr.g = __ldg(J.lines.gns + i);
                        Lr.gam = __ldg(J.lines.gamma + i); Lr.nexp = __ldg(J.lines.n + i);
                        lq = line_quantities<true>(J, Lr);
                    }
                    Derived<PK_VOIGT> d = derive_line<PK_VOIGT>(T, lq, 10.5);
                    if (lo16(d.c1) < hi16(d.c1)) {
                        has = true;
                        core_ranges(d.c1, d.c2, d.c3, c1a, c1b, c2a, c2b, c3a, c3b);
                        const double ic = fmin(fmax(floor(d.tc), -8388608.0), 8388607.0);
                        nu = d.nu; invw = d.invw; y = d.y;
                        amp = dmul(dmul(d.S, d.invw), J.out_scale);
                        icf = (float)ic; fc = (float)(d.tc - ic);
                        dx = (float)dmul(J.dnu, d.invw);
                        yf = (float)y; ampf = (float)amp;
                    }
                }
                /* union of the warp's cores */
                int ulo = has ? c1a : INT32_MAX, uhi = has ? c1b : INT32_MIN;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ulo = min(ulo, __shfl_xor_sync(0xffffffffu, ulo, o));
                    uhi = max(uhi, __shfl_xor_sync(0xffffffffu, uhi, o));
                }
                auto term = [&](int t) -> double {
                    double v = 0.0;
                    if (has && t >= c1a && t < c1b) {
                        if (t < c2a || t >= c2b) {
                            const float x = fabsf(((float)t - icf) - fc) * dx;
                            v = (double)(ampf * hum_region2<float>(x, yf));
                        } else {
                            const double x = dmul(fabs(dsub(grid_f(J.nu_start, J.dnu, T.j0 + t), nu)), invw);
                            v = amp * ((t >= c3a && t < c3b) ? hum_region3<double>(x, y)
                                                             : hum_region4_core(x, y));
                        }
                    }
                    return v;
                };
                /* two bins per step: their butterflies are independent, so the
                 * shuffles of one overlap the other's; each bin's terms are
                 * summed in the same order as one bin per step */
                for (int t = ulo; t < uhi; t += 2) {
                    const bool two = t + 1 < uhi;      /* warp-uniform */
                    double v0 = term(t);
                    double v1 = two ? term(t + 1) : 0.0;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
                        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
                    }
                    if (lane == 0) {
                        row[t] += v0;
                        if (two) row[t + 1] += v1;
                    }
                }
            }
            __syncthreads();
            if (ns == 1) {
                /* rows in warp order, added to the region-I result */
                for (int t = tid; t < T.jn; t += NT) {
                    double v = 0.0;
                    bool any = false;
#pragma unroll
                    for (int w = 0; w < CORE_WARPS; ++w) {
                        const double r = s_rows[w * CORE_W + t];
                        any |= (r != 0.0);
                        v += r;
                    }
                    if (any) J.out[T.j0 + t] += v;
                }
            } else {
                /* a slice of a split tile: rows in warp order into its partial
                 * row, a ticket, and the last slice adds the partial rows in
                 * slice order (a zero total adds nothing, as above) */
                const int rb = args.csl.rowbase[ti];
                const int W = args.tile_w;
                double* prow = args.csl.rows + (size_t)(rb + sidx) * W;
                for (int t = tid; t < T.jn; t += NT) {
                    double v = 0.0;
#pragma unroll
                    for (int w = 0; w < CORE_WARPS; ++w) v += s_rows[w * CORE_W + t];
                    prow[t] = v;
                }
                __threadfence();
                __syncthreads();
                if (tid == 0) s_last = atomicAdd(args.csl.ticket + ti, 1) == ns - 1;
                __syncthreads();
                if (s_last) {
                    __threadfence();
                    for (int t = tid; t < T.jn; t += NT) {
                        double v = 0.0;
                        for (int q = 0; q < ns; ++q) v += __ldcg(args.csl.rows + (size_t)(rb + q) * W + t);
                        if (v != 0.0) J.out[T.j0 + t] += v;
                    }
                }
            }
            __syncthreads();
        }
    }
}

/* ------------------------------------------------------------ dispatch */
template <int PK, int PREC, int B, int WARPS, bool PREP>
static cudaError_t launch_one(const KArgs& a, int ctas_per_sm, int nsm, cudaStream_t st)
{
    auto kern = tile_kernel<PK, PREC, B, WARPS, PREP>;
    const size_t smem = Smem<PK, PREC, B, WARPS, PREP>::bytes;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, WARPS * 32, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    int per = ctas_per_sm > 0 ? min(ctas_per_sm, occ) : occ;
    /* sliced: the item count is known on the device only */
    int grid = a.sl.prefix ? per * nsm : min(a.nitems, per * nsm);
    if (grid < 1) grid = 1;
    kern<<<grid, WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int B, int CONS, bool PREP, int SR>
static cudaError_t launch_ws_sr(const KArgs& a, int ctas_per_sm, int nsm, cudaStream_t st)
{
    constexpr int PROD = 2;
    auto kern = voigt_ws_kernel<B, CONS, PROD, PREP, SR>;
    const size_t smem = WsSmem<B, CONS, PROD, PREP, SR>::bytes;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, (CONS + PROD) * 32, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    const int per = ctas_per_sm > 0 ? min(ctas_per_sm, occ) : occ;
    /* sliced: the item count is known on the device only */
    const int grid = a.sl.prefix ? per * nsm : max(1, min(a.nitems, per * nsm));
    kern<<<grid, (CONS + PROD) * 32, smem, st>>>(a);
    return cudaGetLastError();
}

/* records per ring stage: 128 (4 stages) by default; 256 (2 stages) on
 * request (GEXS_LAUNCH_LONG_STAGES) for the record-split 512-bin shapes */
template <int B, int CONS, bool PREP>
static cudaError_t launch_ws_one(const KArgs& a, int ctas_per_sm, int nsm, cudaStream_t st,
                                 bool long_stages)
{
    if constexpr (B * CONS == 16) {
        if (long_stages) return launch_ws_sr<B, CONS, PREP, 256>(a, ctas_per_sm, nsm, st);
    }
    (void)long_stages;
    return launch_ws_sr<B, CONS, PREP, 128>(a, ctas_per_sm, nsm, st);
}

/* FP32 Voigt: warp-specialised kernel, `warps` = consumer warps */
template <bool PREP>
static cudaError_t launch_ws(const KArgs& a, const gexs_launch_cfg& c, int nsm, cudaStream_t st)
{
    const bool ls = (c.flags & GEXS_LAUNCH_LONG_STAGES) != 0;
    if (c.warps == 4) {
        switch (c.bins_per_lane) {
        case 2:  return launch_ws_one<2, 4, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        case 4:  return launch_ws_one<4, 4, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        case 8:  return launch_ws_one<8, 4, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        case 16: return launch_ws_one<16, 4, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        }
    } else if (c.warps == 8) {
        switch (c.bins_per_lane) {
        case 2:  return launch_ws_one<2, 8, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        case 4:  return launch_ws_one<4, 8, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        case 8:  return launch_ws_one<8, 8, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        case 16: return launch_ws_one<16, 8, PREP>(a, c.ctas_per_sm, nsm, st, ls);
        }
    }
    return cudaErrorInvalidValue;
}

template <int PK, int PREC, bool PREP>
static cudaError_t launch_cfg(const KArgs& a, const gexs_launch_cfg& c, int nsm, cudaStream_t st)
{
    if (a.sl.prefix) {
        cudaError_t e = launch_slice_plan(a, st);
        if (e != cudaSuccess) return e;
    }
    if constexpr (PK == PK_VOIGT && PREC == GEXS_FP32) {
        return launch_ws<PREP>(a, c, nsm, st);
    } else {
        if (c.bins_per_lane == 16) {
            /* FP32 only: the FP64 form holds 4 doubles per bin in registers */
            if constexpr (PREC == GEXS_FP32) {
                if (c.warps == 8) return launch_one<PK, PREC, 16, 8, PREP>(a, c.ctas_per_sm, nsm, st);
                if (c.warps == 4) return launch_one<PK, PREC, 16, 4, PREP>(a, c.ctas_per_sm, nsm, st);
            }
            return cudaErrorInvalidValue;
        }
        if (c.warps == 8) {
            if (c.bins_per_lane == 8) return launch_one<PK, PREC, 8, 8, PREP>(a, c.ctas_per_sm, nsm, st);
            if (c.bins_per_lane == 4) return launch_one<PK, PREC, 4, 8, PREP>(a, c.ctas_per_sm, nsm, st);
            if (c.bins_per_lane == 2) return launch_one<PK, PREC, 2, 8, PREP>(a, c.ctas_per_sm, nsm, st);
        } else if (c.warps == 4) {
            if (c.bins_per_lane == 8) return launch_one<PK, PREC, 8, 4, PREP>(a, c.ctas_per_sm, nsm, st);
            if (c.bins_per_lane == 4) return launch_one<PK, PREC, 4, 4, PREP>(a, c.ctas_per_sm, nsm, st);
            if (c.bins_per_lane == 2) return launch_one<PK, PREC, 2, 4, PREP>(a, c.ctas_per_sm, nsm, st);
        }
        return cudaErrorInvalidValue;
    }
}

/* the FP32 Voigt core kernel after the tile kernel, on the same stream; its
 * work counter is the int 128 bytes after the tile kernel's (the launch
 * tables reserve 256 bytes for counters) */
constexpr int CORE_COUNTER_OFFSET = 32;

template <bool PREP>
static cudaError_t launch_core(const KArgs& a, int nsm, cudaStream_t st)
{
    auto kern = a.order ? core_kernel<PREP, true> : core_kernel<PREP, false>;
    const size_t smem = CoreSmem::bytes;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, CORE_WARPS * 32, smem);
    if (e != cudaSuccess) return e;
    /* sliced: the item count is known on the device only */
    const int grid = a.csl.prefix ? max(occ, 1) * nsm : max(1, min(a.nitems, max(occ, 1) * nsm));
    KArgs c = a;
    c.counter = a.counter + CORE_COUNTER_OFFSET;
    e = zero_ints(c.counter, 1, st);
    if (e != cudaSuccess) return e;
    if (c.csl.prefix) {
        e = launch_core_slice_plan(c, st);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, CORE_WARPS * 32, smem, st>>>(c);
    return cudaGetLastError();
}

/* every launch shape of one profile class, both precisions, both
 * line-quantity sources (prep arrays or derived on load) */
template <int PK>
static cudaError_t launch_pk(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                             cudaStream_t st)
{
    const bool prep = a.prep != nullptr;
    if (prec == GEXS_FP32) {
        cudaError_t e = prep ? launch_cfg<PK, GEXS_FP32, true>(a, cfg, nsm, st)
                             : launch_cfg<PK, GEXS_FP32, false>(a, cfg, nsm, st);
        if (PK != PK_VOIGT || e != cudaSuccess) return e;
        return prep ? launch_core<true>(a, nsm, st) : launch_core<false>(a, nsm, st);
    }
    return prep ? launch_cfg<PK, GEXS_FP64, true>(a, cfg, nsm, st)
                : launch_cfg<PK, GEXS_FP64, false>(a, cfg, nsm, st);
}

/* defined one per translation unit */
cudaError_t launch_tiles_voigt(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                               cudaStream_t st);
cudaError_t launch_tiles_erf(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                             cudaStream_t st);
cudaError_t launch_tiles_gh16(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                              cudaStream_t st);
cudaError_t launch_tiles_gh32(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                              cudaStream_t st);

}  // namespace gexs
