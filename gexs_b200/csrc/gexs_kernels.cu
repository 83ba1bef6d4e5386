/*
 * gexs_kernels.cu — sm_100a kernels of the cross-section path.
 *
 * Work decomposition (replaces the reference's one-CTA-per-grid-point scan
 * over every line of a chunk, compute/CUDA/cross_kernal_v2.cu:403-457):
 *  - a work item is one tile of W = 32*B*WARPS consecutive bins of one job;
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
 *    over the stage's lines: no atomics, every bin sums its lines in
 *    ascending line order (deterministic, independent of other jobs);
 *  - FP32 form: per-stage FP32 partial sums merged into a Kahan-compensated
 *    (sum, compensation) pair per bin; FP64 form: plain FP64 sums.
 */
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>
#include "gexs_device.cuh"
#include "gexs_internal.h"

namespace gexs {

/* --------------------------------------------------------------- records
 * One derived record per (line, tile), written by the thread that derived
 * the line and read by every warp as 16-byte broadcast loads. */
struct __align__(16) RecF32 {   /* 48 bytes */
    float icf;             /* tile-relative centre bin floor(tc), exact      */
    float dx;              /* dnu * invw: x per bin                          */
    float mfcdx;           /* -(tc - floor(tc)) * dx                         */
    float a1;              /* Voigt: amp*0.5641896*y ; GH: amp*y/pi          */
    float p;               /* Voigt: 0.5 + y^2 ; GH: y^2                     */
    float y;               /* Voigt/GH: y ; Doppler: half bin in x units     */
    float amp;             /* Voigt/GH: S*invw*out_scale ; Doppler: S*out    */
    float fc;              /* tc - floor(tc) in [0, 1)                       */
    int   win;             /* a | b << 16 : bins [a, b) of the tile          */
    int   c1;              /* Voigt: bins not in region I (the core) ;
                              Doppler: bins whose xm <= the zero threshold   */
    int   mask;            /* per warp w: bit w touches, bit 8+w fast tier,
                              bit 16+w mid tier; bit 24: |x| may exceed 1e8
                              in this tile (overflow-free forms)             */
    int   pad;
};

struct __align__(16) RecF64 {   /* 64 bytes */
    double nu;             /* centre after the nu==0 rule                   */
    double invw;
    double y;              /* Voigt/GH: y ; Doppler: unused                 */
    double amp;            /* Voigt/GH: S*invw ; Doppler: S                 */
    int    win, c1, c2, c3;
    int    mask, pad0, pad1, pad2;
};

/* FP64 view of a line for its core (Humlicek regions II-IV), which the
 * FP32 form evaluates in a separate pass */
struct CoreF64 {
    double nu, invw, y, amp;
    int c2;                /* bins in regions III/IV                        */
    int c3;                /* bins satisfying the region-III test           */
};

template <int PREC> struct RecOf;
template <> struct RecOf<GEXS_FP32> { typedef RecF32 T; };
template <> struct RecOf<GEXS_FP64> { typedef RecF64 T; };

__device__ __forceinline__ int pack2(int a, int b) { return a | (b << 16); }
__device__ __forceinline__ int lo16(int v) { return v & 0xffff; }
__device__ __forceinline__ int hi16(int v) { return (int)((unsigned)v >> 16); }

/* profile classes of the kernel template */
enum { PK_VOIGT = 0, PK_ERF = 1, PK_GH16 = 2, PK_GH32 = 3 };

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
    double w = cut / J.dnu;
    int gl = (int)fmin(fmax(ceil(tc - w), 0.0), (double)anchor);
    int gr = (int)fmin(fmax(floor(tc + w) + 1.0, (double)anchor), (double)T.jn);
    *pa = first_true(0, anchor, gl, [&](int t) { return in(t); });
    *pb = first_true(anchor, T.jn, gr, [&](int t) { return !in(t); });
}

/* bins of [wa, wb) (a sub-range of the tile) where dist-predicate `in`
 * holds; `in` must be true on one contiguous interval around the line
 * centre.  d_thr is an estimate of the distance limit for the guesses. */
template <typename P>
__device__ __forceinline__ int centered(const Tile& T, int wa, int wb, double nu, double tc,
                                        double d_thr, const P& in)
{
    if (wa >= wb || !(d_thr >= 0.0)) return 0;
    double fa = grid_f(T.J->nu_start, T.J->dnu, T.j0 + wa);
    double fb = grid_f(T.J->nu_start, T.J->dnu, T.j0 + wb - 1);
    double dmin = nu < fa ? fa - nu : (nu > fb ? nu - fb : 0.0);
    if (dmin > d_thr * (1.0 + 1e-9) + 1e-300) return 0;
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

/* tile-dependent part: centre in bins, window and Humlicek region limits */
template <int PK>
__device__ __noinline__ Derived<PK> derive_line(const Tile& T, const LineQ& q, double zthr)
{
    const gexs_job& J = *T.J;
    Derived<PK> d;
    const double nu = q.nu;
    d.nu = nu; d.S = q.S; d.invw = q.invw; d.y = q.y;
    d.tc = ddiv(dsub(nu, T.f0), J.dnu);
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
        d.c1 = centered(T, a, b, nu, d.tc, (15.0 - y) / invw,
                        [&](int tt) { return dadd(xof(tt), y) < 15.0; });
        if (lo16(d.c1) < hi16(d.c1)) {
            d.c2 = centered(T, lo16(d.c1), hi16(d.c1), nu, d.tc, (5.5 - y) / invw,
                            [&](int tt) { return dadd(xof(tt), y) < 5.5; });
            if (lo16(d.c2) < hi16(d.c2))
                d.c3 = centered(T, lo16(d.c2), hi16(d.c2), nu, d.tc, ((y + 0.176) / 0.195) / invw,
                                [&](int tt) { return y >= dsub(dmul(0.195, xof(tt)), 0.176); });
        }
    } else if constexpr (PK == PK_ERF) {
        /* bins whose lower erf argument is <= zthr; beyond it both erfc
         * terms underflow to exactly zero */
        const double h = 0.5 * dnu;
        d.c1 = centered(T, a, b, nu, d.tc, zthr / invw + h,
                        [&](int tt) {
                            double dist = fabs(dsub(grid_f(nu_s, dnu, j0 + tt), nu));
                            return dmul(invw, dsub(dist, h)) <= zthr;
                        });
    }
    return d;
}

/* ------------------------------------------------------------ prep kernel
 * Per job, the FP64 per-line quantities once: S at base[i], invw at
 * base[N + i], y at base[2N + i] (N = line count).  The tile kernel then
 * reads 32 bytes per line instead of recomputing two exponentials, a power
 * and two divisions for every tile the line reaches. */
__global__ void prep_kernel(const gexs_job* __restrict__ jobs, double* const* __restrict__ prep)
{
    const gexs_job& J = jobs[blockIdx.y];
    double* base = prep[blockIdx.y];
    const int64_t N = J.lines.count;
    const bool press = J.profile == GEXS_VOIGT || J.profile == GEXS_VOIGT_QUAD;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * blockDim.x) {
        RawLine L;
        L.nu = J.lines.nu[i]; L.elow = J.lines.elow[i]; L.aif = J.lines.aif[i];
        L.g = J.lines.gns[i];
        LineQ q;
        if (press) {
            L.gam = J.lines.gamma[i]; L.nexp = J.lines.n[i];
            q = line_quantities<true>(J, L);
        } else {
            L.gam = 0.0; L.nexp = 0.0;
            q = line_quantities<false>(J, L);
        }
        base[i] = q.S;
        base[N + i] = q.invw;
        base[2 * N + i] = q.y;
    }
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
};

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
        const bool full = a <= r0 && b >= r1;
        const bool coredisj = (PK != PK_VOIGT) || c1a >= c1b || c1b <= r0 || c1a >= r1;
        /* the single-FMA x of the fast tier keeps ~1e-7 relative accuracy
         * only when the centre is at least a warp span away */
        const bool far = ic < r0 - 32 * B || ic > r1 + 32 * B;
        if (full && coredisj) m |= 1 << (far ? 8 + w : 16 + w);
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
    if constexpr (PK == PK_VOIGT) {
        q.a1 = (float)(ampd * 0.5641896 * d.y);
        q.p = (float)(0.5 + d.y * d.y);
        q.y = (float)d.y;
    } else if constexpr (PK == PK_ERF) {
        q.a1 = 0.f; q.p = 0.f;
        q.y = (float)(0.5 * dx);
    } else {
        q.a1 = (float)(ampd * d.y * GEXS_INV_PI);
        q.p = (float)(d.y * d.y);
        q.y = (float)d.y;
    }
    q.fc = fc;
    q.win = d.win; q.c1 = d.c1;
    /* largest |x| the line reaches in this tile */
    double dfar = fmax(fabs(d.nu - T.f0), fabs(d.nu - T.fl));
    const int wide = (dfar * d.invw > 1e8) ? 1 : 0;
    q.mask = (d.win == 0) ? 0 : warp_mask<PK, B, WARPS>(d, wide);
    q.pad = 0;
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

/* FP64 Humlicek for a core bin of the FP32 form, kept out of line so the
 * FP32 loop does not carry its registers */
__device__ __noinline__ float core_term_f64(int reg, double f, const CoreF64& cd)
{
    const double xd = dmul(fabs(dsub(f, cd.nu)), cd.invw);
    return (float)(cd.amp * hum_by_region<double>(reg, xd, cd.y));
}

/* ------------------------------------------------- per-warp line loops
 * FP32 form.  Lane l of warp w owns bins t_k = wb + l + 32k (k < B).
 * fast tier: whole warp in the window, in region I, centre >= one warp
 *   span away: x_k = fma(32k, dx, fma(l, dx, q)) and the region-I closed
 *   form, 7 issue slots + 1 MUFU per bin;
 * mid tier: as fast but the centre is near: x = ((l+32k + wb-ic) - fc)*dx
 *   exactly, so bins next to the centre keep full relative accuracy;
 * general: per-bin window and region tests; Humlicek regions II-IV (the
 *   line core, which carries most of its area) in FP64. */
template <int PK, int B>
__device__ __forceinline__ void lines_f32(const RecF32* __restrict__ rec,
                                          const CoreF64* __restrict__ core, int nrec, int warp,
                                          int lane, float (&part)[B], double nu_start, double dnu,
                                          int64_t j0)
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
        if constexpr (PK == PK_VOIGT) {
            if (mask & (bit << 8)) {
                const float x0 = fmaf(lanef, q0.y, fmaf(ncf, q0.y, q0.z));
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const float x = fmaf((float)(32 * k), q0.y, x0);
                    const float x2 = x * x;
                    const float num = x2 + q1.x;
                    const float den = fmaf(x2, -2.f, num * num);
                    part[k] = fmaf(num * rcp_approx(den), q0.w, part[k]);
                }
                continue;
            }
            const float t0 = lanef + ncf;   /* exact: small integers */
            if (mask & (bit << 16)) {
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const float x = ((t0 + (float)(32 * k)) - q1.w) * q0.y;
                    const float x2 = x * x;
                    const float num = x2 + q1.x;
                    const float den = fmaf(x2, -2.f, num * num);
                    part[k] = fmaf(num * rcp_approx(den), q0.w, part[k]);
                }
                continue;
            }
            /* general tier: window edges and region-I bins of warps that
             * hold part of the core; the core bins themselves are left to
             * core_pass_f32.  Every bin is evaluated and the accumulation
             * is predicated, so the warp does not diverge. */
            const int a = lo16(qi.x), b = hi16(qi.x);
            const int c1a = lo16(qi.y), c1b = hi16(qi.y);
            if (!((mask >> 24) & 1)) {
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = wb + lane + 32 * k;
                    const float x = ((t0 + (float)(32 * k)) - q1.w) * q0.y;
                    const float x2 = x * x;
                    const float num = x2 + q1.x;
                    const float den = fmaf(x2, -2.f, num * num);
                    const float v = num * rcp_approx(den) * q0.w;
                    const bool in = (unsigned)(t - a) < (unsigned)(b - a) &&
                                    !((unsigned)(t - c1a) < (unsigned)(c1b - c1a));
                    part[k] += in ? v : 0.f;
                }
            } else {
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = wb + lane + 32 * k;
                    if (t < a || t >= b || (t >= c1a && t < c1b)) continue;
                    const float x = fabsf(((t0 + (float)(32 * k)) - q1.w) * q0.y);
                    const float x2 = x * x;
                    const float num = x2 + q1.x;
                    /* num/den = 1/(num - 2 x^2/num) without num^2 */
                    part[k] += (x < 1e18f) ? q0.w / (num - 2.f * (x2 / num)) : 0.f;
                }
            }
        } else if constexpr (PK == PK_ERF) {
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
                part[k] = fmaf(q1.z, erf_bin_f32(xd - q1.y, xd + q1.y, GEXS_ERF_STABLE), part[k]);
            }
        } else {
            constexpr int NODES = (PK == PK_GH16) ? 16 : 32;
            if (mask & (bit << 8)) {
                const float x0 = fmaf(lanef, q0.y, fmaf(ncf, q0.y, q0.z));
#pragma unroll
                for (int k = 0; k < B; ++k)
                    part[k] = fmaf(q0.w, gh_sum_f32<NODES>(fabsf(fmaf((float)(32 * k), q0.y, x0)), q1.x),
                                   part[k]);
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
                part[k] = fmaf(q0.w, g, part[k]);
            }
        }
    }
}

/* Core pass of the FP32 Voigt form: the bins of each line's core (not in
 * Humlicek region I) in this phase.  Lines are dealt to warps round-robin
 * and a warp's lanes take consecutive core bins, so the FP64 work is spread
 * evenly over the CTA instead of landing on the warp that owns the bins.
 * Region II is evaluated in FP32, regions III/IV (where extracting the real
 * part of a mostly imaginary w(z) amplifies FP32 rounding ~100x) in FP64.
 * Each warp adds into its own accumulator row: every bin receives its core
 * terms in a fixed order. */
template <int WARPS>
__device__ __forceinline__ void core_pass_f32(const RecF32* __restrict__ rec,
                                              const CoreF64* __restrict__ core, int nrec,
                                              int warp, int lane, float* __restrict__ wacc,
                                              double nu_start, double dnu, int64_t j0)
{
    for (int i = warp; i < nrec; i += WARPS) {
        const int c1 = rec[i].c1;
        const int c1a = lo16(c1), c1b = hi16(c1);
        if (c1a >= c1b) continue;
        /* the core as contiguous single-region ranges, in a fixed order:
         * II [c1a, c2a) | IV [c2a, c3a) | III [c3a, c3b) | IV [c3b, c2b) |
         * II [c2b, c1b), c3 within c2 within c1 (empty ranges skipped) */
        const int c2 = core[i].c2, c3 = core[i].c3;
        int c2a = lo16(c2), c2b = hi16(c2);
        if (c2a >= c2b) c2a = c2b = c1b;
        int c3a = lo16(c3), c3b = hi16(c3);
        if (c3a >= c3b) c3a = c3b = c2b;
        const int lo[5] = {c1a, c2a, c3a, c3b, c2b};
        const int hi[5] = {c2a, c3a, c3b, c2b, c1b};
        const int rg[5] = {2, 4, 3, 4, 2};
        const float icf = rec[i].icf, fc = rec[i].fc, dx = rec[i].dx, y = rec[i].y;
        const float amp = rec[i].amp;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            if (rg[r] == 2) {
                for (int t = lo[r] + lane; t < hi[r]; t += 32) {
                    const float x = fabsf(((float)t - icf) - fc) * dx;
                    wacc[t] += amp * hum_region2<float>(x, y);
                }
            } else {
                for (int t = lo[r] + lane; t < hi[r]; t += 32)
                    wacc[t] += core_term_f64(rg[r], grid_f(nu_start, dnu, j0 + t), core[i]);
            }
        }
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
    static constexpr bool CORE = (PREC == GEXS_FP32 && PK == PK_VOIGT);
    static constexpr size_t raw_d = (size_t)2 * NT * sizeof(double);   /* one f64 array, 2 bufs */
    /* staged per line: PREP nu S invw y ; on-load nu elow aif [gamma n] gns */
    static constexpr int NF64 = PREP ? 4 : (PRESS ? 5 : 3);
    static constexpr size_t off_gn = NF64 * raw_d;
    static constexpr size_t off_rec = (off_gn + (PREP ? 0 : (size_t)2 * NT * sizeof(int)) + 15) & ~size_t(15);
    static constexpr size_t rec_sz = (PREC == GEXS_FP32) ? sizeof(RecF32) : sizeof(RecF64);
    static constexpr size_t off_core = off_rec + (size_t)R * rec_sz;
    static constexpr size_t off_wacc = (off_core + (CORE ? (size_t)R * sizeof(CoreF64) : 0) + 15) & ~size_t(15);
    static constexpr size_t bytes = off_wacc + (CORE ? (size_t)WARPS * W * sizeof(float) : 0);
};

/* ---------------------------------------------------------------- kernel */
/* resident CTAs per SM the register budget is sized for */
template <int B, int WARPS>
constexpr int min_ctas() { return WARPS == 8 ? (B == 8 ? 2 : 3) : (B == 8 ? 4 : 6); }

template <int PK, int PREC, int B, int WARPS, bool PREP>
__global__ void __launch_bounds__(WARPS * 32, min_ctas<B, WARPS>())
tile_kernel(const KArgs args)
{
    typedef Smem<PK, PREC, B, WARPS, PREP> L;
    constexpr int NT = L::NT;
    constexpr int R = L::R;
    constexpr int W = 32 * B * WARPS;
    typedef typename RecOf<PREC>::T Rec;

    extern __shared__ __align__(16) unsigned char smem[];
    /* staging arrays f[k][2*NT] (k < NF64) and gns[2*NT] */
    double* s_f = reinterpret_cast<double*>(smem);
    int*    s_gn = reinterpret_cast<int*>(smem + L::off_gn);
    Rec*    s_rec = reinterpret_cast<Rec*>(smem + L::off_rec);
    CoreF64* s_core = reinterpret_cast<CoreF64*>(smem + L::off_core);
    float*  s_wacc = reinterpret_cast<float*>(smem + L::off_wacc);
    __shared__ int s_item;
    __shared__ long long s_lohi[2];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double zthr = (PREC == GEXS_FP32) ? 10.5 : 27.5;

    for (;;) {
        if (tid == 0) s_item = atomicAdd(args.counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= args.nitems) break;

        /* job of this item: last prefix entry <= item */
        int jl = 0, jh = args.njobs;
        while (jh - jl > 1) { int m = (jl + jh) >> 1; if (__ldg(args.prefix + m) <= item) jl = m; else jh = m; }
        const gexs_job* Jp = args.jobs + jl;
        const gexs_job& J = *Jp;
        Tile T;
        T.J = Jp;
        T.j0 = J.start_idx + (int64_t)(item - __ldg(args.prefix + jl)) * W;
        T.jn = (int)min((int64_t)W, J.start_idx + J.n_points - T.j0);
        T.f0 = grid_f(J.nu_start, J.dnu, T.j0);
        T.fl = grid_f(J.nu_start, J.dnu, T.j0 + T.jn - 1);

        const int64_t nl = J.lines.count;
        const double margin = 2.0 * J.dnu + 1e-9 * (fabs(T.fl) + J.cutoff);
        if (warp == 0) {
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
        if constexpr (L::CORE) {
            for (int z = tid; z < WARPS * W; z += NT) s_wacc[z] = 0.f;
            __syncthreads();
        }

        float  ks[B], kc[B], part[B];
        double acc[B], fbin[B];
#pragma unroll
        for (int k = 0; k < B; ++k) {
            ks[k] = kc[k] = part[k] = 0.f; acc[k] = 0.0;
            if (PREC == GEXS_FP64) fbin[k] = grid_f(J.nu_start, J.dnu, T.j0 + warp * 32 * B + lane + 32 * k);
        }

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
                    if constexpr (L::CORE) {
                        CoreF64 cd;
                        cd.nu = d.nu; cd.invw = d.invw; cd.y = d.y;
                        cd.amp = dmul(dmul(d.S, d.invw), J.out_scale);
                        cd.c2 = d.c2; cd.c3 = d.c3;
                        s_core[r] = cd;
                    }
                }
                issue(u + 2);
            }
            __syncthreads();

            if constexpr (PREC == GEXS_FP32) {
                /* Kahan merge of FP32 partial sums every 128 lines */
                for (int c0 = 0; c0 < nrec; c0 += 128) {
                    const int cn = min(128, nrec - c0);
                    lines_f32<PK, B>(reinterpret_cast<const RecF32*>(s_rec) + c0, s_core + c0, cn,
                                     warp, lane, part, J.nu_start, J.dnu, T.j0);
#pragma unroll
                    for (int k = 0; k < B; ++k) { kahan_add(ks[k], kc[k], part[k]); part[k] = 0.f; }
                }
                if constexpr (L::CORE)
                    core_pass_f32<WARPS>(reinterpret_cast<const RecF32*>(s_rec), s_core, nrec, warp,
                                         lane, s_wacc + warp * W, J.nu_start, J.dnu, T.j0);
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
#pragma unroll
        for (int k = 0; k < B; ++k) {
            const int t = warp * 32 * B + lane + 32 * k;
            if (t < T.jn) {
                double v = (PREC == GEXS_FP32) ? ((double)ks[k] - (double)kc[k]) : acc[k];
                if constexpr (L::CORE) {
                    /* core terms of every warp row, in warp order */
#pragma unroll
                    for (int w2 = 0; w2 < WARPS; ++w2) v += (double)s_wacc[w2 * W + t];
                }
                int64_t j = T.j0 + t;
                out[j] = acc_mode ? out[j] + v : v;
            }
        }
        __syncthreads();
    }
}

/* ------------------------------------------------------ eval counting */
__global__ void count_kernel(const gexs_job* __restrict__ jobs, unsigned long long* counts)
{
    const gexs_job& J = jobs[blockIdx.y];
    unsigned long long local = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < J.lines.count;
         i += (int64_t)gridDim.x * blockDim.x) {
        double nu = J.lines.nu[i];
        if (nu == 0.0) nu = 1e-6;
        int64_t s0 = J.start_idx, s1 = J.start_idx + J.n_points;
        int64_t jl, jh;
        if (J.window_rule == GEXS_WINDOW_ROUNDED) {
            double ib = round(ddiv(dsub(dsub(nu, J.cutoff), J.nu_start), J.dnu));
            double ie = round(ddiv(dsub(dadd(nu, J.cutoff), J.nu_start), J.dnu));
            ib = fmax(ib, (double)s0); ie = fmin(ie, (double)s1);
            jl = (int64_t)ib; jh = (int64_t)ie; if (jh < jl) jh = jl;
        } else {
            auto in = [&](int64_t j) { return fabs(dsub(grid_f(J.nu_start, J.dnu, j), nu)) <= J.cutoff; };
            double c = ddiv(dsub(nu, J.nu_start), J.dnu), w = ddiv(J.cutoff, J.dnu);
            double le = floor(c - w) - 2.0, he = ceil(c + w) + 2.0;
            jl = (int64_t)fmax((double)s0, fmin(le, (double)s1));
            jh = (int64_t)fmax((double)s0, fmin(he, (double)s1));
            int guard = 0;
            while (jl > s0 && in(jl - 1) && guard++ < 64) --jl;
            while (jl < jh && !in(jl) && guard++ < 128) ++jl;
            while (jh < s1 && in(jh) && guard++ < 192) ++jh;
            while (jh > jl && !in(jh - 1) && guard++ < 256) --jh;
        }
        local += (unsigned long long)(jh - jl);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(counts + blockIdx.y, local);
}

/* ------------------------------------------------ partition function Q(T) */
__global__ void partition_partial(const double* __restrict__ e, const int32_t* __restrict__ g,
                                  int64_t n, const double* __restrict__ betas, double* partial)
{
    /* block (x = chunk, y = temperature); fixed-order tree reduction */
    __shared__ double red[256];
    const double beta = betas[blockIdx.y];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += (double)g[i] * exp(-beta * e[i]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = red[0];
}

__global__ void partition_final(const double* partial, int nchunk, int nt, double* q)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    double s = 0.0;
    for (int c = 0; c < nchunk; ++c) s += partial[t * nchunk + c];
    q[t] = s;
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
    int grid = min(a.nitems, per * nsm);
    if (grid < 1) grid = 1;
    kern<<<grid, WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int PK, int PREC, bool PREP>
static cudaError_t launch_cfg(const KArgs& a, const gexs_launch_cfg& c, int nsm, cudaStream_t st)
{
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

template <bool PREP>
static cudaError_t launch_prec(int pk, int prec, const KArgs& a, const gexs_launch_cfg& cfg,
                               int nsm, cudaStream_t st)
{
    if (prec == GEXS_FP32) {
        switch (pk) {
        case PK_VOIGT: return launch_cfg<PK_VOIGT, GEXS_FP32, PREP>(a, cfg, nsm, st);
        case PK_ERF:   return launch_cfg<PK_ERF, GEXS_FP32, PREP>(a, cfg, nsm, st);
        case PK_GH16:  return launch_cfg<PK_GH16, GEXS_FP32, PREP>(a, cfg, nsm, st);
        case PK_GH32:  return launch_cfg<PK_GH32, GEXS_FP32, PREP>(a, cfg, nsm, st);
        }
    } else {
        switch (pk) {
        case PK_VOIGT: return launch_cfg<PK_VOIGT, GEXS_FP64, PREP>(a, cfg, nsm, st);
        case PK_ERF:   return launch_cfg<PK_ERF, GEXS_FP64, PREP>(a, cfg, nsm, st);
        case PK_GH16:  return launch_cfg<PK_GH16, GEXS_FP64, PREP>(a, cfg, nsm, st);
        case PK_GH32:  return launch_cfg<PK_GH32, GEXS_FP64, PREP>(a, cfg, nsm, st);
        }
    }
    return cudaErrorInvalidValue;
}

int profile_class(const gexs_job& j)
{
    if (j.profile == GEXS_VOIGT) return PK_VOIGT;
    if (j.profile == GEXS_DOPPLER || j.profile == GEXS_GAUSSIAN) return PK_ERF;
    if (j.profile == GEXS_VOIGT_QUAD) return j.quad_nodes == 16 ? PK_GH16 : PK_GH32;
    return -1;
}

cudaError_t launch_tiles(int pk, int prec, const gexs_job* d_jobs, const int* d_prefix,
                         int njobs, int nitems, int* d_counter, int* d_err,
                         double* const* d_prep, const gexs_launch_cfg& cfg, int nsm,
                         cudaStream_t st)
{
    KArgs a;
    a.jobs = d_jobs; a.prefix = d_prefix; a.njobs = njobs; a.nitems = nitems;
    a.counter = d_counter; a.err = d_err; a.prep = d_prep;
    return d_prep ? launch_prec<true>(pk, prec, a, cfg, nsm, st)
                  : launch_prec<false>(pk, prec, a, cfg, nsm, st);
}

cudaError_t launch_prep(const gexs_job* d_jobs, double* const* d_prep, int njobs,
                        int64_t max_lines, int nsm, cudaStream_t st)
{
    if (max_lines <= 0) return cudaSuccess;
    int bx = (int)std::min<int64_t>((max_lines + 255) / 256, (int64_t)nsm * 8);
    dim3 grid(bx, njobs);
    prep_kernel<<<grid, 256, 0, st>>>(d_jobs, d_prep);
    return cudaGetLastError();
}

int tile_bins(const gexs_launch_cfg& c) { return 32 * c.bins_per_lane * c.warps; }

cudaError_t launch_count(const gexs_job* d_jobs, int njobs, unsigned long long* d_counts,
                         int nsm, cudaStream_t st)
{
    dim3 grid(nsm * 4, njobs);
    count_kernel<<<grid, 256, 0, st>>>(d_jobs, d_counts);
    return cudaGetLastError();
}

cudaError_t launch_partition(const double* d_e, const int32_t* d_g, int64_t n,
                             const double* d_betas, int nt, double* d_partial, int nchunk,
                             double* d_q, cudaStream_t st)
{
    dim3 grid(nchunk, nt);
    partition_partial<<<grid, 256, 0, st>>>(d_e, d_g, n, d_betas, d_partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    partition_final<<<(nt + 127) / 128, 128, 0, st>>>(d_partial, nchunk, nt, d_q);
    return cudaGetLastError();
}

}  // namespace gexs
