/*
 * gexs_device.cuh — device arithmetic of the cross-section kernels.
 *
 * FP64 helpers round every operation as written (no fused multiply-add), so
 * that grid frequencies, window limits and Humlicek region limits are the
 * same doubles the reference computes: BaseProfile.cpp:17-21 builds the
 * grid as start + i*dfreq and Managers/CPU/OpenMPManager.cpp:399-408 and
 * compute/CPU/profiles.cpp:17-28 compare such values against thresholds.
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gexs_b200.h"
#include "gh_nodes.h"

namespace gexs {

/* ------------------------------------------------ exactly-rounded FP64 ops */
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

/* grid frequency f_j = nu_start + j*dnu, two roundings */
__device__ __forceinline__ double grid_f(double nu_start, double dnu, int64_t j)
{
    return dadd(nu_start, dmul((double)j, dnu));
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

/* ---------------------------------------------------- Humlicek W4 pieces
 * K(x, y) = Re w(x + iy) by Humlicek's four regions (compute/CPU/profiles.cpp
 * :11-44, constants as there).  T = y - i x.  The caller selects the region.
 * Region I has the closed form Re[T c/(1/2 + T^2)] = c y (p + x^2) /
 * ((p + x^2)^2 - 2 x^2), p = 1/2 + y^2; regions II-IV use complex Horner
 * evaluation in real arithmetic and Re(N/D) = (Nr Dr + Ni Di)/|D|^2. */
template <typename R> struct HC;
template <> struct HC<float> {
    static __device__ __forceinline__ float k(double v) { return (float)v; }
};
template <> struct HC<double> {
    static __device__ __forceinline__ double k(double v) { return v; }
};

template <typename R>
__device__ __forceinline__ R hum_region1(R x, R y)
{
    R x2 = x * x;
    R num = x2 + (R(0.5) + y * y);
    R den = num * num - R(2) * x2;
    return HC<R>::k(0.5641896) * y * num / den;
}

template <typename R>
__device__ __forceinline__ R re_div(R nr, R ni, R dr, R di)
{
    return (nr * dr + ni * di) / (dr * dr + di * di);
}
/* FP32: one approximate reciprocal (1 ulp) instead of an IEEE division */
template <>
__device__ __forceinline__ float re_div<float>(float nr, float ni, float dr, float di)
{
    return fmaf(nr, dr, ni * di) * rcp_approx(fmaf(dr, dr, di * di));
}

template <typename R>
__device__ __forceinline__ R hum_region2(R x, R y)
{
    /* T (1.410474 + .5641896 U) / (.75 + U (3 + U)), U = T^2 */
    R ur = y * y - x * x, ui = R(-2) * x * y;
    R ar = HC<R>::k(1.410474) + HC<R>::k(.5641896) * ur, ai = HC<R>::k(.5641896) * ui;
    /* N = T * a, T = (y, -x) */
    R nr = y * ar + x * ai, ni = y * ai - x * ar;
    /* D = .75 + U*(3+U) */
    R br = R(3) + ur;
    R dr = HC<R>::k(.75) + (ur * br - ui * ui);
    R di = ur * ui + ui * br;
    return re_div(nr, ni, dr, di);
}

template <typename R>
__device__ __forceinline__ void cmul_add(R& pr, R& pi, R tr, R ti, R c)
{
    /* p = c + t*p */
    R r = tr * pr - ti * pi;
    R i = tr * pi + ti * pr;
    pr = c + r; pi = i;
}

template <typename R>
__device__ __forceinline__ R hum_region3(R x, R y)
{
    R tr = y, ti = -x;
    R nr = HC<R>::k(.5642236), ni = R(0);
    cmul_add(nr, ni, tr, ti, HC<R>::k(3.778987));
    cmul_add(nr, ni, tr, ti, HC<R>::k(11.96482));
    cmul_add(nr, ni, tr, ti, HC<R>::k(20.20933));
    cmul_add(nr, ni, tr, ti, HC<R>::k(16.4955));
    R dr = R(1), di = R(0);
    cmul_add(dr, di, tr, ti, HC<R>::k(6.699398));
    cmul_add(dr, di, tr, ti, HC<R>::k(21.69274));
    cmul_add(dr, di, tr, ti, HC<R>::k(39.27121));
    cmul_add(dr, di, tr, ti, HC<R>::k(38.82363));
    cmul_add(dr, di, tr, ti, HC<R>::k(16.4955));
    return re_div(nr, ni, dr, di);
}

template <typename R> __device__ __forceinline__ R expcos(R a, R b);
template <> __device__ __forceinline__ float expcos<float>(float a, float b) { return expf(a) * cosf(b); }
template <> __device__ __forceinline__ double expcos<double>(double a, double b) { return exp(a) * cos(b); }

template <typename R>
__device__ __forceinline__ R hum_region4(R x, R y)
{
    /* exp(U) - T P(U)/Q(U); P, Q written as polynomials in V = -U */
    R ur = y * y - x * x, ui = R(-2) * x * y;
    R vr = -ur, vi = -ui;
    R pr = HC<R>::k(.56419), pi = R(0);
    cmul_add(pr, pi, vr, vi, HC<R>::k(1.320522));
    cmul_add(pr, pi, vr, vi, HC<R>::k(35.76683));
    cmul_add(pr, pi, vr, vi, HC<R>::k(219.0313));
    cmul_add(pr, pi, vr, vi, HC<R>::k(1540.787));
    cmul_add(pr, pi, vr, vi, HC<R>::k(3321.9905));
    cmul_add(pr, pi, vr, vi, HC<R>::k(36183.31));
    R qr = R(1), qi = R(0);
    cmul_add(qr, qi, vr, vi, HC<R>::k(1.841439));
    cmul_add(qr, qi, vr, vi, HC<R>::k(61.57037));
    cmul_add(qr, qi, vr, vi, HC<R>::k(364.2191));
    cmul_add(qr, qi, vr, vi, HC<R>::k(2186.181));
    cmul_add(qr, qi, vr, vi, HC<R>::k(9022.228));
    cmul_add(qr, qi, vr, vi, HC<R>::k(24322.84));
    cmul_add(qr, qi, vr, vi, HC<R>::k(32066.6));
    /* T * P, T = (y, -x) */
    R nr = y * pr + x * pi, ni = y * pi - x * pr;
    return expcos(ur, ui) - re_div(nr, ni, qr, qi);
}

/* Region IV for the FP32 form's core kernel: the rational part in FP64
 * (its real part comes out of a mostly imaginary quotient, so FP32 rounding
 * would be amplified), exp(U) cos(Im U) in FP32.  In region IV |x| < 5.5 and
 * y < 0.195|x| - 0.176, so Re U >= -30.25 (no underflow), |Im U| < 10, and
 * Re w = exp-term + a non-negative part: the FP32 error of the exp term
 * (a few 1e-7 of that term) is at most a few 1e-7 of the result. */
__device__ __forceinline__ double hum_region4_core(double x, double y)
{
    const double ur = y * y - x * x, ui = -2.0 * x * y;
    const double vr = -ur, vi = -ui;
    double pr = .56419, pi = 0.0;
    cmul_add(pr, pi, vr, vi, 1.320522);
    cmul_add(pr, pi, vr, vi, 35.76683);
    cmul_add(pr, pi, vr, vi, 219.0313);
    cmul_add(pr, pi, vr, vi, 1540.787);
    cmul_add(pr, pi, vr, vi, 3321.9905);
    cmul_add(pr, pi, vr, vi, 36183.31);
    double qr = 1.0, qi = 0.0;
    cmul_add(qr, qi, vr, vi, 1.841439);
    cmul_add(qr, qi, vr, vi, 61.57037);
    cmul_add(qr, qi, vr, vi, 364.2191);
    cmul_add(qr, qi, vr, vi, 2186.181);
    cmul_add(qr, qi, vr, vi, 9022.228);
    cmul_add(qr, qi, vr, vi, 24322.84);
    cmul_add(qr, qi, vr, vi, 32066.6);
    const double nr = y * pr + x * pi, ni = y * pi - x * pr;
    return (double)expcos<float>((float)ur, (float)ui) - re_div(nr, ni, qr, qi);
}

/* region selected by integer bin limits: 1..4 */
template <typename R>
__device__ __forceinline__ R hum_by_region(int reg, R x, R y)
{
    if (reg == 1) return hum_region1(x, y);
    if (reg == 2) return hum_region2(x, y);
    if (reg == 3) return hum_region3(x, y);
    return hum_region4(x, y);
}

/* --------------------------------------------------- Gauss-Hermite Voigt
 * sum_k w_k (A + B)/(A B), A = y2 + (x - t_k)^2, B = y2 + (x + t_k)^2,
 * ascending t_k; the caller multiplies by y/pi. */
template <int NODES> struct GH;
template <> struct GH<16> { static constexpr int NP = 8; };
template <> struct GH<32> { static constexpr int NP = 16; };

template <int NODES>
__device__ __forceinline__ double gh_t(int k)
{
    constexpr double t16[8] = {GEXS_GH16_T_LIST};
    constexpr double t32[16] = {GEXS_GH32_T_LIST};
    return NODES == 16 ? t16[k] : t32[k];
}
template <int NODES>
__device__ __forceinline__ double gh_w(int k)
{
    constexpr double w16[8] = {GEXS_GH16_W_LIST};
    constexpr double w32[16] = {GEXS_GH32_W_LIST};
    return NODES == 16 ? w16[k] : w32[k];
}

template <int NODES>
__device__ __forceinline__ float gh_sum_f32(float x, float y2)
{
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < GH<NODES>::NP; ++k) {
        float t = (float)gh_t<NODES>(k), w = (float)gh_w<NODES>(k);
        float d1 = x - t, d2 = x + t;
        float A = fmaf(d1, d1, y2), B = fmaf(d2, d2, y2);
        acc = fmaf(w * (A + B), rcp_approx(A * B), acc);
    }
    return acc;
}

/* Lines much narrower than a node spacing (y < 1/8): near a node t_k the
 * term w_k / (y^2 + (x - t_k)^2) is a spike of width y, and an x carried
 * in one float (absolute error ~1e-7 x) would put a relative error of
 * about 1e-7 x / |x - t_k| on it.  Here x is the unevaluated pair xs + xl
 * (x_pair below, error ~1e-13) and x - t_k is taken against the node split
 * the same way, so every difference keeps its relative accuracy. */
template <int NODES>
__device__ __forceinline__ float gh_sum_f32_pair(float xs, float xl, float y2)
{
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < GH<NODES>::NP; ++k) {
        const double tk = gh_t<NODES>(k);
        const float th = (float)tk, tl = (float)(tk - (double)th), w = (float)gh_w<NODES>(k);
        /* xs - th is exact when xs is within a factor 2 of th (Sterbenz) */
        const float d1 = __fadd_rn(__fsub_rn(xs, th), __fsub_rn(xl, tl));
        const float d2 = __fadd_rn(xs, th);
        const float A = fmaf(d1, d1, y2), B = fmaf(d2, d2, y2);
        acc = fmaf(w * (A + B), rcp_approx(A * B), acc);
    }
    return acc;
}

/* x = (n - fc) dx as the pair xs + xl from n (an exact integer in float),
 * dx = dxh + dxl and mf = -fc dx = mfh + mfl (each split from FP64 on the
 * host of the record): TwoProduct of n dxh and TwoSum with mfh, written
 * with _rn intrinsics so that no step is contracted into an FMA. */
__device__ __forceinline__ void x_pair(float n, float dxh, float dxl, float mfh, float mfl,
                                       float& xs, float& xl)
{
    const float p = __fmul_rn(n, dxh);
    const float e1 = __fmaf_rn(n, dxh, -p);
    const float s = __fadd_rn(p, mfh);
    const float bb = __fsub_rn(s, p);
    const float e2 = __fadd_rn(__fsub_rn(p, __fsub_rn(s, bb)), __fsub_rn(mfh, bb));
    const float lo = __fadd_rn(__fadd_rn(e1, e2), __fmaf_rn(n, dxl, mfl));
    /* |x|: the profile is even in x */
    if (s < 0.f) { xs = -s; xl = -lo; } else { xs = s; xl = lo; }
}

/* same sum as 1/A + 1/B per pair: no A*B product, safe for |x| > 1e9 */
template <int NODES>
__device__ __forceinline__ float gh_sum_f32_wide(float x, float y2)
{
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < GH<NODES>::NP; ++k) {
        float t = (float)gh_t<NODES>(k), w = (float)gh_w<NODES>(k);
        float d1 = x - t, d2 = x + t;
        float A = fmaf(d1, d1, y2), B = fmaf(d2, d2, y2);
        acc = fmaf(w, 1.f / A + 1.f / B, acc);
    }
    return acc;
}

template <int NODES>
__device__ __forceinline__ double gh_sum_f64(double x, double y2)
{
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < GH<NODES>::NP; ++k) {
        double d1 = dsub(x, gh_t<NODES>(k)), d2 = dadd(x, gh_t<NODES>(k));
        double A = dadd(y2, dmul(d1, d1)), B = dadd(y2, dmul(d2, d2));
        acc = dadd(acc, dmul(gh_w<NODES>(k), ddiv(dadd(A, B), dmul(A, B))));
    }
    return acc;
}

/* ------------------------------------------------ bin-averaged erf difference */
__device__ __forceinline__ float erf_bin_f32(float xm, float xp, int form)
{
    if (form == GEXS_ERF_LITERAL || xm < 0.f) return erff(xp) - erff(xm);
    return erfcf(xm) - erfcf(xp);
}
__device__ __forceinline__ double erf_bin_f64(double xm, double xp, int form)
{
    if (form == GEXS_ERF_LITERAL || xm < 0.0) return dsub(erf(xp), erf(xm));
    return dsub(erfc(xm), erfc(xp));
}

/* ---------------------------------------------------- interval search
 * first t in [lo, hi] with pred(t) true, pred monotone false -> true and
 * pred(hi) assumed true (hi may be one past the range).  Gallops from the
 * guess g, then bisects. */
template <typename P>
__device__ __forceinline__ int first_true(int lo, int hi, int g, const P& pred)
{
    if (lo >= hi) return hi;
    g = max(lo, min(g, hi - 1));
    int l, r;                        /* pred(l) false (or l = lo-1), pred(r) true */
    if (pred(g)) {
        r = g; int step = 1;
        for (;;) {
            int c = r - step;
            if (c < lo) { l = lo - 1; break; }
            if (!pred(c)) { l = c; break; }
            r = c; step <<= 1;
        }
    } else {
        l = g; int step = 1;
        for (;;) {
            int c = l + step;
            if (c >= hi) { r = hi; break; }
            if (pred(c)) { r = c; break; }
            l = c; step <<= 1;
        }
    }
    while (r - l > 1) {
        int m = l + ((r - l) >> 1);
        if (pred(m)) r = m; else l = m;
    }
    return r;
}

}  // namespace gexs
