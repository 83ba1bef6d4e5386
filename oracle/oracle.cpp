/*
 * oracle.cpp — FP64 CPU restatement of the GEXS cross-section hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only
 * as the checker.  The product path (gexs_b200/) never links or calls it.
 *
 * Parity is pinned by tests/test_oracle_pin.py against the reference's own
 * CPU code compiled from its sources (oracle/Makefile -> oracle/_ref/) and
 * against the committed fixtures in tests/golden/ produced by that build.
 *
 * Every function follows a reference file (paths relative to the GEXS tree):
 *   orc_humlicek        compute/CPU/profiles.cpp:11-44
 *   orc_partition       Readers/Exomol/exomol_functions.cpp:50-73
 *   line intensity S    Managers/CPU/OpenMPManager.cpp:394-396,
 *                       compute/CUDA/cross_kernal_v2.cu:111-134
 *   gammaL              Managers/CPU/OpenMPManager.cpp:398,
 *                       compute/CUDA/cross_kernal_v2.cu:136-146
 *   windows             Managers/CPU/OpenMPManager.cpp:399-400 (rounded),
 *                       compute/CUDA/cross_kernal_v2.cu:434-438 (inclusive)
 *   Voigt sum           Managers/CPU/OpenMPManager.cpp:376-426
 *   Doppler sum         Managers/CPU/OpenMPManager.cpp:280-323,
 *                       compute/CUDA/cross_kernal_v2.cu:330-402
 *   Gaussian            compute/CUDA/cross_kernal.cu:647-716
 *   Gauss-Hermite       compute/CUDA/cross_kernal.cu:189-217 (node-pair
 *                       idea; nodes/weights recomputed, the reference's are
 *                       shifted one slot)
 *
 * Build with -ffp-contract=off: grid frequencies and every product must be
 * rounded exactly as written, because the window and region rules compare
 * FP64 values against thresholds.
 */
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <thread>
#include <atomic>

#include "../include/gexs_b200.h"
#include "../gexs_b200/csrc/gh_nodes.h"

typedef std::complex<double> dcomp;

extern "C" {

/* Humlicek W4 real part, the four regions of compute/CPU/profiles.cpp:11-44
 * evaluated with std::complex<double> exactly as the reference does. */
double orc_humlicek(double x, double y)
{
    dcomp T(y, -x);
    double S = std::fabs(x) + y;
    if (S >= 15) {
        dcomp r = T * 0.5641896 / (0.5 + T * T);
        return r.real();
    }
    if (S >= 5.5) {
        dcomp U = T * T;
        dcomp r = T * (1.410474 + U * .5641896) / (.75 + U * (3. + U));
        return r.real();
    }
    if (y >= 0.195 * std::fabs(x) - 0.176) {
        dcomp r = (16.4955 + T * (20.20933 + T * (11.96482
                  + T * (3.778987 + T * .5642236)))) / (16.4955 + T * (38.82363
                  + T * (39.27121 + T * (21.69274 + T * (6.699398 + T)))));
        return r.real();
    }
    dcomp U = T * T;
    dcomp r = std::exp(U) - T * (36183.31 - U * (3321.9905 - U * (1540.787 - U * (219.0313 - U *
              (35.76683 - U * (1.320522 - U * .56419)))))) / (32066.6 - U * (24322.84 - U *
              (9022.228 - U * (2186.181 - U * (364.2191 - U * (61.57037 - U * (1.841439 - U)))))));
    return r.real();
}

/* Region (1..4) that orc_humlicek uses for (x, y). */
int orc_humlicek_region(double x, double y)
{
    double S = std::fabs(x) + y;
    if (S >= 15) return 1;
    if (S >= 5.5) return 2;
    if (y >= 0.195 * std::fabs(x) - 0.176) return 3;
    return 4;
}

/* Gauss-Hermite Voigt K_N(x,y) = (y/pi) sum_k w_k / (y^2 + (x - t_k)^2),
 * summed over symmetric node pairs (+t_k, -t_k) in ascending t_k order:
 * w_k*(1/A + 1/B) with A = y^2+(x-t)^2, B = y^2+(x+t)^2, as (A+B)/(A*B). */
double orc_voigt_gh(double x, double y, int nodes)
{
    const double* t; const double* w; int npair;
    if (nodes == 16) { t = GEXS_GH16_T; w = GEXS_GH16_W; npair = 8; }
    else if (nodes == 32) { t = GEXS_GH32_T; w = GEXS_GH32_W; npair = 16; }
    else return NAN;
    double y2 = y * y, acc = 0.0;
    for (int k = 0; k < npair; ++k) {
        double d1 = x - t[k], d2 = x + t[k];
        double A = y2 + d1 * d1, B = y2 + d2 * d2;
        acc += w[k] * ((A + B) / (A * B));
    }
    return acc * (y * GEXS_INV_PI);
}

/* Q(T) = sum g exp(-beta E), sequential, constants of
 * Readers/Exomol/exomol_functions.cpp:54-60. */
double orc_partition(const double* energy, const int32_t* g, int64_t n, double temp)
{
    const double planck = 6.6260693e-27, vellgt = 2.99792458e10, boltz = 1.380658e-16;
    double beta = planck * vellgt / (boltz * temp);
    double q = 0.0;
    for (int64_t i = 0; i < n; ++i) q += g[i] * std::exp(-beta * energy[i]);
    return q;
}

/* Bin-averaged erf difference for one (line, bin) with xs = |f-nu0|. */
static inline double erf_bin(double dist, double half, double invw, int form)
{
    double xp = invw * (dist + half);
    double xm = invw * (dist - half);
    if (form == GEXS_ERF_LITERAL || xm < 0.0) return std::erf(xp) - std::erf(xm);
    return std::erfc(xm) - std::erfc(xp);
}

static inline double grid_f(const gexs_job* J, int64_t j)
{
    double p = (double)j * J->dnu;   /* -ffp-contract=off: two roundings */
    return J->nu_start + p;
}

struct LineDerived { double nu, S, invw, y; };

static inline LineDerived derive(const gexs_job* J, int64_t i)
{
    LineDerived d;
    double nu = J->lines.nu[i];
    if (nu == 0.0) nu = 1e-6;
    double t = J->s_scale * J->lines.aif[i];
    t = t * (double)J->lines.gns[i];
    t = t * J->s_scale2;
    t = t * std::exp(-J->beta * J->lines.elow[i]);
    t = t * (1.0 - std::exp(-J->beta * nu));
    double den = nu * nu;
    den = den * J->partition;
    d.nu = nu;
    d.S = t / den;
    if (J->profile == GEXS_GAUSSIAN) d.invw = J->inv_width;
    else d.invw = 1.0 / (nu * J->dop_coef);
    if (J->profile == GEXS_VOIGT || J->profile == GEXS_VOIGT_QUAD) {
        double gl = J->lines.gamma[i] * std::pow(J->t_ratio, J->lines.n[i]);
        gl = gl * J->gamma_scale;
        d.y = gl * d.invw;
    } else {
        d.y = 0.0;
    }
    return d;
}

/* Window of line (centre nu, after the nu==0 rule) as [jl, jh) within the
 * job's sub-range [start_idx, start_idx+n_points). */
static inline void window(const gexs_job* J, double nu, int64_t* jl, int64_t* jh)
{
    int64_t s0 = J->start_idx, s1 = J->start_idx + J->n_points;
    if (J->window_rule == GEXS_WINDOW_ROUNDED) {
        double a = nu - J->cutoff; a = a - J->nu_start;
        double b = nu + J->cutoff; b = b - J->nu_start;
        double ib = std::round(a / J->dnu), ie = std::round(b / J->dnu);
        ib = std::max(ib, (double)s0);
        ie = std::min(ie, (double)s1);
        *jl = (int64_t)ib; *jh = (int64_t)ie;
        if (*jh < *jl) *jh = *jl;
        return;
    }
    /* inclusive: the contiguous set {j : |f_j - nu| <= cut} */
    double c = (nu - J->nu_start) / J->dnu;
    double w = J->cutoff / J->dnu;
    double lo_est = std::floor(c - w) - 2, hi_est = std::ceil(c + w) + 2;
    int64_t lo = (int64_t)std::max((double)s0, std::min(lo_est, (double)s1));
    int64_t hi = (int64_t)std::max((double)s0, std::min(hi_est, (double)s1));
    auto in = [&](int64_t j) { return std::fabs(grid_f(J, j) - nu) <= J->cutoff; };
    while (lo > s0 && in(lo - 1)) --lo;
    while (lo < hi && !in(lo)) ++lo;
    while (hi < s1 && in(hi)) ++hi;
    while (hi > lo && !in(hi - 1)) --hi;
    *jl = lo; *jh = hi;
}

static inline double line_term(const gexs_job* J, const LineDerived& d, double f)
{
    double dist = std::fabs(f - d.nu);
    switch (J->profile) {
    case GEXS_VOIGT: {
        double x = dist * d.invw;
        double r = d.S * orc_humlicek(x, d.y);
        r = r * d.invw;
        return r * J->out_scale;
    }
    case GEXS_VOIGT_QUAD: {
        double x = dist * d.invw;
        double r = d.S * orc_voigt_gh(x, d.y, J->quad_nodes);
        r = r * d.invw;
        return r * J->out_scale;
    }
    default: {
        double de = erf_bin(dist, 0.5 * J->dnu, d.invw, J->erf_form);
        double r = d.S * de;
        return r * J->out_scale;
    }
    }
}

/* Cross-section of one job on the host.  `lines` pointers are host arrays;
 * out has grid_points entries.  Each bin sums its lines in ascending line
 * order, then is added to out when accumulate is set.  Work is split into
 * contiguous bin blocks over nthreads threads (<=0: all cores); the result
 * does not depend on the thread count. */
int orc_cross_section(const gexs_job* J, double* out, int nthreads)
{
    if (!J || !out || J->n_points < 0 || J->start_idx < 0 ||
        J->start_idx + J->n_points > J->grid_points) return GEXS_ERR_INVALID;
    int64_t n = J->n_points, s0 = J->start_idx;
    if (n == 0) return GEXS_OK;
    std::vector<double> local((size_t)n, 0.0);
    int64_t N = J->lines.count;
    std::vector<LineDerived> der((size_t)N);
    std::vector<int64_t> jl((size_t)N), jh((size_t)N);
    for (int64_t i = 0; i < N; ++i) {
        der[i] = derive(J, i);
        window(J, der[i].nu, &jl[i], &jh[i]);
    }
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    int64_t nblk = std::min<int64_t>(n, (int64_t)nthreads * 8);
    std::vector<std::thread> th;
    std::atomic<int64_t> next(0);
    auto work = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(1);
            if (b >= nblk) break;
            int64_t b0 = s0 + n * b / nblk, b1 = s0 + n * (b + 1) / nblk;
            for (int64_t i = 0; i < N; ++i) {
                int64_t a = std::max(jl[i], b0), e = std::min(jh[i], b1);
                if (a >= e) continue;
                if (der[i].S == 0.0) continue;      /* OpenMPManager.cpp:402 */
                for (int64_t j = a; j < e; ++j)
                    local[(size_t)(j - s0)] += line_term(J, der[i], grid_f(J, j));
            }
        }
    };
    for (int t = 0; t < nthreads; ++t) th.emplace_back(work);
    for (auto& t : th) t.join();
    for (int64_t j = 0; j < n; ++j)
        out[s0 + j] = J->accumulate ? out[s0 + j] + local[(size_t)j] : local[(size_t)j];
    return GEXS_OK;
}

/* Exact number of (line, bin) evaluations of a job (sum of window sizes). */
int64_t orc_count_evals(const gexs_job* J)
{
    int64_t tot = 0;
    for (int64_t i = 0; i < J->lines.count; ++i) {
        double nu = J->lines.nu[i];
        if (nu == 0.0) nu = 1e-6;
        int64_t a, b;
        window(J, nu, &a, &b);
        tot += b - a;
    }
    return tot;
}

/* Voigt: counts of (line, bin) evaluations per Humlicek region 1..4 into
 * hist[0..3], for the FLOP accounting of the roofline. */
int orc_region_hist(const gexs_job* J, int64_t* hist)
{
    for (int r = 0; r < 4; ++r) hist[r] = 0;
    for (int64_t i = 0; i < J->lines.count; ++i) {
        LineDerived d = derive(J, i);
        int64_t a, b;
        window(J, d.nu, &a, &b);
        for (int64_t j = a; j < b; ++j) {
            double x = std::fabs(grid_f(J, j) - d.nu) * d.invw;
            hist[orc_humlicek_region(x, d.y) - 1]++;
        }
    }
    return GEXS_OK;
}

/* Per-line derived values (for tests of the S(T) / width stage). */
int orc_line_params(const gexs_job* J, double* S, double* invw, double* y)
{
    for (int64_t i = 0; i < J->lines.count; ++i) {
        LineDerived d = derive(J, i);
        if (S) S[i] = d.S;
        if (invw) invw[i] = d.invw;
        if (y) y[i] = d.y;
    }
    return GEXS_OK;
}

} /* extern "C" */
