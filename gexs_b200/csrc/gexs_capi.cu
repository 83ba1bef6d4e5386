/*
 * gexs_capi.cu — C ABI of the engine: contexts, one-shot runs, batches
 * captured into CUDA graphs, the launch-shape autotuner, convention presets,
 * eval counting and the partition function.
 *
 * Errors never print or exit (the reference's CheckCudaError prints and
 * calls exit(-1), compute/CUDA/cuda_utils.cu:8-17): every entry point
 * returns a status and leaves a message for gexs_last_error().
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "gexs_internal.h"

namespace gexs {

static thread_local std::string g_last_error;

int set_error(int status, const std::string& msg)
{
    g_last_error = msg;
    return status;
}

int cuda_error(cudaError_t e, const char* where)
{
    return set_error(GEXS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorName(e) + " (" +
                                        cudaGetErrorString(e) + ")");
}

int validate_job(const gexs_job& j, int i)
{
    auto bad = [&](const char* what) {
        return set_error(GEXS_ERR_INVALID, "job " + std::to_string(i) + ": " + what);
    };
    if (profile_class(j) < 0) return bad("unsupported profile (or quad_nodes not 16/32)");
    if (j.precision != GEXS_FP32 && j.precision != GEXS_FP64) return bad("precision");
    if (j.window_rule != GEXS_WINDOW_INCLUSIVE && j.window_rule != GEXS_WINDOW_ROUNDED)
        return bad("window_rule");
    if (j.erf_form != GEXS_ERF_STABLE && j.erf_form != GEXS_ERF_LITERAL) return bad("erf_form");
    if (!j.out) return bad("out is NULL");
    if (j.lines.count < 0) return bad("negative line count");
    if (j.lines.format != GEXS_LINES_FP64 && j.lines.format != GEXS_LINES_COMPACT)
        return bad("line format");
    const bool compact = j.lines.format == GEXS_LINES_COMPACT;
    if (j.lines.count > 0 && (!j.lines.nu || !j.lines.elow || !j.lines.aif || (!compact && !j.lines.gns)))
        return bad("line arrays are NULL");
    bool press = j.profile == GEXS_VOIGT || j.profile == GEXS_VOIGT_QUAD;
    if (press && j.lines.count > 0 && (!j.lines.gamma || !j.lines.n))
        return bad("gamma/n arrays required by this profile");
    if (!(j.dnu > 0.0) || !std::isfinite(j.nu_start)) return bad("grid spacing must be > 0");
    if (j.grid_points < 1 || j.start_idx < 0 || j.n_points < 0 ||
        j.start_idx + j.n_points > j.grid_points)
        return bad("sub-range outside the grid");
    if (!(j.cutoff >= 0.0) || !std::isfinite(j.cutoff)) return bad("cutoff");
    if (j.cutoff / j.dnu > 4.0e6) return bad("cutoff/dnu above 4e6 bins");
    if (!(j.partition > 0.0)) return bad("partition must be > 0");
    if (j.profile == GEXS_GAUSSIAN && !(j.inv_width > 0.0)) return bad("inv_width");
    if (j.profile != GEXS_GAUSSIAN && !(j.dop_coef > 0.0)) return bad("dop_coef");
    return GEXS_OK;
}

}  // namespace gexs

using namespace gexs;

/* ----------------------------------------------------------- context */
struct gexs_ctx {
    int device = 0;
    int nsm = 148;
    int* d_err = nullptr;            /* kernel error word; d_err[1]: its last reading */
    /* launch tables and per-line prep arrays: kept mapped between calls (no
     * release threshold) and never made to wait on a free from another
     * stream (no internal dependencies), so calls on two streams overlap */
    cudaMemPool_t pool = nullptr;
    std::mutex mu;
    std::map<int, gexs_launch_cfg> tuned;   /* key: pk*4 + prec */
};

namespace gexs {
int ctx_device(gexs_ctx* c) { return c->device; }
int ctx_sm_count(gexs_ctx* c) { return c->nsm; }
cudaMemPool_t ctx_pool(gexs_ctx* c) { return c->pool; }

/* gexs_debug_fail_allocs: allocations still to refuse (host-side fault
 * injection for the out-of-memory paths; nothing reaches the device) */
static std::atomic<int> g_fail_allocs{0};

cudaError_t pool_alloc(cudaMemPool_t pool, void** p, size_t bytes, cudaStream_t s)
{
    for (int n = g_fail_allocs.load(); n > 0; n = g_fail_allocs.load())
        if (g_fail_allocs.compare_exchange_weak(n, n - 1)) return cudaErrorMemoryAllocation;
    if (!pool) return cudaMallocAsync(p, bytes, s);
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, s);
    if (e == cudaErrorMemoryAllocation) {
        /* the pool keeps freed pages mapped; when they are too fragmented
         * for this size, give back what no allocation uses and retry once */
        cudaGetLastError();
        cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocFromPoolAsync(p, bytes, pool, s);
    }
    return e;
}
}  // namespace gexs

/* profile_class() of GEXS_VOIGT */
constexpr int PK_VOIGT_CLASS = 0;

static gexs_launch_cfg default_cfg(int pk, int prec)
{
    /* measured best on B200 for the 1e8-line Voigt workload (FP32: 4 bins x
     * 4 warps with 256-line stages, FP64: 4 x 8); gexs_autotune replaces it
     * per (profile, precision) */
    gexs_launch_cfg c{};
    c.bins_per_lane = 4;
    c.warps = (prec == GEXS_FP64) ? 8 : 4;
    c.ctas_per_sm = 0;
    c.flags = (pk == PK_VOIGT_CLASS && prec == GEXS_FP32) ? GEXS_LAUNCH_LONG_STAGES : 0;
    return c;
}

static bool cfg_ok(const gexs_launch_cfg& c, int prec)
{
    /* 16 bins per lane only for the FP32 form */
    return (c.bins_per_lane == 2 || c.bins_per_lane == 4 || c.bins_per_lane == 8 ||
            (c.bins_per_lane == 16 && prec == GEXS_FP32)) &&
           (c.warps == 4 || c.warps == 8) && c.ctas_per_sm >= 0 && c.wait_spins >= 0 &&
           (c.flags & ~(GEXS_LAUNCH_DERIVE_ON_LOAD | GEXS_LAUNCH_LONG_STAGES |
                        GEXS_LAUNCH_JOB_MAJOR)) == 0;
}

static gexs_launch_cfg ctx_cfg(gexs_ctx* ctx, int pk, int prec)
{
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->tuned.find(pk * 4 + prec);
    return it == ctx->tuned.end() ? default_cfg(pk, prec) : it->second;
}

/* a group = jobs of one (profile class, precision): one kernel launch */
struct Group {
    int pk, prec;
    std::vector<gexs_job> jobs;
    std::vector<int> prefix;
    std::vector<int> order;   /* tile-major order tables, empty: job-major */
    int nitems = 0;
};

/* Tile-major item order of a group with several jobs (GEXS_LAUNCH_JOB_MAJOR
 * unset): item rows t = 0, 1, ... each hold tile t of every job that has
 * more than t tiles.  With the jobs ranked by tile count (descending,
 * stable), the rows fall into segments s = 0..nj-1 in which the first
 * nj - s ranked jobs are active:
 *   F[s]  first item of segment s (F[nj] = item count)
 *   R[s]  first tile row of segment s
 *   P[k]  job of rank k
 * laid out as F | R | P (3 nj + 1 ints); decoded by tile_job on the device. */
static std::vector<int> tile_order(const std::vector<int>& n)
{
    const int nj = (int)n.size();
    std::vector<int> perm(nj);
    for (int i = 0; i < nj; ++i) perm[i] = i;
    std::stable_sort(perm.begin(), perm.end(), [&](int x, int y) { return n[x] > n[y]; });
    std::vector<int> out(3 * (size_t)nj + 1);
    int* F = out.data();
    int* R = F + nj + 1;
    int* P = R + nj;
    long long f = 0;
    for (int s = 0; s < nj; ++s) {
        const int active = nj - s;
        const int r0 = s == 0 ? 0 : n[perm[nj - s]];   /* rows of the job that dropped out */
        const int r1 = n[perm[nj - s - 1]];            /* fewest tiles among the active */
        F[s] = (int)f;
        R[s] = r0;
        f += (long long)active * (r1 - r0);
    }
    F[nj] = (int)f;
    for (int k = 0; k < nj; ++k) P[k] = perm[k];
    return out;
}

static int build_groups(const gexs_job* jobs, int njobs, const gexs_launch_cfg* cfg_in,
                        gexs_ctx* ctx, std::vector<Group>& groups,
                        std::vector<gexs_launch_cfg>& cfgs)
{
    groups.clear(); cfgs.clear();
    if (njobs < 0 || (njobs > 0 && !jobs)) return set_error(GEXS_ERR_INVALID, "jobs");
    std::map<int, int> gi;
    for (int i = 0; i < njobs; ++i) {
        int st = validate_job(jobs[i], i);
        if (st) return st;
        int pk = profile_class(jobs[i]), prec = jobs[i].precision;
        int key = pk * 4 + prec;
        if (!gi.count(key)) {
            gi[key] = (int)groups.size();
            Group g; g.pk = pk; g.prec = prec; g.prefix.push_back(0);
            groups.push_back(g);
            gexs_launch_cfg c = cfg_in ? *cfg_in : ctx_cfg(ctx, pk, prec);
            if (!cfg_ok(c, prec)) return set_error(GEXS_ERR_INVALID, "launch configuration");
            cfgs.push_back(c);
        }
        Group& g = groups[gi[key]];
        int W = tile_bins(cfgs[gi[key]]);
        int64_t tiles = (jobs[i].n_points + W - 1) / W;
        if ((int64_t)g.nitems + tiles > (int64_t)INT32_MAX)
            return set_error(GEXS_ERR_INVALID, "too many tiles in one launch");
        g.jobs.push_back(jobs[i]);
        g.nitems += (int)tiles;
        g.prefix.push_back(g.nitems);
    }
    for (size_t k = 0; k < groups.size(); ++k)
        if (groups[k].jobs.size() > 1 && !(cfgs[k].flags & GEXS_LAUNCH_JOB_MAJOR))
        {
            const Group& g = groups[k];
            std::vector<int> n(g.jobs.size());
            for (size_t i = 0; i < n.size(); ++i) n[i] = g.prefix[i + 1] - g.prefix[i];
            groups[k].order = tile_order(n);
        }
    return GEXS_OK;
}

/* device image of a group:
 *   [jobs][prefix][counter][prep pointers][prep arrays (S|invw|y per job)]
 * prep arrays only when the group derives per job (the default). */
struct Layout {
    size_t op, oc, opp, oprep, bytes;
    std::vector<size_t> job_prep;   /* byte offset of each job's prep arrays */
    /* line-slice tables (FP32 Voigt groups): offsets, item bound, lines per slice */
    bool sliced = false;
    size_t os_prefix = 0, os_counts = 0, os_rowbase = 0, os_ticket = 0, os_lohi = 0, os_nitems = 0,
           os_rows = 0;
    int max_rows = 0;
    long long lines_per_slice = 0;
    /* the FP32 Voigt core kernel's slice tables */
    bool csliced = false;
    size_t oc_prefix = 0, oc_counts = 0, oc_rowbase = 0, oc_ticket = 0, oc_lohi = 0, oc_nitems = 0,
           oc_rows = 0;
    int cmax_rows = 0;
    long long clines_per_slice = 0;
};

static Layout group_layout(const Group& g, bool prep, const gexs_launch_cfg& cfg)
{
    Layout L;
    auto up = [](size_t a) { return (a + 255) & ~size_t(255); };
    size_t a = up(g.jobs.size() * sizeof(gexs_job));
    L.op = a;
    a = up(a + (g.prefix.size() + g.order.size()) * sizeof(int));
    L.oc = a;
    a += 256;
    L.opp = a;
    a = up(a + g.jobs.size() * sizeof(double*));
    L.oprep = a;
    for (const gexs_job& j : g.jobs) {
        L.job_prep.push_back(a);
        if (prep) a = up(a + (size_t)j.lines.count * 3 * sizeof(double));
    }
    if (slices_apply(g.pk, g.prec) && g.nitems > 0) {
        const int W = tile_bins(cfg);
        const size_t nt = (size_t)g.nitems;
        L.sliced = true;
        L.lines_per_slice = slice_lines(g.jobs.data(), (int)g.jobs.size(), W, &L.max_rows);
        L.os_prefix = up(a); a = L.os_prefix + (nt + 1) * sizeof(int);
        L.os_counts = up(a); a = L.os_counts + nt * sizeof(int);
        L.os_rowbase = up(a); a = L.os_rowbase + nt * sizeof(int);
        L.os_ticket = up(a); a = L.os_ticket + nt * sizeof(int);
        L.os_lohi = up(a);   a = L.os_lohi + 2 * nt * sizeof(long long);
        L.os_nitems = up(a); a = L.os_nitems + 256;
        L.os_rows = up(a);   a = L.os_rows + (size_t)L.max_rows * W * sizeof(double);
        if (core_slices_apply(g.pk, g.prec, W)) {
            L.csliced = true;
            L.clines_per_slice = core_slice_lines(g.jobs.data(), (int)g.jobs.size(), W, &L.cmax_rows);
            L.oc_prefix = up(a); a = L.oc_prefix + (nt + 1) * sizeof(int);
            L.oc_counts = up(a); a = L.oc_counts + nt * sizeof(int);
            L.oc_rowbase = up(a); a = L.oc_rowbase + nt * sizeof(int);
            L.oc_ticket = up(a); a = L.oc_ticket + nt * sizeof(int);
            L.oc_lohi = up(a);   a = L.oc_lohi + 2 * nt * sizeof(long long);
            L.oc_nitems = up(a); a = L.oc_nitems + 256;
            L.oc_rows = up(a);   a = L.oc_rows + (size_t)L.cmax_rows * W * sizeof(double);
        }
    }
    L.bytes = a + 256;
    return L;
}

static std::vector<unsigned char> group_image(const Group& g, const Layout& L, unsigned char* dev,
                                              bool prep)
{
    std::vector<unsigned char> h(L.oprep, 0);
    std::memcpy(h.data(), g.jobs.data(), g.jobs.size() * sizeof(gexs_job));
    std::memcpy(h.data() + L.op, g.prefix.data(), g.prefix.size() * sizeof(int));
    if (!g.order.empty())
        std::memcpy(h.data() + L.op + g.prefix.size() * sizeof(int), g.order.data(),
                    g.order.size() * sizeof(int));
    double** pp = reinterpret_cast<double**>(h.data() + L.opp);
    for (size_t i = 0; i < g.jobs.size(); ++i)
        pp[i] = prep ? reinterpret_cast<double*>(dev + L.job_prep[i]) : nullptr;
    return h;
}

static bool has_compact(const Group& g)
{
    for (const gexs_job& j : g.jobs)
        if (j.lines.format == GEXS_LINES_COMPACT) return true;
    return false;
}

static int64_t max_lines(const Group& g)
{
    int64_t m = 0;
    for (const gexs_job& j : g.jobs) m = std::max<int64_t>(m, j.lines.count);
    return m;
}

/* prep kernel then tile kernel for one group whose image is at d */
static cudaError_t enqueue_group(const Group& g, const Layout& L, unsigned char* d, bool prep,
                                 const gexs_launch_cfg& cfg, int* d_err, int nsm, cudaStream_t s)
{
    double* const* pp = reinterpret_cast<double* const*>(d + L.opp);
    cudaError_t e = cudaSuccess;
    if (prep) e = launch_prep((const gexs_job*)d, pp, (int)g.jobs.size(), max_lines(g), nsm, s);
    if (e != cudaSuccess) return e;
    SliceTables sl;
    std::memset(&sl, 0, sizeof(sl));
    if (L.sliced) {
        sl.prefix = (int*)(d + L.os_prefix);
        sl.counts = (int*)(d + L.os_counts);
        sl.rowbase = (int*)(d + L.os_rowbase);
        sl.ticket = (int*)(d + L.os_ticket);
        sl.lohi = (long long*)(d + L.os_lohi);
        sl.nitems = (int*)(d + L.os_nitems);
        sl.rows = (double*)(d + L.os_rows);
        sl.max_rows = L.max_rows;
        sl.lines_per_slice = L.lines_per_slice;
    }
    SliceTables csl;
    std::memset(&csl, 0, sizeof(csl));
    if (L.csliced) {
        csl.prefix = (int*)(d + L.oc_prefix);
        csl.counts = (int*)(d + L.oc_counts);
        csl.rowbase = (int*)(d + L.oc_rowbase);
        csl.ticket = (int*)(d + L.oc_ticket);
        csl.lohi = (long long*)(d + L.oc_lohi);
        csl.nitems = (int*)(d + L.oc_nitems);
        csl.rows = (double*)(d + L.oc_rows);
        csl.max_rows = L.cmax_rows;
        csl.lines_per_slice = L.clines_per_slice;
    }
    return launch_tiles(g.pk, g.prec, (const gexs_job*)d, (const int*)(d + L.op),
                        (int)g.jobs.size(), g.nitems, (int*)(d + L.oc), d_err,
                        prep ? pp : nullptr, cfg, nsm, s, L.sliced ? &sl : nullptr,
                        L.csliced ? &csl : nullptr,
                        g.order.empty() ? nullptr : (const int*)(d + L.op) + g.prefix.size());
}

extern "C" {

int gexs_version(void) { return 100; }

int gexs_debug_tile_order(const int32_t* tiles, int njobs, int32_t* out)
{
    if (!tiles || !out || njobs < 1) return set_error(GEXS_ERR_INVALID, "gexs_debug_tile_order: arguments");
    std::vector<int> n(tiles, tiles + njobs);
    long long total = 0;
    for (int v : n) {
        if (v < 0) return set_error(GEXS_ERR_INVALID, "gexs_debug_tile_order: negative tile count");
        total += v;
    }
    if (total > (long long)INT32_MAX) return set_error(GEXS_ERR_INVALID, "gexs_debug_tile_order: too many tiles");
    const std::vector<int> o = tile_order(n);
    std::memcpy(out, o.data(), o.size() * sizeof(int32_t));
    return GEXS_OK;
}

int gexs_debug_fail_allocs(int n)
{
    if (n < 0) return set_error(GEXS_ERR_INVALID, "gexs_debug_fail_allocs: n < 0");
    g_fail_allocs.store(n);
    return GEXS_OK;
}

const char* gexs_status_string(int s)
{
    switch (s) {
    case GEXS_OK: return "ok";
    case GEXS_ERR_INVALID: return "invalid argument";
    case GEXS_ERR_OOM: return "out of memory";
    case GEXS_ERR_CUDA: return "CUDA error";
    case GEXS_ERR_TIMEOUT: return "timeout";
    case GEXS_ERR_NOT_READY: return "not ready";
    case GEXS_ERR_ADMISSION: return "exceeds memory budget";
    case GEXS_ERR_SHUTDOWN: return "shutting down";
    case GEXS_ERR_KERNEL: return "kernel error flag set";
    }
    return "unknown status";
}

const char* gexs_last_error(void) { return g_last_error.c_str(); }

int gexs_job_init(gexs_job* job, int convention, int profile, double temperature,
                  double pressure, double partition, double mean_mass, double ref_temp,
                  double ref_press, double half_width, double cutoff, double nu_start,
                  double dnu, int64_t grid_points)
{
    if (!job) return set_error(GEXS_ERR_INVALID, "job is NULL");
    if (!(temperature > 0.0) || !(mean_mass > 0.0 || profile == GEXS_GAUSSIAN))
        return set_error(GEXS_ERR_INVALID, "temperature and mass must be > 0");
    if (!(dnu > 0.0) || grid_points < 1) return set_error(GEXS_ERR_INVALID, "grid");
    gexs_job j;
    std::memset(&j, 0, sizeof(j));
    j.profile = profile;
    j.precision = GEXS_FP64;
    j.quad_nodes = 16;
    j.nu_start = nu_start; j.dnu = dnu; j.grid_points = grid_points;
    j.start_idx = 0; j.n_points = grid_points;
    j.partition = partition;
    j.s_scale2 = 1.0;
    j.gamma_scale = 1.0;
    j.t_ratio = ref_temp / temperature;
    /* cgs constants of common/defines.h:23-25 */
    const double PLANCK = 6.6260693e-27, VELLGT = 2.99792458e+10, BOLTZ = 1.380658e-16;
    const bool press = profile == GEXS_VOIGT || profile == GEXS_VOIGT_QUAD;
    if (convention == GEXS_CONV_PHYSICAL) {
        const double NA = 6.02214129e+23;                 /* GPUManager.cpp:34 */
        const double pi = std::acos(-1.0);
        j.beta = PLANCK * VELLGT / (BOLTZ * temperature);
        j.s_scale = 1.0 / (8.0 * pi * VELLGT);
        j.dop_coef = std::sqrt(2.0 * BOLTZ * temperature * NA / mean_mass) / VELLGT;
        if (profile == GEXS_GAUSSIAN) j.inv_width = std::sqrt(std::log(2.0)) / half_width;
        j.gamma_scale = pressure / 1.01325;               /* bar -> atm */
        j.cutoff = cutoff >= 0.0 ? cutoff : 25.0;
        j.window_rule = GEXS_WINDOW_INCLUSIVE;
        j.erf_form = GEXS_ERF_STABLE;
        j.out_scale = press ? 1.0 / std::sqrt(pi) : 0.5 / dnu;
    } else if (convention == GEXS_CONV_REF_CPU) {
        /* Managers/CPU/OpenMPManager.cpp: constants of common/defines.h */
        const double PI = 3.14159265359, LN2 = 0.69314718056, NA = 6.0221412927e23;
        const double ISQRTPI = 0.564189584;
        j.beta = PLANCK * VELLGT / (BOLTZ * temperature);
        j.s_scale = 1.0 / (8.0 * PI * VELLGT);             /* :115 */
        j.s_scale2 = press ? ISQRTPI : 1.0;                 /* :394 vs :296 */
        j.dop_coef = std::sqrt(2.0 * LN2 * BOLTZ * temperature * NA / (mean_mass)) / VELLGT;
        if (profile == GEXS_GAUSSIAN) j.inv_width = 0.832554611 / half_width;
        j.gamma_scale = 1.0;                                /* :398, no pressure */
        if (cutoff >= 0.0) j.cutoff = cutoff;
        else if (press) j.cutoff = std::min(25.0 * pressure, 100.0);   /* :386 */
        else if (profile == GEXS_GAUSSIAN) j.cutoff = 10.0 * half_width;
        else j.cutoff = 100.0;                              /* DOPPLER_CUTOFF */
        j.window_rule = GEXS_WINDOW_ROUNDED;
        j.erf_form = GEXS_ERF_LITERAL;
        j.out_scale = (profile == GEXS_GAUSSIAN) ? 0.5 / dnu : 1.0;
    } else if (convention == GEXS_CONV_REF_GPU) {
        /* compute/CUDA/cross_kernal_v2.cu with GPUManager.cpp:29-49 */
        const double SQRTLN2 = 0.832554611, ISQRTPI = 0.564189584, CM_COEF = 1.327209365e-12;
        const double avogno = 6.02214129e+23, ln2 = std::log(2.0);
        const double dpwco = std::sqrt(2.0 * ln2 * BOLTZ * avogno / mean_mass) / VELLGT;
        j.beta = PLANCK * VELLGT / (BOLTZ * temperature);
        j.s_scale = CM_COEF;
        j.dop_coef = std::sqrt(temperature) * dpwco / SQRTLN2;
        if (profile == GEXS_GAUSSIAN) j.inv_width = SQRTLN2 / half_width;
        j.gamma_scale = pressure * ref_press;               /* :142 */
        if (cutoff >= 0.0) j.cutoff = cutoff;
        else if (profile == GEXS_GAUSSIAN) j.cutoff = 10.0 * half_width;
        else j.cutoff = 100.0;                              /* LORENTZ/DOPPLER_CUTOFF */
        j.window_rule = GEXS_WINDOW_INCLUSIVE;
        j.erf_form = GEXS_ERF_LITERAL;
        j.out_scale = press ? ISQRTPI : 0.5 / dnu;
    } else {
        return set_error(GEXS_ERR_INVALID, "unknown convention");
    }
    *job = j;
    return GEXS_OK;
}

int gexs_ctx_create(int device, gexs_ctx** out)
{
    if (!out) return set_error(GEXS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    gexs_ctx* c = new gexs_ctx();
    c->device = device;
    e = cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) { delete c; return cuda_error(e, "cudaDeviceGetAttribute"); }
    e = cudaMalloc(&c->d_err, 2 * sizeof(int));
    if (e != cudaSuccess) { delete c; return set_error(GEXS_ERR_OOM, "error word"); }
    cudaMemset(c->d_err, 0, 2 * sizeof(int));
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &props) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        int no = 0;
        if (cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess ||
            cudaMemPoolSetAttribute(c->pool, cudaMemPoolReuseAllowInternalDependencies, &no) != cudaSuccess) {
            cudaMemPoolDestroy(c->pool);
            c->pool = nullptr;
        }
    } else {
        c->pool = nullptr;
    }
    cudaGetLastError();
    *out = c;
    return GEXS_OK;
}

int gexs_ctx_destroy(gexs_ctx* ctx)
{
    if (!ctx) return GEXS_OK;
    cudaSetDevice(ctx->device);
    cudaFree(ctx->d_err);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return GEXS_OK;
}

int gexs_ctx_check(gexs_ctx* ctx, void* stream)
{
    if (!ctx) return set_error(GEXS_ERR_INVALID, "ctx is NULL");
    cudaSetDevice(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamSynchronize");
    int flag = 0;
    /* one reading slot per context: checks from several threads take turns */
    std::lock_guard<std::mutex> g(ctx->mu);
    e = take_word(ctx->d_err, ctx->d_err + 1, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, ctx->d_err + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "read error word");
    if (flag) return set_error(GEXS_ERR_KERNEL, "kernel error flag " + std::to_string(flag));
    return GEXS_OK;
}

int gexs_run(gexs_ctx* ctx, const gexs_job* jobs, int njobs, const gexs_launch_cfg* cfg,
             void* stream)
{
    if (!ctx) return set_error(GEXS_ERR_INVALID, "ctx is NULL");
    return gexs::run_jobs(ctx, jobs, njobs, cfg, stream, nullptr);
}

}  // extern "C"

int gexs::run_scratch_bytes(gexs_ctx* ctx, const gexs_job* jobs, int njobs,
                            const gexs_launch_cfg* cfg, size_t* bytes)
{
    if (!ctx || !bytes) return set_error(GEXS_ERR_INVALID, "arguments");
    std::vector<Group> groups;
    std::vector<gexs_launch_cfg> cfgs;
    int st = build_groups(jobs, njobs, cfg, ctx, groups, cfgs);
    if (st) return st;
    size_t total = 0;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        if (groups[gi].nitems == 0) continue;
        const bool prep = !(cfgs[gi].flags & GEXS_LAUNCH_DERIVE_ON_LOAD);
        total += group_layout(groups[gi], prep, cfgs[gi]).bytes;
    }
    *bytes = total;
    return GEXS_OK;
}

int gexs::run_jobs(gexs_ctx* ctx, const gexs_job* jobs, int njobs, const gexs_launch_cfg* cfg,
                   void* stream, int* d_err)
{
    if (!ctx) return set_error(GEXS_ERR_INVALID, "ctx is NULL");
    if (!d_err) d_err = ctx->d_err;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    std::vector<Group> groups;
    std::vector<gexs_launch_cfg> cfgs;
    int st = build_groups(jobs, njobs, cfg, ctx, groups, cfgs);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        if (g.nitems == 0) continue;
        const bool prep = !(cfgs[gi].flags & GEXS_LAUNCH_DERIVE_ON_LOAD);
        if (!prep && has_compact(g)) return set_error(GEXS_ERR_INVALID, "compact line lists need the prep arrays");
        Layout L = group_layout(g, prep, cfgs[gi]);
        void* d = nullptr;
        e = pool_alloc(ctx->pool, &d, L.bytes, s);
        if (e != cudaSuccess) return set_error(GEXS_ERR_OOM, "launch tables");
        /* the image carries the zeroed work counters */
        std::vector<unsigned char> h = group_image(g, L, (unsigned char*)d, prep);
        e = put_bytes(d, h.data(), h.size(), s);
        if (e != cudaSuccess) { cudaFreeAsync(d, s); return cuda_error(e, "upload launch tables"); }
        e = enqueue_group(g, L, (unsigned char*)d, prep, cfgs[gi], d_err, ctx->nsm, s);
        cudaFreeAsync(d, s);
        if (e != cudaSuccess) return cuda_error(e, "tile kernel launch");
    }
    return GEXS_OK;
}

extern "C" {

int gexs_count_evals(gexs_ctx* ctx, const gexs_job* jobs, int njobs, int64_t* h_counts)
{
    if (!ctx || !jobs || njobs <= 0 || !h_counts) return set_error(GEXS_ERR_INVALID, "arguments");
    for (int i = 0; i < njobs; ++i) {
        int st = validate_job(jobs[i], i);
        if (st) return st;
    }
    cudaSetDevice(ctx->device);
    gexs_job* dj = nullptr; unsigned long long* dc = nullptr;
    cudaError_t e = cudaMalloc(&dj, sizeof(gexs_job) * njobs);
    if (e != cudaSuccess) return set_error(GEXS_ERR_OOM, "count tables");
    e = cudaMalloc(&dc, sizeof(unsigned long long) * njobs);
    if (e != cudaSuccess) { cudaFree(dj); return set_error(GEXS_ERR_OOM, "count tables"); }
    cudaMemcpy(dj, jobs, sizeof(gexs_job) * njobs, cudaMemcpyHostToDevice);
    cudaMemset(dc, 0, sizeof(unsigned long long) * njobs);
    e = launch_count(dj, njobs, dc, ctx->nsm, 0);
    std::vector<unsigned long long> hc(njobs);
    if (e == cudaSuccess) e = cudaMemcpy(hc.data(), dc, sizeof(unsigned long long) * njobs, cudaMemcpyDeviceToHost);
    cudaFree(dj); cudaFree(dc);
    if (e != cudaSuccess) return cuda_error(e, "count kernel");
    for (int i = 0; i < njobs; ++i) h_counts[i] = (int64_t)hc[i];
    return GEXS_OK;
}

}  // extern "C"

/* ------------------------------------------------------------ batches */
struct gexs_batch {
    gexs_ctx* ctx = nullptr;
    std::vector<Group> groups;
    std::vector<gexs_launch_cfg> cfgs;
    std::vector<void*> dmem;          /* per group device image */
    std::vector<Layout> layouts;
    std::vector<bool> prep;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static int batch_enqueue(gexs_batch* b, cudaStream_t s)
{
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        const Group& g = b->groups[gi];
        if (g.nitems == 0) continue;
        unsigned char* d = (unsigned char*)b->dmem[gi];
        cudaError_t e = zero_ints((int*)(d + b->layouts[gi].oc), 1, s);
        if (e != cudaSuccess) return cuda_error(e, "reset work counter");
        e = enqueue_group(g, b->layouts[gi], d, b->prep[gi], b->cfgs[gi], b->ctx->d_err,
                          b->ctx->nsm, s);
        if (e != cudaSuccess) return cuda_error(e, "tile kernel launch");
    }
    return GEXS_OK;
}

extern "C" {

int gexs_batch_create(gexs_ctx* ctx, const gexs_job* jobs, int njobs,
                      const gexs_launch_cfg* cfg, gexs_batch** out)
{
    if (!ctx || !out) return set_error(GEXS_ERR_INVALID, "arguments");
    *out = nullptr;
    cudaSetDevice(ctx->device);
    gexs_batch* b = new gexs_batch();
    b->ctx = ctx;
    int st = build_groups(jobs, njobs, cfg, ctx, b->groups, b->cfgs);
    if (st) { delete b; return st; }
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        const Group& g = b->groups[gi];
        const bool prep = !(b->cfgs[gi].flags & GEXS_LAUNCH_DERIVE_ON_LOAD);
        if (!prep && has_compact(g)) {
            gexs_batch_destroy(b);
            return set_error(GEXS_ERR_INVALID, "compact line lists need the prep arrays");
        }
        Layout L = group_layout(g, prep, b->cfgs[gi]);
        void* d = nullptr;
        if (cudaMalloc(&d, L.bytes) != cudaSuccess) { gexs_batch_destroy(b); return set_error(GEXS_ERR_OOM, "batch tables"); }
        b->dmem.push_back(d); b->layouts.push_back(L); b->prep.push_back(prep);
        std::vector<unsigned char> h = group_image(g, L, (unsigned char*)d, prep);
        cudaError_t e = cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { gexs_batch_destroy(b); return cuda_error(e, "upload batch tables"); }
    }
    *out = b;
    return GEXS_OK;
}

int gexs_batch_launch(gexs_batch* b, void* stream)
{
    if (!b) return set_error(GEXS_ERR_INVALID, "batch is NULL");
    cudaSetDevice(b->ctx->device);
    return batch_enqueue(b, (cudaStream_t)stream);
}

int gexs_batch_capture(gexs_batch* b, void* stream)
{
    if (!b) return set_error(GEXS_ERR_INVALID, "batch is NULL");
    cudaSetDevice(b->ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (!s) return set_error(GEXS_ERR_INVALID, "capture needs a non-default stream");
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamBeginCapture");
    int st = batch_enqueue(b, s);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    if (st) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
    return GEXS_OK;
}

int gexs_batch_replay(gexs_batch* b, void* stream)
{
    if (!b || !b->exec) return set_error(GEXS_ERR_INVALID, "batch has no captured graph");
    cudaSetDevice(b->ctx->device);
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_error(e, "cudaGraphLaunch");
    return GEXS_OK;
}

int gexs_batch_destroy(gexs_batch* b)
{
    if (!b) return GEXS_OK;
    cudaSetDevice(b->ctx->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void* d : b->dmem) cudaFree(d);
    delete b;
    return GEXS_OK;
}

int gexs_autotune(gexs_ctx* ctx, const gexs_job* jobs, int njobs, gexs_launch_cfg* best,
                  float* h_ms)
{
    if (!ctx || !jobs || njobs <= 0 || !best) return set_error(GEXS_ERR_INVALID, "arguments");
    cudaSetDevice(ctx->device);
    int pk = profile_class(jobs[0]), prec = jobs[0].precision;
    for (int i = 0; i < njobs; ++i)
        if (profile_class(jobs[i]) != pk || jobs[i].precision != prec)
            return set_error(GEXS_ERR_INVALID, "autotune needs jobs of one profile and precision");
    std::vector<gexs_job> tj(jobs, jobs + njobs);
    for (auto& j : tj) j.accumulate = 0;          /* tuning runs overwrite outputs */
    const int bins[4] = {2, 4, 8, 16}, warps[2] = {4, 8};
    const int nbins = (prec == GEXS_FP32) ? 4 : 3;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return set_error(GEXS_ERR_CUDA, "stream");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    float best_ms = 1e30f; gexs_launch_cfg bc = default_cfg(pk, prec);
    int st = GEXS_OK;
    /* best of two timed launches of one candidate after a warm-up */
    auto time_cfg = [&](const gexs_launch_cfg& c, float* out_ms) -> int {
        gexs_batch* b = nullptr;
        int r = gexs_batch_create(ctx, tj.data(), njobs, &c, &b);
        if (r) return r;
        float ms = 1e30f;
        for (int rep = 0; rep < 3 && !r; ++rep) {
            cudaEventRecord(e0, s);
            r = gexs_batch_launch(b, s);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) r = set_error(GEXS_ERR_CUDA, "autotune run");
            float t = 0.f; cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0) ms = std::min(ms, t);        /* first run warms up */
        }
        gexs_batch_destroy(b);
        *out_ms = ms;
        return r;
    };
    /* stage length is a further candidate where it exists (FP32 Voigt,
     * 512-bin tiles) */
    const bool stages = jobs[0].profile == GEXS_VOIGT && prec == GEXS_FP32;
    for (int bi = 0; bi < nbins && !st; ++bi)
        for (int wi = 0; wi < 2 && !st; ++wi)
        for (int li = 0; li < 2 && !st; ++li) {
            if (li && !(stages && bins[bi] * warps[wi] == 16)) continue;
            gexs_launch_cfg c{}; c.bins_per_lane = bins[bi]; c.warps = warps[wi];
            c.ctas_per_sm = 0; c.flags = li ? GEXS_LAUNCH_LONG_STAGES : 0;
            float ms = 1e30f;
            st = time_cfg(c, &ms);
            if (!st && ms < best_ms) { best_ms = ms; bc = c; }
        }
    /* several jobs: the item order too (tile-major, the default, shares a
     * tile's lines between the jobs through L2; job-major does not), tried
     * on the best shape; both give the same bits */
    if (!st && njobs > 1) {
        gexs_launch_cfg c = bc;
        c.flags |= GEXS_LAUNCH_JOB_MAJOR;
        float ms = 1e30f;
        st = time_cfg(c, &ms);
        if (!st && ms < best_ms) { best_ms = ms; bc = c; }
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (st) return st;
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        ctx->tuned[pk * 4 + prec] = bc;
    }
    *best = bc;
    if (h_ms) *h_ms = best_ms;
    return GEXS_OK;
}

int gexs_partition(gexs_ctx* ctx, const double* d_energy, const int32_t* d_g, int64_t nstates,
                   const double* h_temps, int nt, double* h_q)
{
    if (!ctx || !d_energy || !d_g || nstates <= 0 || !h_temps || nt <= 0 || !h_q)
        return set_error(GEXS_ERR_INVALID, "arguments");
    cudaSetDevice(ctx->device);
    const double planck = 6.6260693e-27, vellgt = 2.99792458e10, boltz = 1.380658e-16;
    std::vector<double> betas(nt);
    for (int i = 0; i < nt; ++i) {
        if (!(h_temps[i] > 0.0)) return set_error(GEXS_ERR_INVALID, "temperature must be > 0");
        betas[i] = planck * vellgt / (boltz * h_temps[i]);
    }
    int nchunk = (int)std::min<int64_t>(ctx->nsm * 2, (nstates + 255) / 256);
    double *db = nullptr, *dp = nullptr, *dq = nullptr;
    if (cudaMalloc(&db, sizeof(double) * nt) != cudaSuccess ||
        cudaMalloc(&dp, sizeof(double) * (size_t)nt * nchunk) != cudaSuccess ||
        cudaMalloc(&dq, sizeof(double) * nt) != cudaSuccess) {
        cudaFree(db); cudaFree(dp); cudaFree(dq);
        return set_error(GEXS_ERR_OOM, "partition buffers");
    }
    cudaMemcpy(db, betas.data(), sizeof(double) * nt, cudaMemcpyHostToDevice);
    cudaError_t e = launch_partition(d_energy, d_g, nstates, db, nt, dp, nchunk, dq, 0);
    if (e == cudaSuccess) e = cudaMemcpy(h_q, dq, sizeof(double) * nt, cudaMemcpyDeviceToHost);
    cudaFree(db); cudaFree(dp); cudaFree(dq);
    if (e != cudaSuccess) return cuda_error(e, "partition kernel");
    return GEXS_OK;
}

}  // extern "C"
