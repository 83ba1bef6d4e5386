/*
 * gexs_kernels.cu — the per-job prep kernel, exact evaluation counting,
 * Q(T), and the front of the tile-kernel dispatch (the tile kernel itself
 * is in gexs_tiles.cuh).
 */
#include <cmath>
#include <cstring>
#include <cub/cub.cuh>
#include "gexs_tiles.cuh"

namespace gexs {

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
    const bool compact = J.lines.format == GEXS_LINES_COMPACT;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * blockDim.x) {
        RawLine L;
        L.nu = J.lines.nu[i];
        if (compact) {
            /* floats widened to FP64; aif holds g' A */
            L.elow = (double)reinterpret_cast<const float*>(J.lines.elow)[i];
            L.aif = (double)reinterpret_cast<const float*>(J.lines.aif)[i];
            L.g = 1;
        } else {
            L.elow = J.lines.elow[i]; L.aif = J.lines.aif[i];
            L.g = J.lines.gns[i];
        }
        LineQ q;
        if (press) {
            if (compact) {
                L.gam = (double)reinterpret_cast<const float*>(J.lines.gamma)[i];
                L.nexp = (double)reinterpret_cast<const float*>(J.lines.n)[i];
            } else {
                L.gam = J.lines.gamma[i]; L.nexp = J.lines.n[i];
            }
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
                         cudaStream_t st, const SliceTables* sl, const SliceTables* csl,
                         const int* d_order)
{
    KArgs a;
    a.jobs = d_jobs; a.prefix = d_prefix; a.njobs = njobs; a.nitems = nitems;
    a.order = njobs > 1 ? d_order : nullptr;
    a.counter = d_counter; a.err = d_err; a.prep = d_prep;
    a.tile_w = tile_bins(cfg);
    a.spin = cfg.wait_spins > 0 ? cfg.wait_spins : WS_SPIN;
    std::memset(&a.sl, 0, sizeof(a.sl));
    std::memset(&a.csl, 0, sizeof(a.csl));
    if (sl && slices_apply(pk, prec)) a.sl = *sl;
    if (csl && core_slices_apply(pk, prec, a.tile_w)) a.csl = *csl;
    switch (pk) {
    case PK_VOIGT: return launch_tiles_voigt(prec, a, cfg, nsm, st);
    case PK_ERF:   return launch_tiles_erf(prec, a, cfg, nsm, st);
    case PK_GH16:  return launch_tiles_gh16(prec, a, cfg, nsm, st);
    case PK_GH32:  return launch_tiles_gh32(prec, a, cfg, nsm, st);
    }
    return cudaErrorInvalidValue;
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

/* ------------------------------------------------------------ line slices */
namespace {
/* one warp per tile: the tile's line range, searched exactly as the
 * region-I kernel's producers search it, and its slice count */
__global__ void slice_plan_kernel(const KArgs a)
{
    const int lane = threadIdx.x & 31;
    const int ti = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (ti >= a.nitems) return;
    int tj = 0;
    const int jl = tile_job(a, ti, &tj);
    const gexs_job& J = a.jobs[jl];
    const int64_t j0 = J.start_idx + (int64_t)tj * a.tile_w;
    const int jn = (int)min((int64_t)a.tile_w, J.start_idx + J.n_points - j0);
    const double f0 = grid_f(J.nu_start, J.dnu, j0);
    const double fl = grid_f(J.nu_start, J.dnu, j0 + jn - 1);
    const int64_t nl = J.lines.count;
    const double margin = 2.0 * J.dnu + 1e-9 * (fabs(fl) + J.cutoff);
    const int64_t lo = warp_bound<false>(J.lines.nu, nl, f0 - J.cutoff - margin, lane);
    const int64_t hi = max(warp_bound<true>(J.lines.nu, nl, fl + J.cutoff + margin, lane), lo);
    if (lane == 0) {
        const long long n = hi - lo, per = a.sl.lines_per_slice;
        a.sl.lohi[2 * ti] = lo;
        a.sl.lohi[2 * ti + 1] = hi;
        a.sl.counts[ti] = n > per ? (int)((n + per - 1) / per) : 1;
        a.sl.ticket[ti] = 0;
    }
}

/* the same for the FP32 Voigt core kernel: its line range per tile is the
 * core kernel's own search (lines whose core, |f - nu| < 15 nu dop_coef,
 * can reach the tile), computed with the same expressions */
__global__ void core_slice_plan_kernel(const KArgs a)
{
    const int lane = threadIdx.x & 31;
    const int ti = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (ti >= a.nitems) return;
    int tj = 0;
    const int jl = tile_job(a, ti, &tj);
    const gexs_job& J = a.jobs[jl];
    const int64_t t0 = J.start_idx + (int64_t)tj * a.tile_w;
    const int64_t tend = min((int64_t)(t0 + a.tile_w), J.start_idx + J.n_points);
    const int jn = (int)min((int64_t)CORE_W, tend - t0);
    const double f0 = grid_f(J.nu_start, J.dnu, t0);
    const double fl = grid_f(J.nu_start, J.dnu, t0 + jn - 1);
    const int64_t nl = J.lines.count;
    const double margin = 2.0 * J.dnu + 1e-9 * (fabs(fl) + J.cutoff);
    const double k15 = 15.0 * J.dop_coef;
    double vlo = f0 - J.cutoff, vhi = fl + J.cutoff;
    vlo = fmax(vlo, f0 / (1.0 + k15));
    if (k15 < 1.0) vhi = fmin(vhi, fl / (1.0 - k15));
    vlo -= margin; vhi += margin;
    if (vlo < 1e-6 + margin) vlo = -1.0;
    const int64_t lo = warp_bound<false>(J.lines.nu, nl, vlo, lane);
    const int64_t hi = max(warp_bound<true>(J.lines.nu, nl, vhi, lane), lo);
    if (lane == 0) {
        const long long n = hi - lo, per = a.csl.lines_per_slice;
        a.csl.lohi[2 * ti] = lo;
        a.csl.lohi[2 * ti + 1] = hi;
        a.csl.counts[ti] = n > per ? (int)((n + per - 1) / per) : 1;
        a.csl.ticket[ti] = 0;
    }
}

/* one CTA: exclusive prefixes of the slice counts (items) and of the
 * slices of split tiles (partial rows), and the item count */
__global__ void __launch_bounds__(1024) slice_scan_kernel(const KArgs a)
{
    typedef cub::BlockScan<int, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ long long carry, rcarry;
    if (threadIdx.x == 0) { carry = 0; rcarry = 0; }
    __syncthreads();
    for (int base = 0; base < a.nitems; base += 1024) {
        const int i = base + (int)threadIdx.x;
        const int v = i < a.nitems ? a.sl.counts[i] : 0;
        const int r = v > 1 ? v : 0;
        int ex = 0, tot = 0, rex = 0, rtot = 0;
        Scan(tmp).ExclusiveSum(v, ex, tot);
        __syncthreads();
        Scan(tmp).ExclusiveSum(r, rex, rtot);
        if (i < a.nitems) {
            a.sl.prefix[i] = (int)min(carry + ex, (long long)INT32_MAX);
            a.sl.rowbase[i] = (int)min(rcarry + rex, (long long)INT32_MAX);
        }
        __syncthreads();
        if (threadIdx.x == 0) { carry += tot; rcarry += rtot; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (rcarry > a.sl.max_rows || carry > INT32_MAX) {
            /* cannot happen with the host's bound; run no item rather than
             * write past the partial rows */
            atomicOr(a.err, GEXS_KERR_SLICES);
            *a.sl.nitems = 0;
        } else {
            a.sl.prefix[a.nitems] = (int)carry;
            *a.sl.nitems = (int)carry;
        }
    }
}
}  // namespace

cudaError_t launch_slice_plan(const KArgs& a, cudaStream_t st)
{
    if (a.nitems <= 0) return cudaSuccess;
    slice_plan_kernel<<<(a.nitems + 7) / 8, 256, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    slice_scan_kernel<<<1, 1024, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_core_slice_plan(const KArgs& a, cudaStream_t st)
{
    if (a.nitems <= 0) return cudaSuccess;
    core_slice_plan_kernel<<<(a.nitems + 7) / 8, 256, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    KArgs c = a;
    c.sl = a.csl;
    slice_scan_kernel<<<1, 1024, 0, st>>>(c);
    return cudaGetLastError();
}

bool slices_apply(int, int) { return true; }

bool core_slices_apply(int pk, int prec, int tile_w)
{
    return pk == PK_VOIGT && prec == GEXS_FP32 && tile_w <= CORE_W;
}

long long core_slice_lines(const gexs_job* jobs, int njobs, int tile_w, int* max_rows)
{
    /* as slice_lines, with a line's reach the core's: at most 15 nu
     * dop_coef / (1 - 15 dop_coef) at the job's highest frequency, and at
     * most the cutoff */
    long long per = 8192;
    for (;;) {
        double rows = 0.0;
        for (int i = 0; i < njobs; ++i) {
            const gexs_job& j = jobs[i];
            const double k15 = 15.0 * j.dop_coef;
            const double nu_hi = j.nu_start + (double)(j.start_idx + j.n_points) * j.dnu + j.cutoff;
            double reach = j.cutoff;
            if (k15 < 1.0) reach = std::min(reach, nu_hi * k15 / (1.0 - k15));
            const double tpl = std::floor((2.0 * reach + 8.0 * j.dnu) / ((double)tile_w * j.dnu)) + 3.0;
            rows += 2.0 * std::ceil((double)j.lines.count * tpl / (double)per);
        }
        if (rows * tile_w * sizeof(double) <= (double)(1ull << 30)) {
            *max_rows = (int)rows;
            return per;
        }
        if (per >= (1ll << 40)) { *max_rows = 0; return 1ll << 62; }
        per *= 2;
    }
}

long long slice_lines(const gexs_job* jobs, int njobs, int tile_w, int* max_rows)
{
    /* A line lies in at most (2 (cutoff + margin)) / (tile width) + 2 tiles,
     * so the tiles hold at most sum(lines x that) = M line entries.  A split
     * tile (n > per lines) has ceil(n / per) < 2 n / per slices, so the
     * slices of split tiles, which alone need partial rows, are fewer than
     * 2 M / per.  per doubles until those rows fit in 1 GiB; past 2^40 no
     * tile can be split at all.  16384 lines per slice: measured on one
     * B200, the 1e8-line workload is indifferent to it (16k-128k) and a
     * dense band of 1e6 lines in 80 cm^-1 runs 25% faster than at 65536. */
    long long per = 16384;
    for (;;) {
        double rows = 0.0;
        for (int i = 0; i < njobs; ++i) {
            const gexs_job& j = jobs[i];
            const double tpl = std::floor((2.0 * j.cutoff + 8.0 * j.dnu) / ((double)tile_w * j.dnu)) + 3.0;
            rows += 2.0 * std::ceil((double)j.lines.count * tpl / (double)per);
        }
        if (rows * tile_w * sizeof(double) <= (double)(1ull << 30)) {
            *max_rows = (int)rows;
            return per;
        }
        if (per >= (1ll << 40)) { *max_rows = 0; return 1ll << 62; }
        per *= 2;
    }
}

/* ----------------------------------------------- control writes as kernels */
namespace {
const int kBlobBytes = 4000;                /* under the 4 KB kernel-parameter limit */
struct Blob { unsigned char b[kBlobBytes]; };

__global__ void put_blob_kernel(const Blob p, unsigned char* dst, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = p.b[i];
}

__global__ void zero_ints_kernel(int* p, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 0;
}

__global__ void take_word_kernel(int* word, int* out)
{
    *out = atomicExch(word, 0);
}
}  // namespace

cudaError_t take_word(int* word, int* out, cudaStream_t st)
{
    take_word_kernel<<<1, 1, 0, st>>>(word, out);
    return cudaGetLastError();
}

cudaError_t put_bytes(void* dst, const void* src, size_t n, cudaStream_t st)
{
    if (n > kMaxParamUpload) return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st);
    const unsigned char* s = static_cast<const unsigned char*>(src);
    unsigned char* d = static_cast<unsigned char*>(dst);
    for (size_t o = 0; o < n; o += kBlobBytes) {
        const int k = (int)std::min<size_t>(kBlobBytes, n - o);
        Blob b;
        std::memcpy(b.b, s + o, (size_t)k);
        put_blob_kernel<<<1, 256, 0, st>>>(b, d + o, k);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t zero_ints(int* p, int n, cudaStream_t st)
{
    zero_ints_kernel<<<1, 64, 0, st>>>(p, n);
    return cudaGetLastError();
}

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
