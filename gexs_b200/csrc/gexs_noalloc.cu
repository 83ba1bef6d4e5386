/*
 * gexs_noalloc.cu — gexs_run_noalloc: the tile kernel launched with its
 * scratch memory (job table, tile prefix sums, work counter, error word) in
 * a fixed array that lives in the library's own device image instead of
 * memory from cudaMallocAsync.
 *
 * Who needs it: a caller that must not allocate device memory while it
 * runs - for example a plug-in inside a host program that reserves all of
 * the GPU's memory for its own pool, or a latency-sensitive loop in which a
 * device allocation may stall the other streams or fail.  Such a caller
 * still provides the line arrays and the output grids; this path adds no
 * allocation of its own.
 *
 * The array is a file-scope __device__ object: every GPU that loads the
 * library holds GEXS_NOALLOC_SCRATCH_BYTES of it until the process exits,
 * and all calls on a device share it.
 */
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>
#include "gexs_internal.h"

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kJobsBytes = sizeof(gexs_job) * GEXS_NOALLOC_MAX_JOBS;
constexpr size_t kPrefixOff = (kJobsBytes + 255) & ~size_t(255);
constexpr size_t kCounterOff = (kPrefixOff + sizeof(int) * (GEXS_NOALLOC_MAX_JOBS + 1) + 255) & ~size_t(255);
constexpr size_t kErrOff = kCounterOff + 256;   /* kernel error word of the last call */
constexpr size_t kScratchBytes = kErrOff + 256;
static_assert(kScratchBytes <= GEXS_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds its array");
static_assert(kJobsBytes <= gexs::kMaxParamUpload, "the job table must fit in kernel parameters");

/* Host code must never pass this name to a kernel: on the host it is a
 * stand-in symbol, not a device address.  Its device address comes from
 * cudaGetSymbolAddress below. */
static __device__ __align__(256) unsigned char g_scratch[GEXS_NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
void* g_addr[kMaxDevices] = {nullptr};

/* once per device, with that device current */
int scratch_address(int dev, unsigned char** out)
{
    if (dev < 0 || dev >= kMaxDevices)
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_run_noalloc: device index out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return gexs::cuda_error(e, "gexs_run_noalloc: cudaGetSymbolAddress");
        g_addr[dev] = p;
    }
    *out = (unsigned char*)g_addr[dev];
    return GEXS_OK;
}

}  // namespace

extern "C" int gexs_run_noalloc(const gexs_job* jobs, int njobs, const gexs_launch_cfg* cfg,
                                void* stream)
{
    using namespace gexs;
    if (!jobs || njobs < 1 || njobs > GEXS_NOALLOC_MAX_JOBS)
        return set_error(GEXS_ERR_INVALID, "gexs_run_noalloc: njobs must be 1.." +
                                               std::to_string(GEXS_NOALLOC_MAX_JOBS));
    const int pk = profile_class(jobs[0]), prec = jobs[0].precision;
    /* gexs_run's defaults: 4 bins per lane, 4 warps (FP32) or 8 (FP64) */
    gexs_launch_cfg c{};
    c.bins_per_lane = 4; c.warps = (prec == GEXS_FP64) ? 8 : 4;
    if (cfg) c = *cfg;
    /* no per-job prep arrays: every line is derived as it is loaded */
    c.flags |= GEXS_LAUNCH_DERIVE_ON_LOAD;
    if (!((c.bins_per_lane == 2 || c.bins_per_lane == 4 || c.bins_per_lane == 8) &&
          (c.warps == 4 || c.warps == 8) && c.ctas_per_sm >= 0 && c.wait_spins >= 0))
        return set_error(GEXS_ERR_INVALID, "gexs_run_noalloc: launch configuration");

    /* host image: job table and tile prefix sums */
    struct Image {
        gexs_job jobs[GEXS_NOALLOC_MAX_JOBS];
        int prefix[GEXS_NOALLOC_MAX_JOBS + 1];
    } img;
    const int W = tile_bins(c);
    int64_t nitems = 0;
    img.prefix[0] = 0;
    for (int i = 0; i < njobs; ++i) {
        int st = validate_job(jobs[i], i);
        if (st) return st;
        if (jobs[i].lines.format != GEXS_LINES_FP64)
            return set_error(GEXS_ERR_INVALID, "gexs_run_noalloc: compact line lists need prep arrays");
        if (profile_class(jobs[i]) != pk || jobs[i].precision != prec)
            return set_error(GEXS_ERR_INVALID,
                             "gexs_run_noalloc: all jobs of a call need one profile and precision");
        nitems += (jobs[i].n_points + W - 1) / W;
        if (nitems > (int64_t)INT32_MAX)
            return set_error(GEXS_ERR_INVALID, "gexs_run_noalloc: too many tiles");
        img.jobs[i] = jobs[i];
        img.prefix[i + 1] = (int)nitems;
    }
    if (nitems == 0) return GEXS_OK;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "gexs_run_noalloc: cudaGetDevice");
    unsigned char* base = nullptr;
    int st = scratch_address(dev, &base);
    if (st) return st;
    int nsm = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_error(e, "gexs_run_noalloc: cudaDeviceGetAttribute");

    cudaStream_t s = (cudaStream_t)stream;
    /* the tables travel as kernel parameters (put_bytes), so the call
     * reads nothing from host memory once it has returned */
    e = put_bytes(base, img.jobs, sizeof(gexs_job) * njobs, s);
    if (e == cudaSuccess) e = put_bytes(base + kPrefixOff, img.prefix, sizeof(int) * (njobs + 1), s);
    /* the work counter and the error word start at zero on every call */
    if (e == cudaSuccess)
        e = zero_ints((int*)(base + kCounterOff), (int)((kErrOff - kCounterOff) / sizeof(int)) + 1, s);
    if (e != cudaSuccess) return cuda_error(e, "gexs_run_noalloc: upload launch tables");
    e = launch_tiles(pk, prec, (const gexs_job*)base, (const int*)(base + kPrefixOff), njobs,
                     (int)nitems, (int*)(base + kCounterOff), (int*)(base + kErrOff), nullptr, c, nsm,
                     s);
    if (e != cudaSuccess) return cuda_error(e, "gexs_run_noalloc: tile kernel launch");
    return GEXS_OK;
}

extern "C" int gexs_noalloc_status(void* stream, int* flags)
{
    using namespace gexs;
    if (!flags) return set_error(GEXS_ERR_INVALID, "gexs_noalloc_status: flags is NULL");
    *flags = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "gexs_noalloc_status: cudaGetDevice");
    unsigned char* base = nullptr;
    int st = scratch_address(dev, &base);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    int word = 0;
    e = cudaMemcpyAsync(&word, base + kErrOff, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "gexs_noalloc_status: read error word");
    *flags = word;
    if (word)
        return set_error(GEXS_ERR_KERNEL, "gexs_run_noalloc: kernel error flags " + std::to_string(word));
    return GEXS_OK;
}
