/* gexs_internal.h — declarations shared by the library's translation units. */
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "../../include/gexs_b200.h"

namespace gexs {

/* kernel launchers (gexs_kernels.cu; tile kernels in gexs_tiles.cuh) */
int profile_class(const gexs_job& j);
int tile_bins(const gexs_launch_cfg& c);
/* Line slices of the tile kernels (the FP32 Voigt region-I kernel and
 * tile_kernel; the FP32 Voigt core kernel has its own, below): a tile
 * whose line range
 * holds more than `lines_per_slice` lines (16384 unless the partial rows
 * would pass 1 GiB) is cut into ceil(n / lines_per_slice) work items (the
 * count depends on the tile alone, so the same tile is cut the same way
 * in every launch).  A split tile's slices write
 * partial rows; the last one to finish sums them in slice order into the
 * output.  All arrays live in the launch table; slice_plan_kernel fills
 * them (and zeroes the tickets) before the region-I kernel runs. */
struct SliceTables {
    int*       prefix;      /* ntiles + 1: first item of each tile       */
    int*       counts;      /* ntiles: slices per tile                   */
    int*       rowbase;     /* ntiles: first partial row of a split tile */
    int*       ticket;      /* ntiles: slices finished                   */
    long long* lohi;        /* 2 ntiles: each tile's line range          */
    int*       nitems;      /* 1: items of the launch                    */
    double*    rows;        /* max_rows x tile bins: partial rows        */
    int        max_rows;
    long long  lines_per_slice;
};

/* d_prep: device array of per-job prep arrays (S | invw | y, 3 N doubles
 * each, from launch_prep), or NULL to derive every line on load.
 * d_order: tile-major order tables of a launch with several jobs (F | R | P,
 * 3 njobs + 1 ints, see tile_order in gexs_capi.cu), or NULL for job-major
 * items.
 * d_counter: a 256-byte block of work counters; the caller zeroes the
 * first int, the FP32 Voigt core kernel's counter (int 32) is zeroed here
 * (by zero_ints). */
cudaError_t launch_tiles(int pk, int prec, const gexs_job* d_jobs, const int* d_prefix,
                         int njobs, int nitems, int* d_counter, int* d_err,
                         double* const* d_prep, const gexs_launch_cfg& cfg, int nsm,
                         cudaStream_t st, const SliceTables* sl = nullptr,
                         const SliceTables* csl = nullptr, const int* d_order = nullptr);
/* which groups are sliced (all); lines_per_slice for a group (grows only
 * when the partial rows of its split tiles could pass 1 GiB) and the bound
 * on those rows */
bool slices_apply(int pk, int prec);
long long slice_lines(const gexs_job* jobs, int njobs, int tile_w, int* max_rows);
/* the FP32 Voigt core kernel's own slices (its line range per tile is the
 * lines whose core can reach the tile): only when a tile is one core
 * sub-tile (tile_w <= 1024); 8192 lines per slice unless the rows, bounded
 * by the core reach 15 nu dop_coef instead of the cutoff, would pass 1 GiB */
bool core_slices_apply(int pk, int prec, int tile_w);
long long core_slice_lines(const gexs_job* jobs, int njobs, int tile_w, int* max_rows);
cudaError_t launch_prep(const gexs_job* d_jobs, double* const* d_prep, int njobs,
                        int64_t max_lines, int nsm, cudaStream_t st);
cudaError_t launch_count(const gexs_job* d_jobs, int njobs, unsigned long long* d_counts,
                         int nsm, cudaStream_t st);
cudaError_t launch_partition(const double* d_e, const int32_t* d_g, int64_t n,
                             const double* d_betas, int nt, double* d_partial, int nchunk,
                             double* d_q, cudaStream_t st);

/* small control writes done by kernels (gexs_kernels.cu): a launch table
 * passed as kernel parameters (at most kMaxParamUpload bytes) and zeroed
 * work counters, so that they never queue on a copy engine behind bulk
 * host-to-device copies of lines running on another stream */
const size_t kMaxParamUpload = 64 * 1024;
cudaError_t put_bytes(void* dst, const void* src, size_t n, cudaStream_t st);
cudaError_t zero_ints(int* p, int n, cudaStream_t st);
/* *out = the error word, which is set to zero in the same atomic step */
cudaError_t take_word(int* word, int* out, cudaStream_t st);

/* gexs_run with the kernels' error flags going to d_err (device int)
 * instead of the context's own word (NULL: the context's) */
int run_jobs(gexs_ctx* ctx, const gexs_job* jobs, int njobs, const gexs_launch_cfg* cfg,
             void* stream, int* d_err);

/* device scratch run_jobs takes from the context's pool for these jobs
 * (launch tables, per-job prep arrays, line-slice rows), in bytes */
int run_scratch_bytes(gexs_ctx* ctx, const gexs_job* jobs, int njobs, const gexs_launch_cfg* cfg,
                      size_t* bytes);

/* context accessors (gexs_capi.cu); ctx_pool may be NULL (then the
 * device's default pool serves the context) */
int ctx_device(gexs_ctx* c);
int ctx_sm_count(gexs_ctx* c);
cudaMemPool_t ctx_pool(gexs_ctx* c);
/* stream-ordered allocation from a pool (NULL: the device default); on an
 * out-of-memory the pool's unused pages are released and the call retried */
cudaError_t pool_alloc(cudaMemPool_t pool, void** p, size_t bytes, cudaStream_t s);

/* error reporting (gexs_capi.cu): thread-local message, returns status */
int set_error(int status, const std::string& msg);
int cuda_error(cudaError_t e, const char* where);

/* validation shared by the run paths */
int validate_job(const gexs_job& j, int index);

}  // namespace gexs
