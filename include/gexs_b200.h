/*
 * gexs_b200.h — C ABI of the B200 (sm_100a) cross-section engine.
 *
 * The engine computes molecular absorption cross-sections: for every line
 * (transition) it derives the intensity S(T) and a line width, then sums a
 * Doppler, Gaussian, Voigt (Humlicek W4) or Voigt-Quad (Gauss-Hermite)
 * profile onto a uniform wavenumber grid.  It is the compute path that the
 * reference GEXS reaches through its manager plug-in interface
 * (Managers/BaseManager.h:6-38): BaseProfile::PerformCrossSection
 * (Profiles/BaseProfile.cpp:100-116) hands a chunk of lines to
 * BaseManager::TransferVectors and then calls
 * BaseManager::ExecuteCrossSection once per (T, P) pair.
 *
 * Every function returns an int status: GEXS_OK (0) or a negative GEXS_ERR_*
 * code; gexs_last_error() gives a message for the calling thread.  No
 * function prints or exits (the reference prints and calls exit(-1),
 * compute/CUDA/cuda_utils.cu:8-17).  Pointers named d_* / fields documented
 * as device pointers refer to CUDA device memory of the context's device;
 * h_* are host pointers.  `stream` is a cudaStream_t passed as void*
 * (NULL = the legacy default stream).
 */
#ifndef GEXS_B200_H
#define GEXS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define GEXS_OK              0
#define GEXS_ERR_INVALID    -1  /* bad argument or unsupported combination    */
#define GEXS_ERR_OOM        -2  /* device or host allocation failed           */
#define GEXS_ERR_CUDA       -3  /* a CUDA runtime call failed                 */
#define GEXS_ERR_TIMEOUT    -4  /* a bounded wait ran out                     */
#define GEXS_ERR_NOT_READY  -5  /* asynchronous result not available yet      */
#define GEXS_ERR_ADMISSION  -6  /* request exceeds the memory budget          */
#define GEXS_ERR_SHUTDOWN   -7  /* object is shutting down                    */
#define GEXS_ERR_KERNEL     -8  /* a kernel reported an internal error flag   */

/* --------------------------------------------------------------- profiles
 * Values of GAUSSIAN, DOPPLER, VOIGT and VOIGT_QUAD equal the reference's
 * ProfileType enum (common/Input.h:10-17) so a ProfileType converts 1:1. */
#define GEXS_GAUSSIAN    0  /* fixed half-width Gaussian, bin-averaged        */
#define GEXS_DOPPLER     1  /* thermal Gaussian, bin-averaged                 */
#define GEXS_VOIGT       2  /* Humlicek W4 Faddeeva real part                 */
#define GEXS_VOIGT_QUAD  4  /* Gauss-Hermite quadrature Voigt (16/32 nodes)   */

/* precision of the profile arithmetic */
#define GEXS_FP64  0  /* plain FP64 throughout                                 */
#define GEXS_FP32  1  /* FP64 line centres/S(T)/Q(T); FP32 profile; Kahan bins */

/* which grid bins a line reaches */
#define GEXS_WINDOW_INCLUSIVE 0 /* bins j with |f_j - nu0| <= cutoff (FP64)    */
#define GEXS_WINDOW_ROUNDED   1 /* [round((nu0-cut-f_0)/dnu), round((nu0+cut-f_0)/dnu))
                                   as Managers/CPU/OpenMPManager.cpp:399-400    */

/* form of the bin-averaged erf difference (Doppler, Gaussian) in the FP64
 * form; the FP32 form always evaluates the stable form */
#define GEXS_ERF_STABLE   0 /* erfc(xm)-erfc(xp) when xm>=0: no cancellation  */
#define GEXS_ERF_LITERAL  1 /* erf(xp)-erf(xm) exactly as the reference       */

/* conventions reproduced by gexs_job_init (see that function) */
#define GEXS_CONV_PHYSICAL 0
#define GEXS_CONV_REF_CPU  1
#define GEXS_CONV_REF_GPU  2

/* ------------------------------------------------------------- line lists
 * Structure-of-arrays, exactly the arrays BaseManager::TransferVectors
 * receives (Managers/BaseManager.h:26).  Lines must be sorted by nu
 * ascending (BaseProfile.cpp:152-155 relies on the same order).  gamma and
 * n may be NULL for profiles that do not use pressure broadening.
 *
 * format GEXS_LINES_COMPACT keeps nu in FP64 and the rest in 4 bytes:
 * elow, aif, gamma and n point to float arrays (cast to these pointer
 * types), aif holding the product g' * A, and gns is unused: 24 bytes per
 * line with broadening instead of 44.  Every kernel widens the floats to
 * FP64 and computes as for the FP64 list (g' = 1, A = g'A); the per-job
 * prep arrays are required (GEXS_LAUNCH_DERIVE_ON_LOAD and
 * gexs_run_noalloc reject compact lists). */
#define GEXS_LINES_FP64    0
#define GEXS_LINES_COMPACT 1

typedef struct gexs_lines {
    const double*  nu;     /* line centre nu0 [cm^-1]                      */
    const double*  elow;   /* lower-state energy [cm^-1]                   */
    const double*  aif;    /* Einstein A coefficient [s^-1]                */
    const int32_t* gns;    /* upper-state degeneracy                       */
    const double*  gamma;  /* Lorentz half-width at T_ref, 1 atm [cm^-1]   */
    const double*  n;      /* temperature exponent of gamma                */
    int64_t        count;
    int32_t        format; /* GEXS_LINES_FP64 or GEXS_LINES_COMPACT        */
    int32_t        reserved;
} gexs_lines;

/* ------------------------------------------------------------------ jobs
 * One cross-section: one line list, one (T, P), one grid.  Bins
 * [start_idx, start_idx + n_points) of the grid f_j = nu_start + j*dnu
 * (j in [0, grid_points), evaluated without fused multiply-add, like
 * BaseProfile.cpp:17-21) are written to out[j].
 *
 * Per line (nu0 == 0 is replaced by 1e-6, OpenMPManager.cpp:392):
 *   S      = ((((s_scale*A)*g)*s_scale2)*exp(-beta*E)) * (1-exp(-beta*nu0))
 *            / ((nu0*nu0)*partition)
 *   invw   = 1/(nu0*dop_coef)           (Doppler, Voigt, Voigt-Quad)
 *          = inv_width                  (Gaussian)
 *   gammaL = (gamma * t_ratio^n) * gamma_scale
 *   y      = gammaL * invw
 *   Voigt:      term_j = ((S*K(x_j,y))*invw)*out_scale, x_j = |f_j-nu0|*invw
 *   Voigt-Quad: same with K = Gauss-Hermite K_N
 *   Doppler, Gaussian: term_j = (S*(erf(xp)-erf(xm)))*out_scale,
 *               xp = invw*(|f_j-nu0|+dnu/2), xm = invw*(|f_j-nu0|-dnu/2)
 *   out[j] = (accumulate ? out[j] : 0) + sum over lines in nu order of term_j
 */
typedef struct gexs_job {
    gexs_lines lines;        /* device pointers                                   */
    double*    out;          /* device, grid_points doubles                        */
    double     nu_start;     /* f_0 [cm^-1]                                        */
    double     dnu;          /* grid spacing [cm^-1]                               */
    int64_t    grid_points;
    int64_t    start_idx;
    int64_t    n_points;
    int32_t    profile;      /* GEXS_GAUSSIAN / DOPPLER / VOIGT / VOIGT_QUAD       */
    int32_t    precision;    /* GEXS_FP64 / GEXS_FP32                              */
    int32_t    window_rule;  /* GEXS_WINDOW_*                                      */
    int32_t    accumulate;   /* 0 overwrite, 1 add into out                        */
    int32_t    quad_nodes;   /* 16 or 32 (GEXS_VOIGT_QUAD)                         */
    int32_t    erf_form;     /* GEXS_ERF_*                                         */
    double     cutoff;       /* window half-width [cm^-1]                          */
    double     partition;    /* Q(T)                                               */
    double     beta;         /* h c / (k T) [cm]                                   */
    double     s_scale;      /* first intensity prefactor                          */
    double     s_scale2;     /* second intensity prefactor                         */
    double     dop_coef;     /* Doppler width per cm^-1 of nu0                     */
    double     inv_width;    /* Gaussian 1/width                                   */
    double     t_ratio;      /* T_ref / T                                          */
    double     gamma_scale;  /* pressure factor of gammaL                          */
    double     out_scale;    /* final multiplier of each term                      */
} gexs_job;

/* Fill a job's physics constants for one of three conventions.  Grid,
 * lines, out, precision and accumulate are left for the caller.
 *  GEXS_CONV_PHYSICAL: 1/e Doppler half-width alpha = nu0/c*sqrt(2kT N_A/m),
 *     gammaL = gamma*(T_ref/T)^n*(P[bar]/1.01325), inclusive window at
 *     `cutoff`, Voigt out_scale = 1/sqrt(pi), Doppler/Gaussian 0.5/dnu.
 *  GEXS_CONV_REF_CPU: Managers/CPU/OpenMPManager.cpp:280-323 (Doppler) and
 *     :376-426 (Voigt): HWHM Doppler scaling, no pressure factor, cutoff
 *     min(25P,100) (Doppler 100, common/defines.h:16), rounded window,
 *     1/sqrt(pi) folded into S, literal erf difference, no 0.5/dnu.
 *  GEXS_CONV_REF_GPU: compute/CUDA/cross_kernal_v2.cu:111-146,330-457 with
 *     constants of Managers/Accel/GPU/GPUManager.cpp:29-49.
 * cutoff < 0 selects the convention's default cutoff.  half_width is the
 * Gaussian HWHM (GEXS_GAUSSIAN only). */
int gexs_job_init(gexs_job* job, int convention, int profile,
                  double temperature, double pressure, double partition,
                  double mean_mass, double ref_temp, double ref_press,
                  double half_width, double cutoff,
                  double nu_start, double dnu, int64_t grid_points);

/* --------------------------------------------------------------- context */
typedef struct gexs_ctx gexs_ctx;

typedef struct gexs_launch_cfg {
    int32_t bins_per_lane;   /* 2, 4 or 8; 16 for the FP32 form only */
    int32_t warps;           /* 4 or 8 (tile = 32*bins*warps)        */
    int32_t ctas_per_sm;     /* resident CTAs per SM (0 = max)       */
    int32_t flags;           /* GEXS_LAUNCH_*                        */
    int32_t wait_spins;      /* attempts of each bounded wait of the FP32
                                Voigt pipeline before it gives up and
                                flags GEXS_ERR_KERNEL (0 = 2^21, about
                                0.5 s of back-off per wait)           */
} gexs_launch_cfg;

/* derive S(T), width and y of every line in the tile loader instead of
 * once per job by a prep kernel (no per-job scratch of 24 B per line) */
#define GEXS_LAUNCH_DERIVE_ON_LOAD 1
/* FP32 Voigt, 512-bin tiles (4 bins x 4 warps, 2 x 8): hand lines from the
 * producer warps to the consumers in stages of 256 instead of 128 (two
 * stages in the ring instead of four).  Fewer hand-overs and Kahan folds,
 * less slack between producers and consumers; gexs_autotune tries both. */
#define GEXS_LAUNCH_LONG_STAGES    2
/* Work-item order of a launch with several jobs.  By default the items go
 * tile-major: tile 0 of every job, then tile 1 of every job, and so on
 * (jobs with fewer tiles drop out as they end), so the jobs of a (T, P)
 * batch over one line list read a tile's lines from HBM once and from L2
 * for the other pairs while the CTAs that run them are resident together.
 * This flag restores job-major order (all tiles of job 0, then job 1, ...).
 * A tile's sums do not depend on the order: results are bitwise equal.
 * gexs_autotune tries both for several jobs. */
#define GEXS_LAUNCH_JOB_MAJOR      4

/* A context owns a stream-ordered memory pool on its device for the
 * launch tables and per-line prep arrays (24 B per line) of gexs_run.  The
 * pool keeps its memory between calls (no remapping per call) and never
 * makes an allocation on one stream wait for a free on another, so
 * gexs_run calls on different streams overlap; its memory goes back to the
 * device at gexs_ctx_destroy. */
int         gexs_ctx_create(int device, gexs_ctx** out);
int         gexs_ctx_destroy(gexs_ctx* ctx);
const char* gexs_status_string(int status);
const char* gexs_last_error(void);
int         gexs_version(void);
/* Testing: refuse the next n stream-ordered device allocations of the
 * library (launch scratch, server outputs) with an out-of-memory status,
 * without calling CUDA, so that callers' out-of-memory paths can be
 * exercised with no real memory pressure; 0 turns it off. */
int         gexs_debug_fail_allocs(int n);
/* Testing: the tile-major order tables a launch of njobs jobs with these
 * tile counts uses (GEXS_LAUNCH_JOB_MAJOR unset), written to out
 * (3 njobs + 1 ints: F[njobs + 1] first item of each segment, R[njobs]
 * first tile row of each segment, P[njobs] job of each rank; in segment s
 * the jobs P[0 .. njobs - s) are active, one tile of each per row).  Host
 * only; no device work. */
int         gexs_debug_tile_order(const int32_t* tiles, int njobs, int32_t* out);

/* Run njobs jobs (host array of descriptors holding device pointers) on
 * `stream`: one persistent launch over every (job, tile) work item.
 * cfg NULL = the context's tuned default for the jobs' profile/precision.
 * Asynchronous; kernel error flags are checked by gexs_ctx_check. */
int gexs_run(gexs_ctx* ctx, const gexs_job* jobs, int njobs,
             const gexs_launch_cfg* cfg, void* stream);

/* Synchronise `stream`, then read and clear the context's kernel error
 * word: GEXS_ERR_KERNEL if a kernel of an earlier gexs_run on this context
 * flagged an error (a bounded wait that ran out, GEXS_KERR_* bits in the
 * message) since the last check, else GEXS_OK.  The word is shared by
 * every stream of the context; the read and the clear are one atomic
 * exchange on the device, so no flag raised meanwhile is lost. */
int gexs_ctx_check(gexs_ctx* ctx, void* stream);

/* Exact number of (line, bin) profile evaluations of each job (the window
 * rule applied to every line): counts[i] for jobs[i]. Synchronous. */
int gexs_count_evals(gexs_ctx* ctx, const gexs_job* jobs, int njobs,
                     int64_t* h_counts);

/* --------------------------------------------- run without allocating
 * No counterpart in the reference.  For callers that must not allocate
 * device memory while they run: for instance a plug-in inside a host
 * program that keeps all of the GPU's memory in its own pool, or a
 * latency-sensitive loop in which a device allocation could stall other
 * streams or fail.  gexs_run takes its launch tables and work counter from
 * cudaMallocAsync; this variant keeps them in a fixed array inside the
 * library's device image (GEXS_NOALLOC_SCRATCH_BYTES on every GPU that
 * loads the library, held until the process exits) and calls no
 * cudaMalloc, cudaFree or other allocating routine.
 *  - The caller still provides the line arrays and the output grids.
 *  - At most GEXS_NOALLOC_MAX_JOBS jobs per call, all of one profile class
 *    and precision; larger or mixed calls return GEXS_ERR_INVALID.
 *  - Runs on the calling thread's current device.  The first call on a
 *    device looks up the array's device address (cudaGetSymbolAddress);
 *    make that first call before any stream capture on that device.
 *  - Every call on a device shares the one array and it keeps the last
 *    call's contents (each call resets the work counter and the error
 *    word): calls whose work overlaps on the GPU, from any stream or
 *    thread, race and must be serialised by the caller.
 *  - Lines are derived as they are loaded (no 24-byte-per-line prep
 *    arrays) and tiles are never cut into line slices (their tables grow
 *    with the grid), so a dense band, where a few tiles hold most of the
 *    lines, runs on fewer SMs than with gexs_run: up to several times
 *    slower there; elsewhere the two run alike.
 *  - Kernel errors (a bounded wait that ran out) are not returned by this
 *    call, which does not wait for the kernels: read them with
 *    gexs_noalloc_status after the call.
 * cfg NULL = gexs_run's default shape (4 bins per lane; 4 warps for FP32,
 * 8 for FP64). */
#define GEXS_NOALLOC_MAX_JOBS      64
#define GEXS_NOALLOC_SCRATCH_BYTES 16384
int gexs_run_noalloc(const gexs_job* jobs, int njobs, const gexs_launch_cfg* cfg,
                     void* stream);
/* Synchronise `stream` and read the error word of the last
 * gexs_run_noalloc on the current device into *flags (GEXS_KERR_* bits):
 * GEXS_OK when it is zero, GEXS_ERR_KERNEL when a kernel flagged an error.
 * A copy of four bytes to the host; allocates nothing.  The word is
 * cleared by the next gexs_run_noalloc, not by this call. */
#define GEXS_KERR_PIPELINE 1   /* a bounded wait of the FP32 Voigt pipeline ran out */
#define GEXS_KERR_SLICES   2   /* line-slice tables overflowed (gexs_run only)      */
int gexs_noalloc_status(void* stream, int* flags);

/* --------------------------------------------------------- ExoMol ingest
 * The reader layer of the reference (Readers/Exomol/ExomolStateReader.cpp,
 * Readers/Exomol/exomol_functions.cpp) on the GPU: text is copied to the
 * device once and parsed there, one thread per record, with the
 * reference's number semantics (see gexs_ingest.cu); results are device
 * tables owned by the caller (free with the *_free functions).
 *  - states: one per text line, in line order (exomol_functions.cpp:8-48:
 *    id/gns/J by strtol base 0, energy by strtod; index = line number);
 *    a line longer than 1022 bytes is an error (the reference's fgets
 *    buffer would split it).
 *  - transitions: per non-empty line `id_upper id_lower A [more fields]`
 *    (ExomolStateReader.cpp:132-172): nu = E_u - E_l, elow = E_l,
 *    gns = g_u; ids must lie in [1, states->count].
 *  - broadening: GEXS_BROAD_DEFAULTS gives every line default_gamma and
 *    default_n, which is what the reference's lookup yields
 *    (ExomolStateReader.cpp:21 keeps the failed key, no entry matches);
 *    GEXS_BROAD_BY_J uses "a1 gamma n J'' J'" entries, then "a0 gamma n J''",
 *    then the defaults.  A missing broadener file means defaults.
 *  - sort_by_nu != 0: lines sorted by nu (stable), as the cross-section
 *    path requires; 0 keeps file order. */
#define GEXS_BROAD_DEFAULTS 0
#define GEXS_BROAD_BY_J     1

typedef struct gexs_state_table {
    double*  energy;   /* device, cm^-1 */
    int32_t* g;        /* device, total degeneracy */
    int32_t* J;        /* device */
    int64_t  count;
} gexs_state_table;

typedef struct gexs_line_table {   /* device arrays, same meaning as gexs_lines */
    double*  nu;
    double*  elow;
    double*  aif;
    int32_t* gns;
    double*  gamma;
    double*  n;
    int64_t  count;
} gexs_line_table;

int gexs_exomol_parse_states(gexs_ctx* ctx, const char* h_text, int64_t nbytes,
                             gexs_state_table* out);
int gexs_exomol_parse_trans(gexs_ctx* ctx, const gexs_state_table* states, const char* h_text,
                            int64_t nbytes, const char* h_broad, int64_t broad_nbytes,
                            int broad_mode, double default_gamma, double default_n,
                            int sort_by_nu, gexs_line_table* out);
/* read the files (broad_path may be NULL) and parse both */
int gexs_exomol_load(gexs_ctx* ctx, const char* states_path, const char* trans_path,
                     const char* broad_path, int broad_mode, double default_gamma,
                     double default_n, int sort_by_nu, gexs_state_table* states_out,
                     gexs_line_table* lines_out);
/* HITRAN .par text (Readers/HITRAN/HITRANStateReader.cpp:137-250) parsed on
 * the GPU, one thread per 160-column record: nu, S, A, gamma_air,
 * gamma_self, E'', n_air and g' by atof of their columns; gamma =
 * (gamma_air*air_mixture + gamma_self*(1-air_mixture))*pressure (:218);
 * where A == 0, A = S*8*pi*c*Q(296)*nu^2/(exp(-c2 E''/296)*(1-exp(-c2
 * nu/296))) and g' = 1 (:222-247).  ref_partition_296 <= 0 takes Q(296)
 * from TIPS-2011 (gexs_tips_2011) for the molecule and isotopologue in
 * columns 1-2 and 3 of the first record, as the reference does (:88-95);
 * a positive value is used as given. */
int gexs_hitran_parse(gexs_ctx* ctx, const char* h_text, int64_t nbytes, double pressure,
                      double air_mixture, double ref_partition_296, int sort_by_nu,
                      gexs_line_table* out);

/* TIPS-2011 total internal partition sum of a HITRAN molecule (HITRAN
 * number) and isotopologue (its 1-based index in the HITRAN file) at
 * `temperature` K: the reference's BD_TIPS_2011
 * (Readers/HITRAN/BD_TIPS_2011_v1p0.for:5-345, called through
 * bd_tips_2011_ at Readers/HITRAN/HITRANStateReader.cpp:62,95,128), its
 * tables (Q at 60, 85, ..., 3010 K) interpolated by the 3/4-point Lagrange
 * rule of its AtoB (:5830-5920).  *gi gets the state-independent
 * degeneracy.  Outside 70-3000 K: *q = -1 and GEXS_ERR_INVALID (the
 * reference returns -1 with a message); molecules 34 and 39: gi = 0, Q = 0
 * and GEXS_OK, as the reference.  Host computation, no device. */
int gexs_tips_2011(int molecule, int isotopologue, double temperature, double* gi, double* q);

/* copy a table into caller-owned device arrays of `count` elements */
int gexs_state_table_export(const gexs_state_table* t, double* d_energy, int32_t* d_g,
                            int32_t* d_J);
int gexs_line_table_export(const gexs_line_table* t, double* d_nu, double* d_elow, double* d_aif,
                           int32_t* d_gns, double* d_gamma, double* d_n);
int gexs_state_table_free(gexs_state_table* t);
int gexs_line_table_free(gexs_line_table* t);

/* ----------------------------------------------------------------- output
 * One (T, P) cross-section to a file (Profiles/BaseProfile.cpp:269-301
 * prints every bin with printf on one thread).
 *  GEXS_OUT_TEXT: exactly the reference's text, "-------T=%12.6f K--------
 *    P=%12.6f atm---------" and a blank line, then "[%i] %12.6f %13.8E" per
 *    bin (index, nu_start + double(j)*dnu, sigma_j), then a blank line;
 *    formatted on nthreads host threads (0 = all) and written in order.
 *  GEXS_OUT_BINARY: a 64-byte header {char magic[8] = "GEXSSIG1"; int64 n;
 *    double nu_start, dnu, temperature, pressure; int32 index, reserved;
 *    int64 pad} then n float64 values.
 * append != 0 adds to the file (one file per run, as the reference's stdout).
 * sigma may be host or device memory. */
#define GEXS_OUT_BINARY 0
#define GEXS_OUT_TEXT   1
int gexs_write_sigma(const char* path, int format, int append, int index, double temperature,
                     double pressure, double nu_start, double dnu, int64_t n,
                     const double* sigma, int nthreads);

/* ------------------------------------------------------ batched launches
 * A batch owns its device job table and work-item table; launching it is
 * a memset of the work counter plus one persistent kernel per group of
 * jobs (FP32 Voigt groups: a second memset and the core kernel), which can
 * be captured once into a CUDA graph and replayed. */
typedef struct gexs_batch gexs_batch;

int gexs_batch_create(gexs_ctx* ctx, const gexs_job* jobs, int njobs,
                      const gexs_launch_cfg* cfg, gexs_batch** out);
int gexs_batch_launch(gexs_batch* b, void* stream);
int gexs_batch_capture(gexs_batch* b, void* stream);  /* build the graph   */
int gexs_batch_replay(gexs_batch* b, void* stream);   /* launch the graph  */
int gexs_batch_destroy(gexs_batch* b);

/* Pick the launch for these jobs by timing each candidate (CUDA events) on
 * the jobs themselves: bins_per_lane x warps (the tile width and CTA
 * shape), the ring's stage length where it applies (GEXS_LAUNCH_LONG_STAGES)
 * and, for several jobs, the item order on the best shape
 * (GEXS_LAUNCH_JOB_MAJOR or the tile-major default).  Writes the winner to
 * *best and records it as the context default for the jobs' profile and
 * precision; h_ms (may be NULL) gets the winner's time. */
int gexs_autotune(gexs_ctx* ctx, const gexs_job* jobs, int njobs,
                  gexs_launch_cfg* best, float* h_ms);

/* ------------------------------------------------------ partition function
 * Q(T) = sum_s g_s exp(-c2 E_s / T) in FP64 for nt temperatures
 * (Readers/Exomol/exomol_functions.cpp:50-73), states resident on device. */
int gexs_partition(gexs_ctx* ctx, const double* d_energy, const int32_t* d_g,
                   int64_t nstates, const double* h_temps, int nt,
                   double* h_q);

/* ------------------------------------------------------------ sharding
 * Split bins [start_idx, start_idx + n_points) of a grid (nu_start, dnu)
 * into nshards ranges bounds[r] .. bounds[r+1] (nshards + 1 entries) with
 * about equal (line, bin) evaluations - a bin's work is the number of
 * lines within `reach` of it, sampled every 256th bin from the sorted
 * centres h_nu (host) - interior cuts on multiples of `align` bins from
 * start_idx (4096 makes every shard's tiles the tiles of one unsplit
 * launch), and give each range the index range [line_lo[r], line_hi[r]) of
 * the lines within `reach` of it.  Host computation.  No counterpart in
 * the reference (its multi-GPU manager splits by line chunks,
 * Managers/Accel/GPU/MultiGPUManager.cpp:59-63). */
int gexs_shard_plan(const double* h_nu, int64_t nlines, double nu_start, double dnu,
                    int64_t start_idx, int64_t n_points, double reach, int align, int nshards,
                    int64_t* bounds, int64_t* line_lo, int64_t* line_hi);

/* ------------------------------------------------------------ calibration
 * Measured FP32 FMA throughput of `device` in TFLOP/s (2 FLOP per FMA):
 * the roofline denominator of the FP32-profile kernels, which are bound by
 * FP32/SFU issue rather than HBM or tensor cores.  No reference
 * counterpart. */
int gexs_probe_fp32_tflops(int device, double* tflops);
/* Measured FP64 FMA throughput in TFLOP/s: the roofline denominator of the
 * plain FP64 form.  No reference counterpart. */
int gexs_probe_fp64_tflops(int device, double* tflops);
/* Measured rate of rcp.approx.f32 (one MUFU reciprocal) in 1e9/s: region I
 * of the FP32 Voigt form takes one per evaluation, so this caps its
 * evaluations/s.  No reference counterpart. */
int gexs_probe_rcp_gops(int device, double* gops);

/* ------------------------------------------------------------ manager ABI
 * Flat C view of the drop-in manager (B200Manager, a BaseManager subclass):
 * one function per BaseManager virtual (Managers/BaseManager.h:22-35) so an
 * FFI caller can drive it exactly as BaseProfile drives a manager. */
typedef struct gexs_manager gexs_manager;

int gexs_manager_create(int profile, int device, int convention,
                        int precision, size_t memory_bytes,
                        gexs_manager** out);
/* The same manager over several GPUs: the drop-in beside the reference's
 * MultiGpuManager (Managers/Accel/GPU/MultiGPUManager.cpp, the manager
 * Profiles/BaseProfile.cpp:61 creates).  Each line chunk is split by grid
 * bins into one range per device (gexs_shard_plan), each device receives
 * only the lines that can reach its range and computes exactly the sums a
 * single launch computes for those bins; transfer_results adds the initial
 * grid once and every device's bins into h_intens (the reference adds each
 * GPU's full grid).  devices may repeat a device (several shards on one
 * GPU); ndev 0 = every visible device.  memory_bytes is per device. */
int gexs_manager_create_multi(int profile, const int* devices, int ndev, int convention,
                              int precision, size_t memory_bytes, gexs_manager** out);
int gexs_manager_destroy(gexs_manager* m);
/* BaseManager::InitializeVectors(int Npoints, int num_cs) */
int gexs_manager_initialize_vectors(gexs_manager* m, int npoints, int num_cs);
/* BaseManager::InitializeConstants(...) */
int gexs_manager_initialize_constants(gexs_manager* m, double half_width,
        double temperature, double partition, double dfreq, double meanmass,
        double pressure, double ref_temp, double ref_press);
/* BaseManager::TransferFreq(double* h_freq, double* h_intens, int N) */
int gexs_manager_transfer_freq(gexs_manager* m, const double* h_freq,
                               const double* h_intens, int n);
/* BaseManager::TransferVectors(...) */
int gexs_manager_transfer_vectors(gexs_manager* m, size_t nener,
        const double* h_energies, const double* h_nu, const double* h_aif,
        const int* h_gns, const double* h_gamma, const double* h_n);
/* BaseManager::ExecuteCrossSection(N, N_ener, start_idx, T, P, Q) */
int gexs_manager_execute(gexs_manager* m, int n, int n_ener, int start_idx,
                         double temperature, double pressure,
                         double partition);
/* BaseManager::TransferResults(h_freq, h_intens, N, I) */
int gexs_manager_transfer_results(gexs_manager* m, double* h_freq,
                                  double* h_intens, int n, int i);
/* BaseManager::GetNtrans() and ReadyForWork() */
int gexs_manager_ntrans(gexs_manager* m, size_t* out);
int gexs_manager_ready(gexs_manager* m, int* ready);

#ifdef __cplusplus
}
#endif
#endif /* GEXS_B200_H */
