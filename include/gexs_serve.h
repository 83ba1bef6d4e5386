/*
 * gexs_serve.h — request loop in front of the cross-section kernels.
 *
 * No counterpart in the reference, which computes one configured run per
 * process (main.cpp:17-42).  The server keeps line lists, their states and
 * a Q(T) table per list resident in HBM, admits requests while their output
 * grids and launch scratch fit in the memory budget, and launches every group of newly
 * admitted requests as one persistent launch on one of several streams, so
 * requests that arrive while others run overlap with them on the device
 * (continuous batching).  The Q(T) table holds the device sum over the
 * list's states (as gexs_partition) at 4096 temperatures log-spaced over
 * 10-10000 K, computed when the list is added; a request's Q(T) is the
 * 4-point Lagrange interpolation of ln Q in ln T (relative error ~1e-14 on
 * smooth state sums), so admission never waits for a reduction; a
 * temperature outside the table takes the exact device sum.
 * Each request's bins sum their lines in the same order whatever it is
 * batched with, so a result is bit-identical alone and in a mix.
 *
 * Thread safety: submit / wait / poll / stats may be called from any
 * number of threads.
 */
#ifndef GEXS_SERVE_H
#define GEXS_SERVE_H

#include <stddef.h>
#include <stdint.h>
#include "gexs_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gexs_server gexs_server;

typedef struct gexs_request {
    int32_t list_id;       /* from gexs_server_add_list                        */
    int32_t profile;       /* GEXS_DOPPLER, GEXS_GAUSSIAN, GEXS_VOIGT, _QUAD   */
    int32_t precision;     /* GEXS_FP32 or GEXS_FP64                           */
    int32_t convention;    /* GEXS_CONV_*                                      */
    int32_t quad_nodes;    /* 16 / 32 for GEXS_VOIGT_QUAD                      */
    int32_t reserved;
    double  temperature;   /* K                                                */
    double  pressure;      /* bar (PHYSICAL) or the convention's unit           */
    double  nu_start;      /* grid f_0 [cm^-1]                                 */
    double  dnu;           /* grid spacing                                     */
    int64_t grid_points;
    double  cutoff;        /* < 0: the convention's default                    */
    double  half_width;    /* Gaussian HWHM                                    */
    double  ref_temp;      /* T_ref of gamma                                   */
    double  ref_press;     /* reference-GPU pressure factor                    */
} gexs_request;

typedef struct gexs_request_info {
    double  submit_ms;     /* times on the server's clock (ms since creation)  */
    double  admit_ms;
    double  done_ms;       /* kernel completion observed                       */
    double  fetched_ms;    /* result copied to the caller                      */
    int64_t evals;         /* (line, bin) evaluations of the request          */
    int32_t batch_size;    /* requests launched together with it               */
    int32_t status;
} gexs_request_info;

/* device: CUDA device; hbm_budget: bytes the server may use for resident
 * lists plus in-flight requests (0 = 90% of the memory free when it is
 * created: memory the caller allocates afterwards is not seen, so pass a
 * budget then); max_inflight: admitted-but-unfetched requests at most
 * (0 = 256); streams: launch streams (0 = 4).  A request is charged its
 * output grid plus the scratch its launch takes from the context's memory
 * pool (launch tables, 24 B per line of prep arrays, line-slice rows), held
 * until the result is fetched; outputs come from the same pool, which keeps
 * freed pages mapped, so what the server holds stays within the budget. */
int gexs_server_create(int device, size_t hbm_budget, int max_inflight, int streams,
                       gexs_server** out);
int gexs_server_destroy(gexs_server* s);

/* Upload a line list (sorted by nu) and the states used for its Q(T)
 * (energies, degeneracies).  The arrays may be host or device memory
 * (copied with cudaMemcpyDefault).  gamma / n may be NULL (Doppler and
 * Gaussian requests only).  Fails with GEXS_ERR_ADMISSION when the list
 * does not fit in the budget. */
int gexs_server_add_list(gexs_server* s, const double* nu, const double* elow,
                         const double* aif, const int32_t* gns, const double* gamma,
                         const double* n, int64_t count, const double* state_energy,
                         const int32_t* state_g, int64_t nstates, double mean_mass,
                         int* list_id);

/* The same for a list described by a gexs_lines (host or device arrays),
 * kept resident in the format it comes in: GEXS_LINES_FP64 (44 bytes per
 * line with broadening) or GEXS_LINES_COMPACT (FP64 nu, float E'', g'A,
 * gamma and n: 24 bytes per line; requests on it compute with the widened
 * values, as gexs_run does). */
int gexs_server_add_lines(gexs_server* s, const gexs_lines* lines, const double* state_energy,
                          const int32_t* state_g, int64_t nstates, double mean_mass,
                          int* list_id);

/* Queue a request; returns at once with a ticket.  GEXS_ERR_ADMISSION if
 * the request alone can never fit in the budget. */
int gexs_server_submit(gexs_server* s, const gexs_request* r, uint64_t* ticket);

/* Wait up to timeout_ms (< 0: forever) for a request, copy its grid
 * (grid_points doubles) to h_out and release it.  GEXS_ERR_TIMEOUT leaves
 * the request in place; info may be NULL. */
int gexs_server_wait(gexs_server* s, uint64_t ticket, int timeout_ms, double* h_out,
                     gexs_request_info* info);

/* GEXS_OK when the request's result is ready, GEXS_ERR_NOT_READY if not. */
int gexs_server_poll(gexs_server* s, uint64_t ticket);

/* Q(T) of a list as the server uses it: *from_table = 1 when it comes from
 * the resident table, 0 when it is the exact device sum (temperature
 * outside the table). */
int gexs_server_partition(gexs_server* s, int list_id, double temperature, double* q,
                          int* from_table);

/* Counters: submitted, completed, admitted batches, bytes in flight. */
int gexs_server_stats(gexs_server* s, int64_t* submitted, int64_t* completed,
                      int64_t* batches, int64_t* inflight_bytes);

#ifdef __cplusplus
}
#endif
#endif /* GEXS_SERVE_H */
