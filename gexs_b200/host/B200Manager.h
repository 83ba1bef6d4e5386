/*
 * B200Manager.h — drop-in accelerator manager for the GEXS BaseProfile
 * orchestrator, the B200 replacement of GpuManager
 * (Managers/Accel/GPU/GPUManager.h:12-55).
 *
 * Call protocol (Profiles/BaseProfile.cpp:42-116,269-301), unchanged:
 *   InitializeVectors(Npoints, num_cs)   result slot per (T,P) pair
 *   TransferFreq(freq, intens, Npoints)  grid + initial slot contents
 *   InitializeConstants(...)             half width, mass, T_ref, ref_press
 *   per line chunk: TransferVectors(...) then ExecuteCrossSection(N,
 *     N_ener, start_idx, T, P, Q) once per pair; the i-th call after
 *     TransferVectors adds the chunk's cross-section into slot i
 *     (GPUManager.cpp:149,214,234,255)
 *   TransferResults(freq, intens, Npoints, I) copies slot I out.
 *
 * Differences by design: the pairs of a chunk are not launched one kernel
 * per pair on one stream per pair; they are queued and issued as one
 * persistent launch when the chunk is complete (at the next
 * TransferVectors, TransferResults, ReadyForWork or Cleanup).  Errors are
 * kept in last_status() instead of exit(-1).  The lines of a chunk must be
 * sorted by nu, as BaseProfile streams them.
 *
 * Overlapped transfer (lists of 2^21 lines or more): TransferVectors
 * copies the lines in 32 pieces on a copy stream, one event per piece, and
 * keeps every (N/8192)-th nu.  The first launch after it runs each queued
 * pair as grid segments cut at the line quantiles 1/32, 1/8, 1/4, 1/2
 * (each segment starting at a multiple of 4096 bins, the widest tile, from
 * the pair's start_idx, so the tiles are those of one launch); a segment
 * sees only the lines that can reach it and waits only for the pieces
 * holding them, and each segment has a compute stream of its own, so that
 * the long tiles of dense spectral regions start as soon as their lines
 * have arrived while later segments fill the free SMs.  The sums are bit-for-bit those of a single launch.
 * Host buffers must stay valid until TransferResults (or Cleanup), as with
 * any asynchronous copy; pageable buffers work but do not overlap.
 */
#pragma once
#include <cstddef>
#include <vector>
#ifdef GEXS_USE_REFERENCE_BASEMANAGER
/* compile inside the GEXS tree against its own Managers/BaseManager.h */
#include <BaseManager.h>
#else
#include "BaseManager.h"
#endif
#include "../../include/gexs_b200.h"

class B200Manager : public BaseManager {
public:
    /* convention: GEXS_CONV_REF_GPU reproduces GpuManager's physics,
     * GEXS_CONV_REF_CPU OpenMPManager's, GEXS_CONV_PHYSICAL the corrected
     * one.  precision: GEXS_FP64 or GEXS_FP32.  memory_bytes bounds the
     * device memory taken for lines and result slots (0: half the free
     * memory), which sets GetNtrans().  Each launch's scratch (24 B per
     * line of prep arrays, the line-slice tables) comes on top of it from
     * the context's memory pool. */
    B200Manager(ProfileType profile, int device = 0, int convention = GEXS_CONV_REF_GPU,
                int precision = GEXS_FP64, size_t memory_bytes = 0);
    ~B200Manager();

    void InitializeVectors(int Npoints);
    void InitializeVectors(int Npoints, int num_cs);
    void InitializeConstants(double half_width, double temperature, double partition,
                             double dfreq, double meanmass, double pressure = 10.0,
                             double ref_temp = 296.0, double ref_press = 1.0);
    void TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                         int* h_gns, double* h_gamma = NULL, double* h_n = NULL);
    void TransferFreq(double* h_freq, double* h_intens, int N);
    void ExecuteCrossSection(int N, int N_ener, int start_idx);
    void ExecuteCrossSection(int N, int N_ener, int start_idx, double temperature,
                             double pressure, double partition);
    void TransferResults(double* h_freq, double* h_intens, int N);
    void TransferResults(double* h_freq, double* h_intens, int N, int I);
    void Cleanup();
    bool ReadyForWork();

    int last_status() const { return status_; }
    /* add bins [lo, hi) of result slot I into h_intens[lo, hi) (waits for
     * the queued work first); B200MultiManager gathers each device's bins
     * with it */
    void AddResultRange(double* h_intens, int lo, int hi, int I);
    int quad_nodes = 16;     /* Gauss-Hermite nodes for VOIGT_QUAD */

private:
    int flush();
    int run_segmented();
    int fail(int st);
    size_t lines_below(double v) const;
    size_t lines_upto(double v) const;
    double nu_at(size_t i) const;

    int device_, convention_, precision_;
    size_t memory_bytes_;
    gexs_ctx* ctx_ = nullptr;
    void* stream_ = nullptr;
    std::vector<void*> seg_stream_;  /* one compute stream per further segment */
    void* copy_stream_ = nullptr;    /* line pieces host -> device */
    std::vector<void*> chunk_ev_;    /* piece c of the lines has arrived */
    void* done_ev_ = nullptr;        /* queued kernels are done with the lines */
    void* fork_ev_ = nullptr;
    std::vector<void*> join_ev_;     /* segment stream s has finished */
    int status_ = GEXS_OK;

    int npoints_ = 0;
    std::vector<double> h_freq_;
    std::vector<double*> d_slots_;
    double *d_nu_ = nullptr, *d_e_ = nullptr, *d_a_ = nullptr, *d_gam_ = nullptr, *d_n_ = nullptr;
    int* d_g_ = nullptr;
    size_t nlines_ = 0;
    int tasks_ = 0;
    /* overlapped transfer state */
    int nchunks_ = 0;
    size_t chunk_lines_ = 0;
    bool fresh_ = false;             /* pieces not yet all awaited by stream_ */
    std::vector<size_t> samp_idx_;   /* sampled line indices (ascending, last = N-1) */
    std::vector<double> samp_nu_;    /* nu at those indices */

    double half_width_ = 0, temperature_ = 0, partition_ = 0, dfreq_ = 0, mass_ = 0;
    double pressure_ = 0, ref_temp_ = 296.0, ref_press_ = 1.0;
    std::vector<gexs_job> pending_;
};
