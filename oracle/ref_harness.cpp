/*
 * ref_harness.cpp — drives the reference's own CPU path, compiled unmodified
 * from the GEXS sources, for parity pinning and the CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY (built by oracle/Makefile into oracle/_ref/).
 *
 * The reference reaches Managers/CPU only through HybridManager, which cannot
 * be instantiated (Managers/Hybrid/HybridManager.h:26 overrides nothing), so
 * this harness calls OpenMPManager's workers directly:
 *   - OpenMPManager::ComputeVoigtTP (Managers/CPU/OpenMPManager.cpp:376-426)
 *     on its own std::threads, one per requested thread, after zeroing the
 *     result slot that InitializeVectors leaves uninitialised (:62-66);
 *   - OpenMPManager::ComputeDoppler (:280-323), whose per-thread grids are
 *     never merged by the reference, so the harness sums them in thread order;
 *   - compute_partition (Readers/Exomol/exomol_functions.cpp:50-73);
 *   - humlic (compute/CPU/profiles.cpp:11-44).
 * The reference prints progress to stdout; the harness routes stdout to
 * /dev/null around each call so callers keep a clean stdout.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <unistd.h>
#include <fcntl.h>
/* Standard headers first: the access shim below must only touch the
 * reference's own classes. */
#include <cmath>
#include <complex>
#include <condition_variable>
#include <fstream>
#include <iostream>
#include <map>
#include <mutex>
#include <queue>
#include <sstream>
#include <string>

#define private public
#define protected public
#include "OpenMPManager.h"
#undef private
#undef protected
#include "exomol_objects.h"
#include "exomol_functions.h"
#include "profiles.h"

namespace {

struct Quiet {
    int saved;
    Quiet() {
        fflush(stdout);
        saved = dup(1);
        int dn = open("/dev/null", O_WRONLY);
        if (dn >= 0) { dup2(dn, 1); close(dn); }
    }
    ~Quiet() {
        fflush(stdout);
        if (saved >= 0) { dup2(saved, 1); close(saved); }
    }
};

/* Memory figure that makes InitializeVectors size N_trans >= nlines:
 * the manager halves its budget (OpenMPManager.cpp:9) and subtracts the
 * grids before dividing by the per-line footprint (:81-85). */
size_t budget(int npoints, int nthreads, size_t nlines)
{
    size_t grids = (size_t)npoints * sizeof(double) * (size_t)(2 + nthreads);
    size_t per_line = 5 * sizeof(double) + sizeof(int);
    return 2 * (grids + per_line * (nlines + 16)) + 4096;
}

void release(OpenMPManager* m, int nthreads, bool voigt)
{
    if (m->master_thread) { m->master_thread->join(); delete m->master_thread; }
    delete[] m->g_freq;
    for (double* p : m->g_tp_intens) delete[] p;
    for (int i = 0; i < nthreads; ++i) delete[] m->t_intens[i];
    delete[] m->t_intens;
    delete[] m->threads_done;
    delete[] m->g_energies; delete[] m->g_nu; delete[] m->g_aif; delete[] m->g_gns;
    if (voigt) { delete[] m->g_gamma; delete[] m->g_n; }
    delete m;
}

}  // namespace

extern "C" {

/* Reference Voigt for one (T, P) on the whole grid (start_idx 0).
 * freq: npoints grid frequencies; out: npoints results. */
int ref_voigt_tp(int npoints, const double* freq, int nlines, const double* nu,
                 const double* elow, const double* aif, const int* gns,
                 const double* gamma, const double* nexp, double temperature,
                 double pressure, double partition, double mean_mass,
                 double ref_temp, double dfreq, int nthreads, double* out)
{
    if (nthreads < 1) nthreads = 1;
    Quiet q;
    OpenMPManager* m = new OpenMPManager(VOIGT, nthreads, budget(npoints, nthreads, nlines));
    m->InitializeVectors(npoints, 1);
    if (m->N_trans < (size_t)nlines) { release(m, nthreads, true); return -1; }
    m->InitializeConstants(0.0, temperature, partition, dfreq, mean_mass, pressure, ref_temp, 1.0);
    std::vector<double> zeros((size_t)npoints, 0.0);
    m->TransferFreq(const_cast<double*>(freq), zeros.data(), npoints);
    m->TransferVectors((size_t)nlines, const_cast<double*>(elow), const_cast<double*>(nu),
                       const_cast<double*>(aif), const_cast<int*>(gns),
                       const_cast<double*>(gamma), const_cast<double*>(nexp));
    std::memset(m->g_tp_intens[0], 0, sizeof(double) * (size_t)npoints);
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i)
        th.emplace_back(&OpenMPManager::ComputeVoigtTP, m, i, npoints, nlines, 0, 0,
                        temperature, pressure, partition);
    for (auto& t : th) t.join();
    std::memcpy(out, m->g_tp_intens[0], sizeof(double) * (size_t)npoints);
    release(m, nthreads, true);
    return 0;
}

/* Reference Doppler (deprecated single-temperature path) on the whole grid. */
int ref_doppler(int npoints, const double* freq, int nlines, const double* nu,
                const double* elow, const double* aif, const int* gns,
                double temperature, double partition, double mean_mass,
                double dfreq, int nthreads, double* out)
{
    if (nthreads < 1) nthreads = 1;
    Quiet q;
    OpenMPManager* m = new OpenMPManager(DOPPLER, nthreads, budget(npoints, nthreads, nlines));
    m->InitializeVectors(npoints, 1);
    if (m->N_trans < (size_t)nlines) { release(m, nthreads, false); return -1; }
    m->InitializeConstants(0.0, temperature, partition, dfreq, mean_mass, 1.0, 296.0, 1.0);
    std::vector<double> zeros((size_t)npoints, 0.0);
    m->TransferFreq(const_cast<double*>(freq), zeros.data(), npoints);
    m->TransferVectors((size_t)nlines, const_cast<double*>(elow), const_cast<double*>(nu),
                       const_cast<double*>(aif), const_cast<int*>(gns), NULL, NULL);
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i)
        th.emplace_back(&OpenMPManager::ComputeDoppler, m, i, npoints, nlines, 0);
    for (auto& t : th) t.join();
    for (int j = 0; j < npoints; ++j) {
        double s = 0.0;
        for (int i = 0; i < nthreads; ++i) s += m->t_intens[i][j];
        out[j] = s;
    }
    release(m, nthreads, false);
    return 0;
}

double ref_partition(int n, const double* energy, const int* g, double temperature)
{
    Quiet q;
    exomol_states st;
    st.N = n;
    st.states = new state[n];
    for (int i = 0; i < n; ++i) {
        st.states[i].id = i;
        st.states[i].energy = energy[i];
        st.states[i].gns = g[i];
        st.states[i].J = 0;
    }
    double qv = compute_partition(&st, temperature);
    delete[] st.states;
    return qv;
}

double ref_humlic(double x, double y) { return humlic(x, y); }

}  // extern "C"
