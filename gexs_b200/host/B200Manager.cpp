/*
 * B200Manager.cpp — BaseManager implementation over the gexs C ABI, and the
 * flat gexs_manager_* C wrappers declared in include/gexs_b200.h.
 */
#include "B200Manager.h"

#include <cmath>
#include <cstring>
#include <string>
#include <cuda_runtime.h>

B200Manager::B200Manager(ProfileType profile, int device, int convention, int precision,
                         size_t memory_bytes)
    : BaseManager(profile), device_(device), convention_(convention), precision_(precision),
      memory_bytes_(memory_bytes)
{
    int st = gexs_ctx_create(device, &ctx_);
    if (st) { fail(st); return; }
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) { fail(GEXS_ERR_CUDA); return; }
    stream_ = (void*)s;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    if (memory_bytes_ == 0) memory_bytes_ = fr / 2;
    InitializeMemory(memory_bytes_);
}

B200Manager::~B200Manager()
{
    Cleanup();
    if (stream_) cudaStreamDestroy((cudaStream_t)stream_);
    gexs_ctx_destroy(ctx_);
}

int B200Manager::fail(int st)
{
    if (status_ == GEXS_OK) status_ = st;
    return st;
}

void B200Manager::InitializeVectors(int Npoints) { InitializeVectors(Npoints, 1); }

/* GPUManager.cpp:84-132: grid, num_cs result slots, then as many lines as
 * the remaining budget holds. */
void B200Manager::InitializeVectors(int Npoints, int num_cs)
{
    if (status_ || Npoints <= 0 || num_cs <= 0) { fail(GEXS_ERR_INVALID); return; }
    cudaSetDevice(device_);
    npoints_ = Npoints;
    h_freq_.assign((size_t)Npoints, 0.0);
    for (int i = 0; i < num_cs; ++i) {
        double* d = nullptr;
        if (cudaMalloc(&d, sizeof(double) * (size_t)Npoints) != cudaSuccess) { fail(GEXS_ERR_OOM); return; }
        cudaMemset(d, 0, sizeof(double) * (size_t)Npoints);
        d_slots_.push_back(d);
        TrackMemory(sizeof(double) * (size_t)Npoints);
    }
    bool press = profile == VOIGT || profile == VOIGT_QUAD;
    size_t per_line = 3 * sizeof(double) + sizeof(int) + (press ? 2 * sizeof(double) : 0);
    N_trans = GetAvailableMemory() / per_line;
    if (N_trans == 0) { fail(GEXS_ERR_OOM); return; }
    bool ok = cudaMalloc(&d_nu_, sizeof(double) * N_trans) == cudaSuccess &&
              cudaMalloc(&d_e_, sizeof(double) * N_trans) == cudaSuccess &&
              cudaMalloc(&d_a_, sizeof(double) * N_trans) == cudaSuccess &&
              cudaMalloc(&d_g_, sizeof(int) * N_trans) == cudaSuccess;
    if (ok && press)
        ok = cudaMalloc(&d_gam_, sizeof(double) * N_trans) == cudaSuccess &&
             cudaMalloc(&d_n_, sizeof(double) * N_trans) == cudaSuccess;
    if (!ok) { fail(GEXS_ERR_OOM); return; }
    TrackMemory(per_line * N_trans);
}

void B200Manager::InitializeConstants(double half_width, double temperature, double partition,
                                      double dfreq, double meanmass, double pressure,
                                      double ref_temp, double ref_press)
{
    half_width_ = half_width; temperature_ = temperature; partition_ = partition;
    dfreq_ = dfreq; mass_ = meanmass; pressure_ = pressure;
    ref_temp_ = ref_temp; ref_press_ = ref_press;
}

/* GPUManager.cpp:134-145: keep the grid and seed every slot with h_intens.
 * The kernels regenerate f_j = f_0 + j*dfreq, so the grid must be that
 * uniform grid (BaseProfile.cpp:17-21 builds exactly that). */
void B200Manager::TransferFreq(double* h_freq, double* h_intens, int N)
{
    if (status_) return;
    if (N != npoints_ || !h_freq || !h_intens) { fail(GEXS_ERR_INVALID); return; }
    cudaSetDevice(device_);
    std::memcpy(h_freq_.data(), h_freq, sizeof(double) * (size_t)N);
    for (double* d : d_slots_)
        if (cudaMemcpyAsync(d, h_intens, sizeof(double) * (size_t)N, cudaMemcpyHostToDevice,
                            (cudaStream_t)stream_) != cudaSuccess) { fail(GEXS_ERR_CUDA); return; }
}

void B200Manager::TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                                  int* h_gns, double* h_gamma, double* h_n)
{
    if (status_) return;
    if (flush()) return;
    if (Nener > N_trans) { fail(GEXS_ERR_INVALID); return; }
    cudaSetDevice(device_);
    cudaStream_t s = (cudaStream_t)stream_;
    tasks_ = 0;
    nlines_ = Nener;
    bool ok = cudaMemcpyAsync(d_e_, h_energies, sizeof(double) * Nener, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(d_nu_, h_nu, sizeof(double) * Nener, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(d_a_, h_aif, sizeof(double) * Nener, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(d_g_, h_gns, sizeof(int) * Nener, cudaMemcpyHostToDevice, s) == cudaSuccess;
    if (ok && h_gamma && h_n && d_gam_ && d_n_)
        ok = cudaMemcpyAsync(d_gam_, h_gamma, sizeof(double) * Nener, cudaMemcpyHostToDevice, s) == cudaSuccess &&
             cudaMemcpyAsync(d_n_, h_n, sizeof(double) * Nener, cudaMemcpyHostToDevice, s) == cudaSuccess;
    if (!ok) fail(GEXS_ERR_CUDA);
}

void B200Manager::ExecuteCrossSection(int, int, int)
{
    /* deprecated in the reference too (GPUManager.cpp:168-184) */
    fail(GEXS_ERR_INVALID);
}

void B200Manager::ExecuteCrossSection(int N, int N_ener, int start_idx, double temperature,
                                      double pressure, double partition)
{
    if (status_) return;
    if (tasks_ >= (int)d_slots_.size() || N < 0 || start_idx < 0 || start_idx + N > npoints_ ||
        N_ener < 0 || (size_t)N_ener > nlines_) { fail(GEXS_ERR_INVALID); return; }
    gexs_job j;
    int gp = profile == VOIGT_QUAD ? GEXS_VOIGT_QUAD : (int)profile;
    int st = gexs_job_init(&j, convention_, gp, temperature, pressure, partition, mass_,
                           ref_temp_, ref_press_, half_width_, -1.0, h_freq_[0], dfreq_,
                           npoints_);
    if (st) { fail(st); return; }
    j.quad_nodes = quad_nodes;
    j.precision = precision_;
    j.accumulate = 1;
    j.start_idx = start_idx;
    j.n_points = N;
    j.out = d_slots_[tasks_];
    j.lines.nu = d_nu_; j.lines.elow = d_e_; j.lines.aif = d_a_; j.lines.gns = d_g_;
    j.lines.gamma = d_gam_; j.lines.n = d_n_; j.lines.count = N_ener;
    pending_.push_back(j);
    ++tasks_;
}

int B200Manager::flush()
{
    if (pending_.empty()) return status_;
    int st = gexs_run(ctx_, pending_.data(), (int)pending_.size(), nullptr, stream_);
    pending_.clear();
    if (st) return fail(st);
    return GEXS_OK;
}

void B200Manager::TransferResults(double* h_freq, double* h_intens, int N)
{
    TransferResults(h_freq, h_intens, N, 0);
}

/* GPUManager.cpp:280-287: wait, then copy grid and slot I out */
void B200Manager::TransferResults(double* h_freq, double* h_intens, int N, int I)
{
    if (status_) return;
    if (I < 0 || I >= (int)d_slots_.size() || N > npoints_ || N < 0) { fail(GEXS_ERR_INVALID); return; }
    if (flush()) return;
    cudaSetDevice(device_);
    int st = gexs_ctx_check(ctx_, stream_);
    if (st) { fail(st); return; }
    if (h_freq) std::memcpy(h_freq, h_freq_.data(), sizeof(double) * (size_t)N);
    if (cudaMemcpy(h_intens, d_slots_[I], sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost) != cudaSuccess)
        fail(GEXS_ERR_CUDA);
}

void B200Manager::Cleanup()
{
    if (ctx_) { flush(); cudaStreamSynchronize((cudaStream_t)stream_); }
    cudaSetDevice(device_);
    for (double* d : d_slots_) cudaFree(d);
    d_slots_.clear();
    cudaFree(d_nu_); cudaFree(d_e_); cudaFree(d_a_); cudaFree(d_g_);
    cudaFree(d_gam_); cudaFree(d_n_);
    d_nu_ = d_e_ = d_a_ = d_gam_ = d_n_ = nullptr; d_g_ = nullptr;
}

/* GPUManager.cpp:303-309: ready while slots remain, else when idle */
bool B200Manager::ReadyForWork()
{
    if (tasks_ < (int)d_slots_.size()) return true;
    flush();
    return cudaStreamQuery((cudaStream_t)stream_) == cudaSuccess;
}

/* ----------------------------------------------------------- C wrappers */
struct gexs_manager { B200Manager* m; };

static int mstat(gexs_manager* h)
{
    int st = h->m->last_status();
    return st;
}

extern "C" {

int gexs_manager_create(int profile, int device, int convention, int precision,
                        size_t memory_bytes, gexs_manager** out)
{
    if (!out) return GEXS_ERR_INVALID;
    *out = nullptr;
    if (profile != GEXS_GAUSSIAN && profile != GEXS_DOPPLER && profile != GEXS_VOIGT &&
        profile != GEXS_VOIGT_QUAD) return GEXS_ERR_INVALID;
    gexs_manager* h = new gexs_manager();
    h->m = new B200Manager((ProfileType)profile, device, convention, precision, memory_bytes);
    int st = h->m->last_status();
    if (st) { delete h->m; delete h; return st; }
    *out = h;
    return GEXS_OK;
}

int gexs_manager_destroy(gexs_manager* h)
{
    if (!h) return GEXS_OK;
    delete h->m;
    delete h;
    return GEXS_OK;
}

int gexs_manager_initialize_vectors(gexs_manager* h, int npoints, int num_cs)
{
    if (!h) return GEXS_ERR_INVALID;
    h->m->InitializeVectors(npoints, num_cs);
    return mstat(h);
}

int gexs_manager_initialize_constants(gexs_manager* h, double half_width, double temperature,
                                      double partition, double dfreq, double meanmass,
                                      double pressure, double ref_temp, double ref_press)
{
    if (!h) return GEXS_ERR_INVALID;
    h->m->InitializeConstants(half_width, temperature, partition, dfreq, meanmass, pressure,
                              ref_temp, ref_press);
    return mstat(h);
}

int gexs_manager_transfer_freq(gexs_manager* h, const double* h_freq, const double* h_intens, int n)
{
    if (!h) return GEXS_ERR_INVALID;
    h->m->TransferFreq(const_cast<double*>(h_freq), const_cast<double*>(h_intens), n);
    return mstat(h);
}

int gexs_manager_transfer_vectors(gexs_manager* h, size_t nener, const double* h_energies,
                                  const double* h_nu, const double* h_aif, const int* h_gns,
                                  const double* h_gamma, const double* h_n)
{
    if (!h) return GEXS_ERR_INVALID;
    h->m->TransferVectors(nener, const_cast<double*>(h_energies), const_cast<double*>(h_nu),
                          const_cast<double*>(h_aif), const_cast<int*>(h_gns),
                          const_cast<double*>(h_gamma), const_cast<double*>(h_n));
    return mstat(h);
}

int gexs_manager_execute(gexs_manager* h, int n, int n_ener, int start_idx, double temperature,
                         double pressure, double partition)
{
    if (!h) return GEXS_ERR_INVALID;
    h->m->ExecuteCrossSection(n, n_ener, start_idx, temperature, pressure, partition);
    return mstat(h);
}

int gexs_manager_transfer_results(gexs_manager* h, double* h_freq, double* h_intens, int n, int i)
{
    if (!h) return GEXS_ERR_INVALID;
    h->m->TransferResults(h_freq, h_intens, n, i);
    return mstat(h);
}

int gexs_manager_ntrans(gexs_manager* h, size_t* out)
{
    if (!h || !out) return GEXS_ERR_INVALID;
    *out = h->m->GetNtrans();
    return mstat(h);
}

int gexs_manager_ready(gexs_manager* h, int* ready)
{
    if (!h || !ready) return GEXS_ERR_INVALID;
    *ready = h->m->ReadyForWork() ? 1 : 0;
    return mstat(h);
}

}  // extern "C"
