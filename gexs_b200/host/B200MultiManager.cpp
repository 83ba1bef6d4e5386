/*
 * B200MultiManager.cpp — BaseManager over several GPUs by bin ranges (see
 * the header), and its flat C constructor gexs_manager_create_multi.
 */
#include "B200MultiManager.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cuda_runtime.h>

namespace {
/* tiles of every launch shape divide 4096 bins */
constexpr int kAlign = 4096;
}  // namespace

B200MultiManager::B200MultiManager(ProfileType profile, const std::vector<int>& devices,
                                   int convention, int precision, size_t memory_bytes)
    : BaseManager(profile), convention_(convention)
{
    std::vector<int> devs = devices;
    if (devs.empty()) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) { fail(GEXS_ERR_CUDA); return; }
        for (int d = 0; d < n; ++d) devs.push_back(d);
    }
    for (int d : devs) {
        B200Manager* m = new B200Manager(profile, d, convention, precision, memory_bytes);
        m_.push_back(m);
        if (m->last_status()) { fail(m->last_status()); return; }
    }
}

B200MultiManager::~B200MultiManager()
{
    for (B200Manager* m : m_) delete m;
}

int B200MultiManager::last_status() const
{
    if (status_) return status_;
    for (const B200Manager* m : m_)
        if (m->last_status()) return m->last_status();
    return GEXS_OK;
}

void B200MultiManager::InitializeVectors(int Npoints) { InitializeVectors(Npoints, 1); }

void B200MultiManager::InitializeVectors(int Npoints, int num_cs)
{
    if (last_status()) return;
    npoints_ = Npoints;
    num_cs_ = num_cs;
    size_t cap = (size_t)-1;
    for (B200Manager* m : m_) {
        m->InitializeVectors(Npoints, num_cs);
        cap = std::min(cap, m->GetNtrans());
    }
    /* a device gets at most the whole chunk */
    N_trans = m_.empty() ? 0 : cap;
    touched_.assign(m_.size(), std::vector<std::pair<int64_t, int64_t>>(num_cs > 0 ? num_cs : 0,
                                                                        {INT64_MAX, INT64_MIN}));
}

void B200MultiManager::InitializeConstants(double half_width, double temperature,
                                           double partition, double dfreq, double meanmass,
                                           double pressure, double ref_temp, double ref_press)
{
    if (last_status()) return;
    half_width_ = half_width;
    dfreq_ = dfreq;
    for (B200Manager* m : m_)
        m->InitializeConstants(half_width, temperature, partition, dfreq, meanmass, pressure,
                               ref_temp, ref_press);
}

void B200MultiManager::TransferFreq(double* h_freq, double* h_intens, int N)
{
    if (last_status()) return;
    if (N != npoints_ || !h_freq || !h_intens) { fail(GEXS_ERR_INVALID); return; }
    freq_.assign(h_freq, h_freq + N);
    /* the initial contents are added once at TransferResults; the devices
     * start from zero */
    init_.assign(h_intens, h_intens + N);
    std::vector<double> zeros((size_t)N, 0.0);
    for (B200Manager* m : m_) m->TransferFreq(h_freq, zeros.data(), N);
}

void B200MultiManager::TransferVectors(size_t Nener, double* h_energies, double* h_nu,
                                       double* h_aif, int* h_gns, double* h_gamma, double* h_n)
{
    if (last_status()) return;
    if (freq_.empty()) { fail(GEXS_ERR_INVALID); return; }
    const int n = (int)m_.size();
    bounds_.assign(n + 1, 0);
    lo_.assign(n, 0);
    hi_.assign(n, 0);
    /* the largest cutoff any convention uses (gexs_job_init: 25, min(25 P,
     * 100), 100, or 10 half-widths for the Gaussian), a margin of bins for
     * the tiles' own searches, and a halo of one alignment step on each
     * side for the per-pair cuts */
    const double reach = std::max(100.0, 10.0 * half_width_) + (kAlign + 8.0) * dfreq_ +
                         1e-9 * (std::fabs(freq_.back()) + 100.0);
    int st = gexs_shard_plan(h_nu, (int64_t)Nener, freq_[0], dfreq_, 0, npoints_, reach, kAlign,
                             n, bounds_.data(), lo_.data(), hi_.data());
    if (st) { fail(st); return; }
    for (int g = 0; g < n; ++g) {
        const size_t a = (size_t)lo_[g];
        m_[g]->TransferVectors((size_t)(hi_[g] - lo_[g]), h_energies + a, h_nu + a, h_aif + a,
                               h_gns + a, h_gamma ? h_gamma + a : nullptr, h_n ? h_n + a : nullptr);
    }
    tasks_ = 0;
}

void B200MultiManager::ExecuteCrossSection(int, int, int)
{
    /* deprecated in the reference too (GPUManager.cpp:168-184) */
    fail(GEXS_ERR_INVALID);
}

void B200MultiManager::ExecuteCrossSection(int N, int N_ener, int start_idx, double temperature,
                                           double pressure, double partition)
{
    if (last_status()) return;
    const int n = (int)m_.size();
    if (bounds_.size() != (size_t)n + 1 || tasks_ >= num_cs_ || N < 0 || start_idx < 0 ||
        start_idx + N > npoints_) { fail(GEXS_ERR_INVALID); return; }
    (void)N_ener;   /* each device takes its own sub-list */
    /* the chunk's cuts moved onto multiples of kAlign from this pair's start */
    std::vector<int64_t> c(n + 1);
    c[0] = start_idx;
    c[n] = (int64_t)start_idx + N;
    for (int g = 1; g < n; ++g) {
        int64_t b = start_idx + (int64_t)std::llround((double)(bounds_[g] - start_idx) / kAlign) * kAlign;
        c[g] = std::min(std::max(b, c[g - 1]), c[n]);
    }
    for (int g = 0; g < n; ++g) {
        const int64_t a = c[g], b = c[g + 1];
        m_[g]->ExecuteCrossSection((int)(b - a), (int)(hi_[g] - lo_[g]), (int)a, temperature,
                                   pressure, partition);
        if (b > a) {
            auto& t = touched_[g][tasks_];
            t.first = std::min(t.first, a);
            t.second = std::max(t.second, b);
        }
    }
    ++tasks_;
}

void B200MultiManager::TransferResults(double* h_freq, double* h_intens, int N)
{
    TransferResults(h_freq, h_intens, N, 0);
}

void B200MultiManager::TransferResults(double* h_freq, double* h_intens, int N, int I)
{
    if (last_status()) return;
    if (I < 0 || I >= num_cs_ || N < 0 || N > npoints_ || !h_intens) { fail(GEXS_ERR_INVALID); return; }
    if (h_freq) std::memcpy(h_freq, freq_.data(), sizeof(double) * (size_t)N);
    for (int j = 0; j < N; ++j) h_intens[j] += init_[(size_t)j];
    for (size_t g = 0; g < m_.size(); ++g) {
        const auto& t = touched_[g][I];
        const int64_t a = std::max<int64_t>(t.first, 0), b = std::min<int64_t>(t.second, N);
        if (b > a) m_[g]->AddResultRange(h_intens, (int)a, (int)b, I);
        if (m_[g]->last_status()) { fail(m_[g]->last_status()); return; }
    }
}

void B200MultiManager::Cleanup()
{
    for (B200Manager* m : m_) m->Cleanup();
}

bool B200MultiManager::ReadyForWork()
{
    bool ready = true;
    for (B200Manager* m : m_) ready = m->ReadyForWork() && ready;
    return ready;
}
