/*
 * B200Manager.cpp — BaseManager implementation over the gexs C ABI, and the
 * flat gexs_manager_* C wrappers declared in include/gexs_b200.h.
 */
#include "B200Manager.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include <cuda_runtime.h>

namespace {
const int kCopyChunks = 64;                     /* pieces of an overlapped line copy */
const int kSegments = 6;                        /* grid segments of the first launch  */
const double kSegmentFrac[kSegments] = {1.0 / 64, 1.0 / 32, 1.0 / 8, 1.0 / 4, 1.0 / 2, 1.0};
const int64_t kSegmentAlign = 4096;             /* widest tile: 32 lanes x 16 bins x 8 warps */
const size_t kSegmentMinLines = (size_t)1 << 21;
const size_t kSamples = 8192;

/* memcpy of a grid-sized host array (tens of MB), split over up to 8
 * threads; serial when a thread cannot be started */
void par_copy(void* dst, const void* src, size_t bytes)
{
    const size_t kPart = (size_t)4 << 20;
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min(std::min((size_t)8, hw), std::max((size_t)1, bytes / kPart));
    const size_t per = (bytes + nt - 1) / nt;
    auto part = [=](size_t t) {
        const size_t o = t * per;
        if (o < bytes) std::memcpy((char*)dst + o, (const char*)src + o, std::min(per, bytes - o));
    };
    std::vector<std::thread> th;
    size_t t = 1;
    try {
        for (; t < nt; ++t) th.emplace_back(part, t);
    } catch (...) {
        for (; t < nt; ++t) part(t);
    }
    part(0);
    for (std::thread& x : th) x.join();
}
}  // namespace

B200Manager::B200Manager(ProfileType profile, int device, int convention, int precision,
                         size_t memory_bytes)
    : BaseManager(profile), device_(device), convention_(convention), precision_(precision),
      memory_bytes_(memory_bytes)
{
    int st = gexs_ctx_create(device, &ctx_);
    if (st) { fail(st); return; }
    cudaStream_t s, cs;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) { fail(GEXS_ERR_CUDA); return; }
    stream_ = (void*)s;
    for (int k = 1; k < kSegments; ++k) {
        cudaStream_t sk;
        if (cudaStreamCreateWithFlags(&sk, cudaStreamNonBlocking) != cudaSuccess) { fail(GEXS_ERR_CUDA); return; }
        seg_stream_.push_back((void*)sk);
    }
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) { fail(GEXS_ERR_CUDA); return; }
    copy_stream_ = (void*)cs;
    for (int c = 0; c < kCopyChunks + kSegments + 1; ++c) {
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) { fail(GEXS_ERR_CUDA); return; }
        if (c < kCopyChunks) chunk_ev_.push_back((void*)e);
        else if (c == kCopyChunks) done_ev_ = (void*)e;
        else if (c == kCopyChunks + 1) fork_ev_ = (void*)e;
        else join_ev_.push_back((void*)e);
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    if (memory_bytes_ == 0) memory_bytes_ = fr / 2;
    InitializeMemory(memory_bytes_);
}

B200Manager::~B200Manager()
{
    Cleanup();
    for (void* e : chunk_ev_) cudaEventDestroy((cudaEvent_t)e);
    for (void* e : join_ev_) cudaEventDestroy((cudaEvent_t)e);
    for (void* e : {done_ev_, fork_ev_})
        if (e) cudaEventDestroy((cudaEvent_t)e);
    if (copy_stream_) cudaStreamDestroy((cudaStream_t)copy_stream_);
    for (void* sk : seg_stream_) cudaStreamDestroy((cudaStream_t)sk);
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
    par_copy(h_freq_.data(), h_freq, sizeof(double) * (size_t)N);
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
    cudaStream_t cs = (cudaStream_t)copy_stream_;
    tasks_ = 0;
    nlines_ = Nener;
    /* kernels queued on the previous lines must finish before they are overwritten */
    if (cudaEventRecord((cudaEvent_t)done_ev_, (cudaStream_t)stream_) != cudaSuccess ||
        cudaStreamWaitEvent(cs, (cudaEvent_t)done_ev_, 0) != cudaSuccess) { fail(GEXS_ERR_CUDA); return; }
    const bool press = h_gamma && h_n && d_gam_ && d_n_;
    nchunks_ = Nener == 0 ? 0 : (Nener >= kSegmentMinLines ? kCopyChunks : 1);
    chunk_lines_ = nchunks_ ? (Nener + nchunks_ - 1) / nchunks_ : 0;
    bool ok = true;
    for (int c = 0; c < nchunks_ && ok; ++c) {
        const size_t i0 = std::min(Nener, (size_t)c * chunk_lines_);
        const size_t n = std::min(chunk_lines_, Nener - i0);
        const size_t d8 = sizeof(double) * n, d4 = sizeof(int) * n;
        if (n) {
            ok = cudaMemcpyAsync(d_nu_ + i0, h_nu + i0, d8, cudaMemcpyHostToDevice, cs) == cudaSuccess &&
                 cudaMemcpyAsync(d_e_ + i0, h_energies + i0, d8, cudaMemcpyHostToDevice, cs) == cudaSuccess &&
                 cudaMemcpyAsync(d_a_ + i0, h_aif + i0, d8, cudaMemcpyHostToDevice, cs) == cudaSuccess &&
                 cudaMemcpyAsync(d_g_ + i0, h_gns + i0, d4, cudaMemcpyHostToDevice, cs) == cudaSuccess;
            if (ok && press)
                ok = cudaMemcpyAsync(d_gam_ + i0, h_gamma + i0, d8, cudaMemcpyHostToDevice, cs) == cudaSuccess &&
                     cudaMemcpyAsync(d_n_ + i0, h_n + i0, d8, cudaMemcpyHostToDevice, cs) == cudaSuccess;
        }
        if (ok) ok = cudaEventRecord((cudaEvent_t)chunk_ev_[c], cs) == cudaSuccess;
    }
    if (!ok) { fail(GEXS_ERR_CUDA); return; }
    /* nu at every stride-th line and at the last: conservative line bounds later */
    samp_idx_.clear(); samp_nu_.clear();
    if (Nener) {
        const size_t stride = std::max<size_t>(1, Nener / kSamples);
        for (size_t i = 0; i < Nener; i += stride) { samp_idx_.push_back(i); samp_nu_.push_back(h_nu[i]); }
        if (samp_idx_.back() != Nener - 1) { samp_idx_.push_back(Nener - 1); samp_nu_.push_back(h_nu[Nener - 1]); }
    }
    fresh_ = nchunks_ > 0;
}

/* first index whose nu can be >= v: lines before it all have nu < v */
size_t B200Manager::lines_below(double v) const
{
    auto it = std::lower_bound(samp_nu_.begin(), samp_nu_.end(), v);   /* first sample >= v */
    if (it == samp_nu_.begin()) return 0;
    return samp_idx_[(size_t)(it - samp_nu_.begin()) - 1];
}

/* an index past every line with nu <= v */
size_t B200Manager::lines_upto(double v) const
{
    auto it = std::upper_bound(samp_nu_.begin(), samp_nu_.end(), v);   /* first sample > v */
    if (it == samp_nu_.end()) return nlines_;
    return samp_idx_[(size_t)(it - samp_nu_.begin())];
}

/* nu of the sampled line at or below index i */
double B200Manager::nu_at(size_t i) const
{
    auto it = std::upper_bound(samp_idx_.begin(), samp_idx_.end(), i);
    return samp_nu_[(size_t)(it - samp_idx_.begin()) - 1];
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
    int st = fresh_ ? run_segmented()
                    : gexs_run(ctx_, pending_.data(), (int)pending_.size(), nullptr, stream_);
    pending_.clear();
    if (st) return fail(st);
    return GEXS_OK;
}

/* The queued pairs right after TransferVectors: grid segments at the line
 * quantiles kSegmentFrac, each given the sub-list of lines that can reach
 * it (every line within cutoff + margin of its bins, a superset of what
 * each tile's own search selects, so each tile finds the same lines in the
 * same order) and started once the pieces holding that sub-list have
 * arrived.  Segment boundaries sit at start_idx + k * kSegmentAlign, so
 * every tile is the tile of a single launch over the pair. */
int B200Manager::run_segmented()
{
    cudaStream_t s0 = (cudaStream_t)stream_;
    std::vector<std::vector<gexs_job>> seg(kSegments);
    std::vector<size_t> need(kSegments, 0);
    for (const gexs_job& j : pending_) {
        const size_t ne = (size_t)j.lines.count;
        const int64_t S = j.start_idx, E = j.start_idx + j.n_points;
        if (ne < kSegmentMinLines || j.n_points < 2 * kSegmentAlign || samp_nu_.empty()) {
            seg[kSegments - 1].push_back(j);
            need[kSegments - 1] = std::max(need[kSegments - 1], ne);
            continue;
        }
        int64_t b0 = S;
        for (int k = 0; k < kSegments && b0 < E; ++k) {
            int64_t b1 = E;
            if (k + 1 < kSegments) {
                const double nu = nu_at((size_t)(kSegmentFrac[k] * (double)(ne - 1)));
                const double bin = std::floor((nu - j.nu_start) / j.dnu);
                if (bin > (double)S) {
                    const int64_t g = S + ((std::min((int64_t)bin, E) - S) / kSegmentAlign) * kSegmentAlign;
                    b1 = std::max(b0, g);
                } else {
                    b1 = b0;
                }
                if (b1 == b0) continue;
            }
            const double f0 = j.nu_start + (double)b0 * j.dnu;
            const double fl = j.nu_start + (double)(b1 - 1) * j.dnu;
            const double m = 8.0 * j.dnu + 1e-8 * (std::fabs(fl) + j.cutoff);
            size_t L0 = std::min(lines_below(f0 - j.cutoff - m), ne);
            size_t L1 = std::min(lines_upto(fl + j.cutoff + m), ne);
            L0 &= ~(size_t)3;
            if (L1 < L0) L1 = L0;
            gexs_job p = j;
            p.start_idx = b0;
            p.n_points = b1 - b0;
            p.lines.nu = j.lines.nu + L0; p.lines.elow = j.lines.elow + L0;
            p.lines.aif = j.lines.aif + L0; p.lines.gns = j.lines.gns + L0;
            if (j.lines.gamma) p.lines.gamma = j.lines.gamma + L0;
            if (j.lines.n) p.lines.n = j.lines.n + L0;
            p.lines.count = (int64_t)(L1 - L0);
            seg[k].push_back(p);
            need[k] = std::max(need[k], L1);
            b0 = b1;
        }
    }
    fresh_ = false;
    /* segment k runs on stream k (stream_ for the first), forked from stream_ */
    if (cudaEventRecord((cudaEvent_t)fork_ev_, s0) != cudaSuccess) return GEXS_ERR_CUDA;
    for (void* sk : seg_stream_)
        if (cudaStreamWaitEvent((cudaStream_t)sk, (cudaEvent_t)fork_ev_, 0) != cudaSuccess)
            return GEXS_ERR_CUDA;
    int st = GEXS_OK;
    for (int k = 0; k < kSegments && st == GEXS_OK; ++k) {
        if (seg[k].empty()) continue;
        cudaStream_t s = k == 0 ? s0 : (cudaStream_t)seg_stream_[k - 1];
        if (need[k] > 0) {
            const size_t c = std::min((size_t)nchunks_ - 1, (need[k] - 1) / chunk_lines_);
            if (cudaStreamWaitEvent(s, (cudaEvent_t)chunk_ev_[c], 0) != cudaSuccess) { st = GEXS_ERR_CUDA; break; }
        }
        st = gexs_run(ctx_, seg[k].data(), (int)seg[k].size(), nullptr, s);
    }
    /* stream_ joins every segment stream and has seen every piece arrive */
    bool ok = true;
    for (size_t k = 0; k < seg_stream_.size() && ok; ++k)
        ok = cudaEventRecord((cudaEvent_t)join_ev_[k], (cudaStream_t)seg_stream_[k]) == cudaSuccess &&
             cudaStreamWaitEvent(s0, (cudaEvent_t)join_ev_[k], 0) == cudaSuccess;
    if (ok) ok = cudaStreamWaitEvent(s0, (cudaEvent_t)chunk_ev_[nchunks_ - 1], 0) == cudaSuccess;
    if (!ok) return st ? st : GEXS_ERR_CUDA;
    return st;
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
    /* the grid is host data: copied while the queued launches run */
    if (h_freq) par_copy(h_freq, h_freq_.data(), sizeof(double) * (size_t)N);
    int st = gexs_ctx_check(ctx_, stream_);
    if (st) { fail(st); return; }
    if (cudaMemcpy(h_intens, d_slots_[I], sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost) != cudaSuccess)
        fail(GEXS_ERR_CUDA);
}

void B200Manager::AddResultRange(double* h_intens, int lo, int hi, int I)
{
    if (status_) return;
    if (I < 0 || I >= (int)d_slots_.size() || lo < 0 || hi > npoints_ || lo > hi || !h_intens) {
        fail(GEXS_ERR_INVALID);
        return;
    }
    if (flush()) return;
    cudaSetDevice(device_);
    int st = gexs_ctx_check(ctx_, stream_);
    if (st) { fail(st); return; }
    std::vector<double> tmp((size_t)(hi - lo));
    if (hi > lo && cudaMemcpy(tmp.data(), d_slots_[I] + lo, sizeof(double) * (size_t)(hi - lo),
                              cudaMemcpyDeviceToHost) != cudaSuccess) {
        fail(GEXS_ERR_CUDA);
        return;
    }
    for (int j = lo; j < hi; ++j) h_intens[j] += tmp[(size_t)(j - lo)];
}

void B200Manager::Cleanup()
{
    if (ctx_) { flush(); cudaStreamSynchronize((cudaStream_t)stream_); }
    if (copy_stream_) cudaStreamSynchronize((cudaStream_t)copy_stream_);
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
#include "B200MultiManager.h"

/* one device (single) or several (multi); m is the one in use */
struct gexs_manager {
    BaseManager* m = nullptr;
    B200Manager* single = nullptr;
    B200MultiManager* multi = nullptr;
};

static int mstat(gexs_manager* h)
{
    return h->single ? h->single->last_status() : h->multi->last_status();
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
    h->single = new B200Manager((ProfileType)profile, device, convention, precision, memory_bytes);
    h->m = h->single;
    int st = h->single->last_status();
    if (st) { delete h->single; delete h; return st; }
    *out = h;
    return GEXS_OK;
}

int gexs_manager_create_multi(int profile, const int* devices, int ndev, int convention,
                              int precision, size_t memory_bytes, gexs_manager** out)
{
    if (!out || ndev < 0 || (ndev > 0 && !devices)) return GEXS_ERR_INVALID;
    *out = nullptr;
    if (profile != GEXS_GAUSSIAN && profile != GEXS_DOPPLER && profile != GEXS_VOIGT &&
        profile != GEXS_VOIGT_QUAD) return GEXS_ERR_INVALID;
    std::vector<int> devs(devices, devices + ndev);
    gexs_manager* h = new gexs_manager();
    h->multi = new B200MultiManager((ProfileType)profile, devs, convention, precision, memory_bytes);
    h->m = h->multi;
    int st = h->multi->last_status();
    if (st) { delete h->multi; delete h; return st; }
    *out = h;
    return GEXS_OK;
}

int gexs_manager_destroy(gexs_manager* h)
{
    if (!h) return GEXS_OK;
    delete h->single;
    delete h->multi;
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
