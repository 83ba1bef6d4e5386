/*
 * gexs_server.cpp — continuous-batching request loop (include/gexs_serve.h).
 *
 * One worker thread owns admission and launches:
 *   1. completed batches are detected with cudaEventQuery and their
 *      requests marked done (waiters are woken);
 *   2. pending requests are admitted in arrival order while their output
 *      grids fit in the HBM budget and the in-flight cap allows;
 *   3. the admitted group gets Q(T) from the resident table of its list
 *      (or the partition kernel on the worker's own stream for temperatures
 *      outside it), stream-ordered output buffers from the context's
 *      memory pool, which also holds the launch's scratch and keeps freed
 *      pages mapped, and one gexs_run launch on the next stream of the
 *      server, followed by an event.  A request is admitted for its output
 *      and the scratch its job takes (prep arrays, tables, slice rows), so
 *      what the pool holds stays within the budget.
 * Nothing on this path synchronises the device (no cudaMalloc/cudaFree),
 * so a new batch starts while earlier ones still run.  A request's output
 * is released when the caller fetches it (gexs_server_wait), which frees
 * budget for the next admissions.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>
#include "../../include/gexs_serve.h"
#include "../csrc/gexs_internal.h"

namespace {

enum { RQ_PENDING = 0, RQ_RUNNING = 1, RQ_DONE = 2, RQ_FAILED = 3 };

/* resident Q(T) table of a list: Q at kQPoints temperatures log-spaced
 * over [kQTmin, kQTmax], computed once on the device when the list is
 * added; a request's Q(T) is the 4-point Lagrange interpolation of ln Q in
 * ln T (relative error ~1e-14 on smooth state sums, checked against the
 * exact device sum in the tests); other temperatures take the exact sum */
constexpr int kQPoints = 4096;
constexpr double kQTmin = 10.0, kQTmax = 10000.0;

struct List {
    /* device copy of the list, in the format it was added in (FP64, or
     * the 24-byte compact layout); the server owns every array */
    gexs_lines lines{};
    int64_t count = 0;
    double* se = nullptr;
    int32_t* sg = nullptr;
    int64_t nstates = 0;
    double mass = 0.0;
    size_t bytes = 0;
    double* d_qtab = nullptr;          /* Q at the table temperatures (HBM)   */
    std::vector<double> lnq;           /* ln Q, host mirror for job setup     */
};

void free_list(List& L)
{
    cudaFree(const_cast<double*>(L.lines.nu)); cudaFree(const_cast<double*>(L.lines.elow));
    cudaFree(const_cast<double*>(L.lines.aif)); cudaFree(const_cast<int32_t*>(L.lines.gns));
    cudaFree(const_cast<double*>(L.lines.gamma)); cudaFree(const_cast<double*>(L.lines.n));
    cudaFree(L.se); cudaFree(L.sg); cudaFree(L.d_qtab);
    L.lines = gexs_lines{};
    L.se = nullptr; L.sg = nullptr; L.d_qtab = nullptr;
}

double qtab_lnt(int k)
{
    return std::log(kQTmin) + (std::log(kQTmax) - std::log(kQTmin)) * (double)k / (kQPoints - 1);
}

/* Q(T) from the resident table; false outside its range */
bool q_from_table(const List& L, double T, double* q)
{
    if (L.lnq.empty() || !(T >= kQTmin && T <= kQTmax)) return false;
    const double h = (std::log(kQTmax) - std::log(kQTmin)) / (kQPoints - 1);
    const double u = std::log(T);
    int i = (int)std::floor((u - std::log(kQTmin)) / h);
    i = std::min(std::max(i, 1), kQPoints - 3);
    double x[4], v = 0.0;
    for (int a = 0; a < 4; ++a) x[a] = qtab_lnt(i - 1 + a);
    for (int a = 0; a < 4; ++a) {
        double w = 1.0;
        for (int b = 0; b < 4; ++b)
            if (b != a) w *= (u - x[b]) / (x[a] - x[b]);
        v += w * L.lnq[i - 1 + a];
    }
    *q = std::exp(v);
    return true;
}

struct Req {
    uint64_t id = 0;
    gexs_request r;
    gexs_job job;
    double* d_out = nullptr;
    size_t bytes = 0;
    int state = RQ_PENDING;
    int status = GEXS_OK;
    cudaEvent_t done = nullptr;        /* owned by the batch */
    gexs_request_info info;
};

struct Batch {
    cudaEvent_t ev = nullptr;
    std::vector<Req*> reqs;
    int slot = -1;                     /* error word of this batch's kernels */
};

constexpr int kMaxBatchTemps = 1024;

}  // namespace

struct gexs_server {
    int device = 0;
    size_t budget = 0;
    int max_inflight = 256;
    gexs_ctx* ctx = nullptr;
    std::vector<cudaStream_t> streams;
    size_t next_stream = 0;
    cudaStream_t part_stream = nullptr;
    double *d_betas = nullptr, *d_partial = nullptr, *d_q = nullptr;
    int part_chunks = 0;
    int nsm = 148;
    /* one kernel error word per running batch (a running batch holds at
     * least one admitted request, so max_inflight slots suffice), read
     * back into pinned host memory behind the batch's kernels */
    int* d_errs = nullptr;
    int* h_errs = nullptr;
    std::vector<int> free_slots;

    /* a deque: adding a list never moves the others, which the worker
     * reads without the lock while it launches */
    std::deque<List> lists;
    size_t resident = 0;
    std::mutex part_mu;           /* the partition buffers (d_betas, d_partial, d_q) */

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> pending;
    std::unordered_map<uint64_t, Req*> reqs;
    std::vector<Batch> running;
    /* a batch's event and the requests of that batch not yet fetched: the
     * last waiter to fetch destroys it (waiters remove their request from
     * `reqs` before they use the event, so `reqs` cannot tell) */
    std::unordered_map<cudaEvent_t, int> ev_refs;
    size_t inflight_bytes = 0;
    int inflight = 0;
    uint64_t next_id = 1;
    bool stop = false;
    bool kick = false;            /* a submission or a released output */
    std::thread worker;

    std::mutex copy_mu;
    std::vector<cudaStream_t> copy_free;

    int64_t n_submitted = 0, n_completed = 0, n_batches = 0;
    /* a group that could not get its memory while other batches ran went
     * back to the queue; admission waits for one of those to complete */
    bool oom_hold = false;
    int64_t oom_mark = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

size_t output_bytes(const gexs_request& r) { return (size_t)r.grid_points * sizeof(double); }

/* exact Q(T) by the device reduction over the list's states (partition
 * kernel on the server's own stream, no device-wide synchronisation);
 * d_out (device, may be NULL) also gets the values */
int exact_partitions(gexs_server* s, const List& L, const std::vector<double>& temps,
                     std::vector<double>& q, double* d_out = nullptr)
{
    const double planck = 6.6260693e-27, vellgt = 2.99792458e10, boltz = 1.380658e-16;
    std::lock_guard<std::mutex> g(s->part_mu);
    q.assign(temps.size(), 0.0);
    for (size_t off = 0; off < temps.size(); off += kMaxBatchTemps) {
        int nt = (int)std::min<size_t>(kMaxBatchTemps, temps.size() - off);
        std::vector<double> betas(nt);
        for (int i = 0; i < nt; ++i) betas[i] = planck * vellgt / (boltz * temps[off + i]);
        cudaError_t e = cudaMemcpyAsync(s->d_betas, betas.data(), sizeof(double) * nt,
                                        cudaMemcpyHostToDevice, s->part_stream);
        if (e == cudaSuccess)
            e = gexs::launch_partition(L.se, L.sg, L.nstates, s->d_betas, nt, s->d_partial,
                                       s->part_chunks, s->d_q, s->part_stream);
        if (e == cudaSuccess && d_out)
            e = cudaMemcpyAsync(d_out + off, s->d_q, sizeof(double) * nt,
                                cudaMemcpyDeviceToDevice, s->part_stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(q.data() + off, s->d_q, sizeof(double) * nt,
                                cudaMemcpyDeviceToHost, s->part_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->part_stream);
        if (e != cudaSuccess) return gexs::cuda_error(e, "server partition");
    }
    return GEXS_OK;
}

/* Q(T) for the admitted requests of one list: from the resident table;
 * only temperatures outside it wait for an exact device reduction */
int partitions(gexs_server* s, const List& L, const std::vector<double>& temps, std::vector<double>& q)
{
    q.assign(temps.size(), 0.0);
    std::vector<double> miss_t;
    std::vector<size_t> miss_i;
    for (size_t i = 0; i < temps.size(); ++i)
        if (!q_from_table(L, temps[i], &q[i])) { miss_t.push_back(temps[i]); miss_i.push_back(i); }
    if (miss_t.empty()) return GEXS_OK;
    std::vector<double> mq;
    int st = exact_partitions(s, L, miss_t, mq);
    if (st) return st;
    for (size_t k = 0; k < miss_i.size(); ++k) q[miss_i[k]] = mq[k];
    return GEXS_OK;
}

/* build jobs, allocate outputs and launch one group; called without the lock */
void launch_group(gexs_server* s, std::vector<Req*>& adm)
{
    cudaSetDevice(s->device);
    cudaStream_t st = s->streams[s->next_stream++ % s->streams.size()];
    int status = GEXS_OK;
    std::map<int, std::vector<Req*>> by_list;
    for (Req* r : adm) by_list[r->r.list_id].push_back(r);
    std::vector<gexs_job> jobs;
    for (auto& kv : by_list) {
        const List& L = s->lists[kv.first];
        std::vector<double> temps, q;
        for (Req* r : kv.second) temps.push_back(r->r.temperature);
        if (!status) status = partitions(s, L, temps, q);
        for (size_t i = 0; i < kv.second.size() && !status; ++i) {
            Req* r = kv.second[i];
            gexs_job j;
            status = gexs_job_init(&j, r->r.convention, r->r.profile, r->r.temperature,
                                   r->r.pressure, q[i], L.mass, r->r.ref_temp, r->r.ref_press,
                                   r->r.half_width, r->r.cutoff, r->r.nu_start, r->r.dnu,
                                   r->r.grid_points);
            if (status) break;
            j.precision = r->r.precision;
            j.quad_nodes = r->r.quad_nodes;
            j.accumulate = 0;
            j.lines = L.lines;
            void* d = nullptr;
            if (gexs::pool_alloc(gexs::ctx_pool(s->ctx), &d, output_bytes(r->r), st) != cudaSuccess) {
                status = GEXS_ERR_OOM;
                break;
            }
            r->d_out = (double*)d;
            j.out = r->d_out;
            r->job = j;
            jobs.push_back(j);
        }
    }
    Batch b;
    if (!status) {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->free_slots.empty()) {
            status = gexs::set_error(GEXS_ERR_INVALID, "server: no free error slot");
        } else {
            b.slot = s->free_slots.back();
            s->free_slots.pop_back();
        }
    }
    int* d_err = status ? nullptr : s->d_errs + b.slot;
    if (!status && gexs::zero_ints(d_err, 1, st) != cudaSuccess) status = GEXS_ERR_CUDA;
    if (!status) status = gexs::run_jobs(s->ctx, jobs.data(), (int)jobs.size(), nullptr, (void*)st, d_err);
    if (!status && cudaMemcpyAsync(s->h_errs + b.slot, d_err, sizeof(int), cudaMemcpyDeviceToHost,
                                   st) != cudaSuccess)
        status = GEXS_ERR_CUDA;
    if (!status && cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming) != cudaSuccess)
        status = GEXS_ERR_CUDA;
    if (!status && cudaEventRecord(b.ev, st) != cudaSuccess) status = GEXS_ERR_CUDA;
    std::lock_guard<std::mutex> g(s->mu);
    if (status == GEXS_ERR_OOM && !s->running.empty()) {
        /* out of memory while earlier batches still hold theirs (the pool's
         * pages can be too fragmented for a large prep array): undo the
         * admission, put the group back at the head of the queue in arrival
         * order and admit again after the next completion */
        cudaStreamSynchronize(st);
        if (b.ev) cudaEventDestroy(b.ev);
        if (b.slot >= 0) s->free_slots.push_back(b.slot);
        for (auto it = adm.rbegin(); it != adm.rend(); ++it) {
            Req* r = *it;
            if (r->d_out) { cudaFreeAsync(r->d_out, st); r->d_out = nullptr; }
            r->state = RQ_PENDING;
            s->inflight--;
            s->inflight_bytes -= r->bytes;
            s->pending.push_front(r);
        }
        cudaGetLastError();
        s->oom_hold = true;
        s->oom_mark = s->n_completed;
        return;
    }
    s->n_batches++;
    for (Req* r : adm) {
        r->info.batch_size = (int)adm.size();
        if (status) {
            r->state = RQ_FAILED;
            r->status = status;
            r->info.done_ms = s->now_ms();
        } else {
            r->state = RQ_RUNNING;
            r->done = b.ev;
        }
    }
    if (!status) s->ev_refs[b.ev] = (int)adm.size();
    if (status) {
        /* nothing of this batch is read back: wait for its work before the
         * slot and the outputs are reused */
        cudaStreamSynchronize(st);
        if (b.ev) cudaEventDestroy(b.ev);
        if (b.slot >= 0) s->free_slots.push_back(b.slot);
        for (Req* r : adm)
            if (r->d_out) { cudaFreeAsync(r->d_out, st); r->d_out = nullptr; }
        s->cv_done.notify_all();
        return;
    }
    b.reqs = adm;
    s->running.push_back(b);
}

void worker_loop(gexs_server* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        /* sleep until kicked, or poll running batches every 100 us */
        s->cv_work.wait_for(lk, std::chrono::microseconds(s->running.empty() ? 20000 : 100),
                            [&] { return s->stop || s->kick; });
        s->kick = false;
        /* 1. completions */
        for (size_t i = 0; i < s->running.size();) {
            cudaError_t q = cudaEventQuery(s->running[i].ev);
            if (q == cudaErrorNotReady) { ++i; continue; }
            double t = s->now_ms();
            /* the batch's kernels flagged an error (a bounded wait ran out):
             * its outputs are incomplete */
            const int slot = s->running[i].slot;
            const int kerr = (q == cudaSuccess) ? s->h_errs[slot] : 0;
            for (Req* r : s->running[i].reqs) {
                r->state = (q == cudaSuccess && !kerr) ? RQ_DONE : RQ_FAILED;
                if (q != cudaSuccess) r->status = GEXS_ERR_CUDA;
                else if (kerr) r->status = GEXS_ERR_KERNEL;
                r->info.done_ms = t;
                r->info.status = r->status;
                s->n_completed++;
            }
            s->free_slots.push_back(slot);
            /* the event is destroyed when its last request is fetched */
            s->running.erase(s->running.begin() + i);
            s->cv_done.notify_all();
        }
        if (s->stop && s->running.empty()) break;
        if (s->stop) continue;
        /* 2. admission in arrival order */
        const size_t cap = s->budget > s->resident ? s->budget - s->resident : 0;
        std::vector<Req*> adm;
        if (s->oom_hold && (s->n_completed != s->oom_mark || s->running.empty())) s->oom_hold = false;
        while (!s->oom_hold && !s->pending.empty()) {
            Req* r = s->pending.front();
            if (s->inflight >= s->max_inflight || s->inflight_bytes + r->bytes > cap) break;
            s->pending.pop_front();
            s->inflight++;
            s->inflight_bytes += r->bytes;
            r->info.admit_ms = s->now_ms();
            adm.push_back(r);
        }
        if (!adm.empty()) {
            lk.unlock();
            launch_group(s, adm);
            lk.lock();
        }
    }
    /* requests never admitted */
    for (Req* r : s->pending) { r->state = RQ_FAILED; r->status = GEXS_ERR_SHUTDOWN; }
    s->pending.clear();
    s->cv_done.notify_all();
}

cudaStream_t take_copy_stream(gexs_server* s)
{
    std::lock_guard<std::mutex> g(s->copy_mu);
    if (!s->copy_free.empty()) {
        cudaStream_t c = s->copy_free.back();
        s->copy_free.pop_back();
        return c;
    }
    cudaStream_t c = nullptr;
    cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking);
    return c;
}

void give_copy_stream(gexs_server* s, cudaStream_t c)
{
    std::lock_guard<std::mutex> g(s->copy_mu);
    s->copy_free.push_back(c);
}

}  // namespace

extern "C" {

int gexs_server_create(int device, size_t hbm_budget, int max_inflight, int streams,
                       gexs_server** out)
{
    if (!out) return gexs::set_error(GEXS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return gexs::cuda_error(e, "cudaSetDevice");
    gexs_server* s = new gexs_server();
    s->device = device;
    int st = gexs_ctx_create(device, &s->ctx);
    if (st) { delete s; return st; }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    s->budget = hbm_budget ? hbm_budget : (size_t)(0.9 * (double)fr);
    s->max_inflight = max_inflight > 0 ? max_inflight : 256;
    int ns = streams > 0 ? streams : 4;
    for (int i = 0; i < ns; ++i) {
        cudaStream_t c;
        cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking);
        s->streams.push_back(c);
    }
    cudaStreamCreateWithFlags(&s->part_stream, cudaStreamNonBlocking);
    cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, device);
    s->part_chunks = s->nsm * 2;
    bool ok = cudaMalloc(&s->d_betas, sizeof(double) * kMaxBatchTemps) == cudaSuccess &&
              cudaMalloc(&s->d_partial, sizeof(double) * kMaxBatchTemps * s->part_chunks) == cudaSuccess &&
              cudaMalloc(&s->d_q, sizeof(double) * kMaxBatchTemps) == cudaSuccess &&
              cudaMalloc(&s->d_errs, sizeof(int) * s->max_inflight) == cudaSuccess &&
              cudaMallocHost(&s->h_errs, sizeof(int) * s->max_inflight) == cudaSuccess;
    for (int i = s->max_inflight - 1; ok && i >= 0; --i) s->free_slots.push_back(i);
    if (!ok) { gexs_server_destroy(s); return gexs::set_error(GEXS_ERR_OOM, "server buffers"); }
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return GEXS_OK;
}

int gexs_server_destroy(gexs_server* s)
{
    if (!s) return GEXS_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    for (auto& kv : s->reqs) {
        Req* r = kv.second;
        if (r->d_out) cudaFree(r->d_out);
        delete r;
    }
    /* every batch event still referenced, running or finished unfetched */
    for (auto& kv : s->ev_refs) cudaEventDestroy(kv.first);
    for (List& L : s->lists) {
        free_list(L);
    }
    for (cudaStream_t c : s->streams) cudaStreamDestroy(c);
    for (cudaStream_t c : s->copy_free) cudaStreamDestroy(c);
    if (s->part_stream) cudaStreamDestroy(s->part_stream);
    cudaFree(s->d_betas); cudaFree(s->d_partial); cudaFree(s->d_q);
    cudaFree(s->d_errs);
    if (s->h_errs) cudaFreeHost(s->h_errs);
    gexs_ctx_destroy(s->ctx);
    delete s;
    return GEXS_OK;
}

int gexs_server_add_list(gexs_server* s, const double* nu, const double* elow, const double* aif,
                         const int32_t* gns, const double* gamma, const double* n, int64_t count,
                         const double* state_energy, const int32_t* state_g, int64_t nstates,
                         double mean_mass, int* list_id)
{
    gexs_lines in;
    std::memset(&in, 0, sizeof(in));
    in.nu = nu; in.elow = elow; in.aif = aif; in.gns = gns; in.gamma = gamma; in.n = n;
    in.count = count;
    in.format = GEXS_LINES_FP64;
    return gexs_server_add_lines(s, &in, state_energy, state_g, nstates, mean_mass, list_id);
}

int gexs_server_add_lines(gexs_server* s, const gexs_lines* in, const double* state_energy,
                          const int32_t* state_g, int64_t nstates, double mean_mass, int* list_id)
{
    if (!s || !in || !list_id || in->count < 0 || nstates <= 0 || !state_energy || !state_g ||
        !(mean_mass > 0.0) || (in->format != GEXS_LINES_FP64 && in->format != GEXS_LINES_COMPACT))
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_server_add_lines: arguments");
    const bool compact = in->format == GEXS_LINES_COMPACT;
    const int64_t count = in->count;
    if (count > 0 && (!in->nu || !in->elow || !in->aif || (!compact && !in->gns)))
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_server_add_lines: arrays");
    const bool press = in->gamma && in->n;
    /* bytes per line of each 4-or-8-byte field */
    const size_t w = compact ? sizeof(float) : sizeof(double);
    const size_t per_line = sizeof(double) + 2 * w + (compact ? 0 : sizeof(int32_t)) + (press ? 2 * w : 0);
    const size_t bytes = (size_t)count * per_line + (size_t)nstates * (sizeof(double) + sizeof(int32_t)) +
                         kQPoints * sizeof(double);
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->resident + s->inflight_bytes + bytes > s->budget)
            return gexs::set_error(GEXS_ERR_ADMISSION, "line list does not fit in the HBM budget");
    }
    cudaSetDevice(s->device);
    List L;
    L.count = count; L.nstates = nstates; L.mass = mean_mass; L.bytes = bytes;
    L.lines.count = count;
    L.lines.format = in->format;
    const size_t c = (size_t)(count > 0 ? count : 1);
    void *d_nu = nullptr, *d_e = nullptr, *d_a = nullptr, *d_g = nullptr, *d_gam = nullptr, *d_n = nullptr;
    bool ok = cudaMalloc(&d_nu, sizeof(double) * c) == cudaSuccess &&
              cudaMalloc(&d_e, w * c) == cudaSuccess && cudaMalloc(&d_a, w * c) == cudaSuccess &&
              (compact || cudaMalloc(&d_g, sizeof(int32_t) * c) == cudaSuccess) &&
              (!press || (cudaMalloc(&d_gam, w * c) == cudaSuccess &&
                          cudaMalloc(&d_n, w * c) == cudaSuccess)) &&
              cudaMalloc(&L.se, sizeof(double) * nstates) == cudaSuccess &&
              cudaMalloc(&L.sg, sizeof(int32_t) * nstates) == cudaSuccess &&
              cudaMalloc(&L.d_qtab, sizeof(double) * kQPoints) == cudaSuccess;
    L.lines.nu = (const double*)d_nu; L.lines.elow = (const double*)d_e; L.lines.aif = (const double*)d_a;
    L.lines.gns = (const int32_t*)d_g; L.lines.gamma = (const double*)d_gam; L.lines.n = (const double*)d_n;
    if (!ok) {
        free_list(L);
        return gexs::set_error(GEXS_ERR_OOM, "line list upload");
    }
    cudaError_t e = cudaSuccess;
    auto put = [&](void* dst, const void* src, size_t n) {
        if (e == cudaSuccess && n) e = cudaMemcpy(dst, src, n, cudaMemcpyDefault);
    };
    if (count > 0) {
        put(d_nu, in->nu, sizeof(double) * count);
        put(d_e, in->elow, w * count);
        put(d_a, in->aif, w * count);
        if (!compact) put(d_g, in->gns, sizeof(int32_t) * count);
        if (press) {
            put(d_gam, in->gamma, w * count);
            put(d_n, in->n, w * count);
        }
    }
    put(L.se, state_energy, sizeof(double) * nstates);
    put(L.sg, state_g, sizeof(int32_t) * nstates);
    if (e != cudaSuccess) {
        free_list(L);
        return gexs::cuda_error(e, "line list upload");
    }
    /* the resident Q(T) table */
    {
        std::vector<double> temps(kQPoints), q;
        for (int k = 0; k < kQPoints; ++k) temps[k] = std::exp(qtab_lnt(k));
        const int st = exact_partitions(s, L, temps, q, L.d_qtab);
        if (st) {
            free_list(L);
            return st;
        }
        L.lnq.resize(kQPoints);
        for (int k = 0; k < kQPoints; ++k) L.lnq[k] = std::log(q[k]);
    }
    std::lock_guard<std::mutex> g(s->mu);
    s->lists.push_back(L);
    s->resident += bytes;
    *list_id = (int)s->lists.size() - 1;
    return GEXS_OK;
}

int gexs_server_submit(gexs_server* s, const gexs_request* r, uint64_t* ticket)
{
    if (!s || !r || !ticket) return gexs::set_error(GEXS_ERR_INVALID, "gexs_server_submit: arguments");
    gexs_job probe;
    int st = gexs_job_init(&probe, r->convention, r->profile, r->temperature, r->pressure, 1.0, 1.0,
                           r->ref_temp > 0 ? r->ref_temp : 296.0, r->ref_press, r->half_width,
                           r->cutoff, r->nu_start, r->dnu, r->grid_points);
    if (st) return st;
    if (r->precision != GEXS_FP32 && r->precision != GEXS_FP64)
        return gexs::set_error(GEXS_ERR_INVALID, "precision");
    if (r->profile == GEXS_VOIGT_QUAD && r->quad_nodes != 16 && r->quad_nodes != 32)
        return gexs::set_error(GEXS_ERR_INVALID, "quad_nodes");
    Req* q = new Req();
    q->r = *r;
    if (!(q->r.ref_temp > 0)) q->r.ref_temp = 296.0;
    if (q->r.profile != GEXS_VOIGT_QUAD) q->r.quad_nodes = 16;
    std::memset(&q->info, 0, sizeof(q->info));
    q->info.evals = -1;
    {
        /* admission counts the output and the scratch of the job's launch
         * (prep arrays, tables, slice rows), all from the context's pool */
        {
            std::lock_guard<std::mutex> g(s->mu);
            if (r->list_id < 0 || r->list_id >= (int)s->lists.size()) {
                delete q;
                return gexs::set_error(GEXS_ERR_INVALID, "unknown list_id");
            }
            const List& L = s->lists[r->list_id];
            probe.lines = L.lines;
        }
        bool press = r->profile == GEXS_VOIGT || r->profile == GEXS_VOIGT_QUAD;
        if (press && !probe.lines.gamma) {
            delete q;
            return gexs::set_error(GEXS_ERR_INVALID, "list has no broadening for this profile");
        }
        probe.precision = q->r.precision;
        probe.quad_nodes = q->r.quad_nodes;
        double placeholder = 0.0;          /* never written: sizes only */
        probe.out = &placeholder;
        size_t scratch = 0;
        st = gexs::run_scratch_bytes(s->ctx, &probe, 1, nullptr, &scratch);
        if (st) { delete q; return st; }
        q->bytes = output_bytes(*r) + scratch;
    }
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->resident + q->bytes > s->budget) {
            delete q;
            return gexs::set_error(GEXS_ERR_ADMISSION, "request output and scratch exceed the HBM budget");
        }
        if (s->stop) { delete q; return gexs::set_error(GEXS_ERR_SHUTDOWN, "server stopping"); }
        q->id = s->next_id++;
        q->info.submit_ms = s->now_ms();
        s->reqs[q->id] = q;
        s->pending.push_back(q);
        s->n_submitted++;
        s->kick = true;
        *ticket = q->id;
    }
    s->cv_work.notify_one();
    return GEXS_OK;
}

int gexs_server_poll(gexs_server* s, uint64_t ticket)
{
    if (!s) return GEXS_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return gexs::set_error(GEXS_ERR_INVALID, "unknown ticket");
    int state = it->second->state;
    if (state == RQ_DONE) return GEXS_OK;
    if (state == RQ_FAILED) return it->second->status;
    return GEXS_ERR_NOT_READY;
}

int gexs_server_wait(gexs_server* s, uint64_t ticket, int timeout_ms, double* h_out,
                     gexs_request_info* info)
{
    if (!s) return GEXS_ERR_INVALID;
    Req* r = nullptr;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return gexs::set_error(GEXS_ERR_INVALID, "unknown ticket");
        r = it->second;
        auto ready = [&] { return r->state == RQ_DONE || r->state == RQ_FAILED; };
        if (timeout_ms < 0) s->cv_done.wait(lk, ready);
        else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return gexs::set_error(GEXS_ERR_TIMEOUT, "request not finished");
        s->reqs.erase(it);
    }
    int status = r->state == RQ_DONE ? GEXS_OK : r->status;
    cudaSetDevice(s->device);
    if (r->d_out) {
        cudaStream_t c = take_copy_stream(s);
        cudaError_t e = cudaSuccess;
        if (r->done) e = cudaStreamWaitEvent(c, r->done, 0);
        if (e == cudaSuccess && h_out && !status)
            e = cudaMemcpyAsync(h_out, r->d_out, output_bytes(r->r), cudaMemcpyDeviceToHost, c);
        cudaError_t e2 = cudaFreeAsync(r->d_out, c);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaStreamSynchronize(c);
        give_copy_stream(s, c);
        if (e != cudaSuccess && !status) status = gexs::cuda_error(e, "result copy");
        r->d_out = nullptr;
    }
    bool last_of_batch = false;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->inflight--;
        s->inflight_bytes -= r->bytes;
        r->info.fetched_ms = s->now_ms();
        r->info.status = status;
        s->kick = true;
        if (r->done) {
            auto e = s->ev_refs.find(r->done);
            if (e != s->ev_refs.end() && --e->second == 0) {
                s->ev_refs.erase(e);
                last_of_batch = true;
            }
        }
    }
    if (r->done && last_of_batch) cudaEventDestroy(r->done);
    if (info) *info = r->info;
    delete r;
    s->cv_work.notify_one();
    if (status) return gexs::set_error(status, "request failed");
    return GEXS_OK;
}

int gexs_server_partition(gexs_server* s, int list_id, double temperature, double* q,
                          int* from_table)
{
    if (!s || !q || !(temperature > 0.0))
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_server_partition: arguments");
    const List* L = nullptr;
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (list_id < 0 || list_id >= (int)s->lists.size())
            return gexs::set_error(GEXS_ERR_INVALID, "unknown list_id");
        L = &s->lists[list_id];
    }
    cudaSetDevice(s->device);
    const bool tab = q_from_table(*L, temperature, q);
    if (from_table) *from_table = tab ? 1 : 0;
    if (tab) return GEXS_OK;
    std::vector<double> t(1, temperature), v;
    const int st = exact_partitions(s, *L, t, v);
    if (st) return st;
    *q = v[0];
    return GEXS_OK;
}

int gexs_server_stats(gexs_server* s, int64_t* submitted, int64_t* completed, int64_t* batches,
                      int64_t* inflight_bytes)
{
    if (!s) return GEXS_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    if (submitted) *submitted = s->n_submitted;
    if (completed) *completed = s->n_completed;
    if (batches) *batches = s->n_batches;
    if (inflight_bytes) *inflight_bytes = (int64_t)s->inflight_bytes;
    return GEXS_OK;
}

}  // extern "C"
