/*
 * B200ExomolReader.cpp — StateReader over the GPU ExoMol ingest, and its
 * flat C view (include/gexs_reader.h).
 */
#include "B200ExomolReader.h"

#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>
#include "../../include/gexs_reader.h"

namespace {

bool read_all(const std::string& path, std::vector<char>& buf)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(buf.data(), 1, (size_t)n, f) : 0;
    std::fclose(f);
    return (long)got == n;
}

}  // namespace

B200ExomolReader::B200ExomolReader(std::string pFilename, double partition, double,
                                   std::string broadeners, double default_gamma,
                                   double default_n, int device, int broad_mode, bool sort_by_nu)
    : StateReader(pFilename, partition), broad_mode_(broad_mode), sort_(sort_by_nu),
      default_gam_(default_gamma), default_n_(default_n)
{
    int st = gexs_ctx_create(device, &ctx_);
    if (st) { fail(st); return; }
    std::vector<char> text;
    if (!read_all(pFilename, text)) { fail(GEXS_ERR_INVALID); return; }
    st = gexs_exomol_parse_states(ctx_, text.data(), (int64_t)text.size(), &states_);
    if (st) { fail(st); return; }
    /* a missing broadener file means defaults (ExomolStateReader.cpp:42-46) */
    std::vector<char> b;
    if (!broadeners.empty() && read_all(broadeners, b)) broad_text_.assign(b.begin(), b.end());
}

B200ExomolReader::~B200ExomolReader()
{
    CloseFile();
    gexs_state_table_free(&states_);
    if (ctx_) gexs_ctx_destroy(ctx_);
}

bool B200ExomolReader::OpenFile(std::string pFilename)
{
    if (status_) return false;
    CloseFile();
    std::vector<char> text;
    if (!read_all(pFilename, text)) { fail(GEXS_ERR_INVALID); return false; }
    int st = gexs_exomol_parse_trans(ctx_, &states_, text.data(), (int64_t)text.size(),
                                     broad_text_.data(), (int64_t)broad_text_.size(), broad_mode_,
                                     default_gam_, default_n_, sort_ ? 1 : 0, &lines_);
    if (st) { fail(st); return false; }
    const size_t n = (size_t)lines_.count;
    h_nu_.resize(n); h_e_.resize(n); h_a_.resize(n); h_gam_.resize(n); h_n_.resize(n); h_g_.resize(n);
    bool ok = true;
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        if (ok && bytes) ok = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
    };
    d2h(h_nu_.data(), lines_.nu, n * 8); d2h(h_e_.data(), lines_.elow, n * 8);
    d2h(h_a_.data(), lines_.aif, n * 8); d2h(h_g_.data(), lines_.gns, n * 4);
    d2h(h_gam_.data(), lines_.gamma, n * 8); d2h(h_n_.data(), lines_.n, n * 8);
    if (!ok) { fail(GEXS_ERR_CUDA); return false; }
    cursor_ = 0;
    open_file = true;
    m_filename = pFilename;
    return true;
}

bool B200ExomolReader::CloseFile()
{
    gexs_line_table_free(&lines_);
    h_nu_.clear(); h_e_.clear(); h_a_.clear(); h_gam_.clear(); h_n_.clear(); h_g_.clear();
    cursor_ = 0;
    open_file = false;
    return true;
}

/* ExomolStateReader.cpp:132-166: nu = E_u - E_l, gns = g_u, e_i = E_l */
bool B200ExomolReader::ReadNextState(double& nu, double& gns, double& e_i, double& aif,
                                     double& gam, double& n)
{
    if (cursor_ >= h_nu_.size()) return false;
    const size_t i = cursor_++;
    nu = h_nu_[i]; gns = (double)h_g_[i]; e_i = h_e_[i]; aif = h_a_[i];
    gam = h_gam_[i]; n = h_n_[i];
    return true;
}

bool B200ExomolReader::ReadNextState(double& nu, double& gns, double& e_i, double& aif)
{
    double g = 0.0, x = 0.0;
    return ReadNextState(nu, gns, e_i, aif, g, x);
}

/* Q(T) = sum g exp(-c2 E / T) over the states (exomol_functions.cpp:50-73) */
double B200ExomolReader::ComputePartition(double temperature)
{
    double q = 0.0;
    if (status_) return 0.0;
    int st = gexs_partition(ctx_, states_.energy, states_.g, states_.count, &temperature, 1, &q);
    if (st) { fail(st); return 0.0; }
    partition = q;
    return q;
}

gexs_lines B200ExomolReader::device_lines() const
{
    gexs_lines l;
    std::memset(&l, 0, sizeof(l));
    l.format = GEXS_LINES_FP64;
    l.nu = lines_.nu; l.elow = lines_.elow; l.aif = lines_.aif; l.gns = lines_.gns;
    l.gamma = lines_.gamma; l.n = lines_.n; l.count = lines_.count;
    return l;
}

/* ------------------------------------------------------------ C wrappers */
struct gexs_reader { B200ExomolReader* r; };

extern "C" {

int gexs_reader_create(const char* states_path, const char* broad_path, double default_gamma,
                       double default_n, int device, int broad_mode, int sort_by_nu,
                       gexs_reader** out)
{
    if (!states_path || !out) return GEXS_ERR_INVALID;
    *out = nullptr;
    B200ExomolReader* r = new B200ExomolReader(states_path, -1.0, 1.0, broad_path ? broad_path : "",
                                               default_gamma, default_n, device, broad_mode,
                                               sort_by_nu != 0);
    const int st = r->last_status();
    if (st) { delete r; return st; }
    *out = new gexs_reader{r};
    return GEXS_OK;
}

int gexs_reader_open(gexs_reader* h, const char* trans_path, int64_t* ntrans)
{
    if (!h || !trans_path) return GEXS_ERR_INVALID;
    if (!h->r->OpenFile(trans_path)) return h->r->last_status() ? h->r->last_status() : GEXS_ERR_INVALID;
    if (ntrans) *ntrans = h->r->num_transitions();
    return GEXS_OK;
}

int gexs_reader_next(gexs_reader* h, double* nu, double* gns, double* e_i, double* aif,
                     double* gam, double* n, int* more)
{
    if (!h || !nu || !gns || !e_i || !aif || !gam || !n || !more) return GEXS_ERR_INVALID;
    *more = h->r->ReadNextState(*nu, *gns, *e_i, *aif, *gam, *n) ? 1 : 0;
    return GEXS_OK;
}

int gexs_reader_partition(gexs_reader* h, double temperature, double* q)
{
    if (!h || !q) return GEXS_ERR_INVALID;
    *q = h->r->ComputePartition(temperature);
    return h->r->last_status();
}

int gexs_reader_device_lines(gexs_reader* h, gexs_lines* out)
{
    if (!h || !out) return GEXS_ERR_INVALID;
    *out = h->r->device_lines();
    return GEXS_OK;
}

int gexs_reader_close(gexs_reader* h)
{
    if (!h) return GEXS_ERR_INVALID;
    h->r->CloseFile();
    return GEXS_OK;
}

int gexs_reader_destroy(gexs_reader* h)
{
    if (!h) return GEXS_OK;
    delete h->r;
    delete h;
    return GEXS_OK;
}

}  // extern "C"
