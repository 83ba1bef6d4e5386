/*
 * gexs_output.cpp — cross-section output (the reference's
 * BaseProfile::OutputProfile, Profiles/BaseProfile.cpp:269-301, prints every
 * bin with printf on one thread).
 *
 * GEXS_OUT_TEXT writes exactly the reference's text for one (T, P) pair:
 *     "-------T=%12.6f K--------P=%12.6f atm---------\n\n"
 *     "[%i] %12.6f %13.8E\n" per bin, freq_j = nu_start + double(j)*dnu
 *     (BaseProfile.cpp:17-21), then "\n"
 * with the same libc formatting, but on all host threads: the grid is split
 * into chunks formatted in parallel and written in order.
 * GEXS_OUT_BINARY writes a 64-byte header (magic "GEXSSIG1", n, nu_start,
 * dnu, T, P, index, zero padding) followed by the n float64 values.
 * sigma may be host or device memory (a device array is copied out first).
 */
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/gexs_b200.h"

namespace {

struct SigHeader {
    char    magic[8];
    int64_t n;
    double  nu_start, dnu, temperature, pressure;
    int32_t index, reserved;
    int64_t pad;
};
static_assert(sizeof(SigHeader) == 64, "header is 64 bytes");

void format_chunk(int index, double nu_start, double dnu, const double* s, int64_t j0, int64_t j1,
                  std::string& out)
{
    char line[96];
    out.clear();
    out.reserve((size_t)(j1 - j0) * 36);
    for (int64_t j = j0; j < j1; ++j) {
        const double f = nu_start + double(j) * dnu;
        const int len = std::snprintf(line, sizeof line, "[%i] %12.6f %13.8E\n", index, f, s[j]);
        out.append(line, (size_t)len);
    }
}

}  // namespace

extern "C" int gexs_write_sigma(const char* path, int format, int append, int index,
                                double temperature, double pressure, double nu_start, double dnu,
                                int64_t n, const double* sigma, int nthreads)
{
    if (!path || n < 0 || (n > 0 && !sigma) || (format != GEXS_OUT_BINARY && format != GEXS_OUT_TEXT))
        return GEXS_ERR_INVALID;
    /* a device array is copied to the host first */
    std::vector<double> host;
    const double* s = sigma;
    cudaPointerAttributes attr;
    if (n > 0 && cudaPointerGetAttributes(&attr, sigma) == cudaSuccess &&
        attr.type == cudaMemoryTypeDevice) {
        host.resize((size_t)n);
        if (cudaMemcpy(host.data(), sigma, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
            return GEXS_ERR_CUDA;
        s = host.data();
    }
    cudaGetLastError();   /* a host pointer may leave an error from the query */
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return GEXS_ERR_INVALID;
    bool ok = true;
    if (format == GEXS_OUT_BINARY) {
        SigHeader h;
        std::memset(&h, 0, sizeof h);
        std::memcpy(h.magic, "GEXSSIG1", 8);
        h.n = n; h.nu_start = nu_start; h.dnu = dnu; h.temperature = temperature;
        h.pressure = pressure; h.index = index;
        ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
             (n == 0 || std::fwrite(s, sizeof(double), (size_t)n, f) == (size_t)n);
    } else {
        char head[160];
        const int hl = std::snprintf(head, sizeof head,
                                     "-------T=%12.6f K--------P=%12.6f atm---------\n\n",
                                     temperature, pressure);
        ok = std::fwrite(head, 1, (size_t)hl, f) == (size_t)hl;
        int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
        nt = (int)std::min<int64_t>(nt, std::max<int64_t>(1, n / 4096));
        const int64_t per = 1 << 18;        /* bins per chunk and round */
        std::vector<std::string> bufs((size_t)nt);
        for (int64_t r0 = 0; ok && r0 < n; r0 += per * nt) {
            std::vector<std::thread> th;
            for (int t = 0; t < nt; ++t) {
                const int64_t a = std::min(n, r0 + per * t), b = std::min(n, a + per);
                th.emplace_back(format_chunk, index, nu_start, dnu, s, a, b, std::ref(bufs[(size_t)t]));
            }
            for (auto& x : th) x.join();
            for (const std::string& b : bufs)
                if (ok && !b.empty()) ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
        }
        if (ok) ok = std::fputc('\n', f) != EOF;
    }
    if (std::fclose(f) != 0) ok = false;
    return ok ? GEXS_OK : GEXS_ERR_INVALID;
}
