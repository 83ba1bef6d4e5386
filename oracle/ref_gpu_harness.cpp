/*
 * ref_gpu_harness.cpp — runs the reference's GPU manager (GpuManager,
 * Managers/Accel/GPU/GPUManager.cpp, with its kernels from
 * compute/CUDA/cross_kernal_v2.cu) for one Voigt (T, P) pair the way
 * BaseProfile drives it (Profiles/BaseProfile.cpp:100-116, 269-301).
 * TEST/BENCH INFRASTRUCTURE ONLY: the timed reference-GPU arm and a checker
 * of the reference-GPU convention; the product never links or calls it.
 *
 *   gexsref_gpu <in.bin> <out.bin>
 *   in:  int64 n, int64 npts, int64 reps, int64 budget_bytes,
 *        double nu_start, dnu, T, P, Q, mass, ref_temp, ref_press, half_width,
 *        then n doubles each of E'', nu, A, n int32 g', n doubles gamma, n doubles n
 *   out: npts doubles, the slot after the last repetition
 *   stdout (last line): {"ms": [...]} per repetition, CUDA events on the
 *   legacy stream around ExecuteCrossSection (the manager launches on a
 *   blocking stream of its own, so the events bracket its kernels).
 *
 * The manager is given budget_bytes (BaseManager::InitializeMemory) instead
 * of 95% of the device, which its constructor would otherwise reserve.
 * Every repetition re-runs TransferFreq and TransferVectors: the kernels
 * overwrite gamma in place (cross_kernal_v2.cu:143) and TransferVectors
 * resets the result-slot index (GPUManager.cpp:149).
 */
#include <cstdint>
#include <cstdio>
#include <vector>
#include <cuda_runtime.h>
#include "GPUManager.h"

namespace {
struct Harness : public GpuManager {
    Harness() : GpuManager(VOIGT, 0) {}
    void budget(size_t b) { InitializeMemory(b); }
};

template <typename T>
bool rd(FILE* f, T* p, size_t n) { return std::fread(p, sizeof(T), n, f) == n; }
}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3) { std::fprintf(stderr, "usage: gexsref_gpu in.bin out.bin\n"); return 2; }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int64_t hdr[4];
    double par[9];
    if (!rd(f, hdr, 4) || !rd(f, par, 9)) return 2;
    const int64_t n = hdr[0], npts = hdr[1], reps = hdr[2];
    const size_t budget = (size_t)hdr[3];
    std::vector<double> e(n), nu(n), a(n), gam(n), nx(n);
    std::vector<int> g(n);
    if (!rd(f, e.data(), n) || !rd(f, nu.data(), n) || !rd(f, a.data(), n) || !rd(f, g.data(), n) ||
        !rd(f, gam.data(), n) || !rd(f, nx.data(), n)) return 2;
    std::fclose(f);
    const double nu0 = par[0], dnu = par[1], T = par[2], P = par[3], Q = par[4], mass = par[5];
    const double ref_t = par[6], ref_p = par[7], hw = par[8];

    Harness m;
    m.budget(budget);
    m.InitializeVectors((int)npts, 1);
    if ((int64_t)m.GetNtrans() < n) { std::fprintf(stderr, "budget too small\n"); return 3; }
    m.InitializeConstants(hw, T, Q, dnu, mass, P, ref_t, ref_p);
    std::vector<double> freq(npts), zero(npts, 0.0), out(npts, 0.0);
    for (int64_t j = 0; j < npts; ++j) freq[j] = nu0 + (double)j * dnu;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> ms;
    for (int64_t r = 0; r < reps; ++r) {
        m.TransferFreq(freq.data(), zero.data(), (int)npts);
        m.TransferVectors((size_t)n, e.data(), nu.data(), a.data(), g.data(), gam.data(), nx.data());
        cudaEventRecord(e0, 0);
        m.ExecuteCrossSection((int)npts, (int)n, 0, T, P, Q);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms.push_back(t);
    }
    m.TransferResults(freq.data(), out.data(), (int)npts, 0);
    FILE* o = std::fopen(argv[2], "wb");
    if (!o || std::fwrite(out.data(), sizeof(double), npts, o) != (size_t)npts) return 2;
    std::fclose(o);
    std::printf("\n{\"ms\": [");
    for (size_t i = 0; i < ms.size(); ++i) std::printf("%s%.6f", i ? ", " : "", ms[i]);
    std::printf("]}\n");
    cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? 0 : 4;
}
