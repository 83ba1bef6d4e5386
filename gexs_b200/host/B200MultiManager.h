/*
 * B200MultiManager.h — the drop-in beside the reference's MultiGpuManager
 * (Managers/Accel/GPU/MultiGPUManager.h), which is the manager
 * BaseProfile::Initialize creates (Profiles/BaseProfile.cpp:61): the same
 * BaseManager protocol over several GPUs, one B200Manager per device.
 *
 * The reference gives each line chunk to whichever GPU is ready and, at
 * TransferResults, adds every GPU's full result grid into the caller's
 * (MultiGPUManager.cpp:59-63,104-126).  Here every chunk is split by bins:
 *  - TransferVectors cuts the grid into one bin range per device with about
 *    equal (line, bin) evaluations (gexs_shard_plan) and copies to each
 *    device only the chunk's lines that can reach its range (the largest
 *    cutoff of the conventions, plus a 4096-bin halo);
 *  - ExecuteCrossSection runs the pair on every device for its bins, with
 *    cuts on multiples of 4096 bins from the pair's start_idx, so each
 *    device computes exactly the tiles, and the sums, of a single launch;
 *  - TransferResults adds the caller's initial grid (TransferFreq) once and
 *    each device's bins of slot I into h_intens (adding, as
 *    MultiGpuManager does; BaseProfile pre-zeroes it, :279-281).
 * Nothing crosses between devices: no collective, each device copies its
 * own bins to the host.  The devices list may name a device more than once
 * (several shards on one GPU).  Objects are destroyed through this class.
 */
#pragma once
#include <cstddef>
#include <vector>
#include "B200Manager.h"

class B200MultiManager : public BaseManager {
public:
    /* devices: CUDA devices, one shard each (empty: every visible device);
     * convention, precision and memory_bytes (per device, 0: half of its
     * free memory) as B200Manager */
    B200MultiManager(ProfileType profile, const std::vector<int>& devices,
                     int convention = GEXS_CONV_REF_GPU, int precision = GEXS_FP64,
                     size_t memory_bytes = 0);
    ~B200MultiManager();

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

    int last_status() const;
    int shards() const { return (int)m_.size(); }
    /* the bin cuts and line ranges of the current chunk (shards + 1 cuts) */
    const std::vector<int64_t>& cuts() const { return bounds_; }

private:
    int fail(int st) { if (!status_) status_ = st; return st; }
    std::vector<B200Manager*> m_;
    int status_ = GEXS_OK;
    int convention_;
    int npoints_ = 0, num_cs_ = 0;
    std::vector<double> freq_, init_;
    double half_width_ = 0.0, dfreq_ = 0.0;
    std::vector<int64_t> bounds_, lo_, hi_;
    int tasks_ = 0;
    /* bins each device wrote, per result slot: [lo, hi) */
    std::vector<std::vector<std::pair<int64_t, int64_t>>> touched_;
};
