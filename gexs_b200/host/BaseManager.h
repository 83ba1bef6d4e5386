/*
 * BaseManager.h — the reference's manager plug-in interface, re-declared with
 * identical signatures (Managers/BaseManager.h:6-38) so that B200Manager can
 * be compiled against either this header or the reference's own.  The
 * ProfileType enum equals common/Input.h:10-17.
 */
#pragma once
#include <cstddef>
#include <cstdlib>

#ifndef GEXS_HAVE_REFERENCE_INPUT_H
enum ProfileType {
    GAUSSIAN,
    DOPPLER,
    VOIGT,
    PSUEDO_VOIGT,
    VOIGT_QUAD
};
#endif

class BaseManager {
private:
    size_t available_memory;
    size_t total_memory;
protected:
    size_t N_trans;
    ProfileType profile;
    void InitializeMemory(size_t bytes) { available_memory = bytes; total_memory = bytes; }
    void TrackMemory(size_t bytes) { available_memory -= bytes; }
    void FreeMemory(size_t bytes) { available_memory += bytes; }
    size_t GetAvailableMemory() { return available_memory; }
    BaseManager(ProfileType pprofile) : available_memory(0), total_memory(0), N_trans(0), profile(pprofile) {}
    ~BaseManager() {}
public:
    virtual void InitializeVectors(int Npoints) = 0;
    virtual void InitializeVectors(int Npoints, int num_cs) = 0;
    virtual void InitializeConstants(double half_width, double temperature, double partition,
                                     double dfreq, double meanmass, double pressure = 10.0,
                                     double ref_temp = 296.0, double ref_press = 1.0) = 0;
    virtual void TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                                 int* h_gns, double* h_gamma = NULL, double* h_n = NULL) = 0;
    virtual void TransferFreq(double* h_freq, double* h_intens, int N) = 0;
    virtual void ExecuteCrossSection(int N, int N_ener, int start_idx) = 0;
    virtual void ExecuteCrossSection(int N, int N_ener, int start_idx, double temperature,
                                     double pressure, double partition) = 0;
    virtual void TransferResults(double* h_freq, double* h_intens, int N) = 0;
    virtual void TransferResults(double* h_freq, double* h_intens, int N, int I) = 0;
    virtual void Cleanup() = 0;
    virtual bool ReadyForWork() { return true; }
    size_t GetNtrans() { return N_trans; }
};
