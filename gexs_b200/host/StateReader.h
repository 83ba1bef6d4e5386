/*
 * StateReader.h — the reference's reader interface (Readers/StateReader.h),
 * re-declared with identical signatures so that B200ExomolReader compiles
 * against either this header or the reference's own: BaseProfile streams
 * transitions through ReadNextState (Profiles/BaseProfile.cpp:143-166) and
 * asks ComputePartition for Q(T) per (T, P) pair (:91-98).
 */
#pragma once
#include <string>

class StateReader {
protected:
    std::string m_filename;
    double partition;
    bool open_file;
public:
    StateReader(std::string pFilename = "", double pPartition = -1.0)
        : m_filename(pFilename), partition(pPartition), open_file(false) {}
    virtual ~StateReader() {}
    virtual bool OpenFile(std::string pFilename) = 0;
    virtual bool CloseFile() = 0;
    virtual bool ReadNextState(double& nu, double& gns, double& e_i, double& aif, double& gam,
                               double& n) = 0;
    virtual bool ReadNextState(double& nu, double& gns, double& e_i, double& aif) = 0;
    virtual double ComputePartition(double temperature) = 0;
};
