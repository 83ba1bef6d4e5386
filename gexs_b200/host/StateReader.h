/*
 * StateReader.h — the reference's reader interface (Readers/StateReader.h),
 * re-declared with the same members, virtual functions and declaration order
 * so that an object of a class built on this header is used unchanged
 * through the reference's own StateReader*: BaseProfile streams transitions
 * through ReadNextState (Profiles/BaseProfile.cpp:143-166) and asks
 * ComputePartition for Q(T) per (T, P) pair (:91-98).  The destructor is
 * not virtual, as in Readers/StateReader.h:12 (a virtual one would add two
 * vtable slots in front of OpenFile); an object is therefore destroyed
 * through its own class, never through a StateReader*.
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
    ~StateReader() {}
    virtual bool OpenFile(std::string pFilename) = 0;
    virtual bool CloseFile() = 0;
    virtual bool ReadNextState(double& nu, double& gns, double& e_i, double& aif, double& gam,
                               double& n) = 0;
    virtual bool ReadNextState(double& nu, double& gns, double& e_i, double& aif) = 0;
    virtual double ComputePartition(double temperature) = 0;
};
