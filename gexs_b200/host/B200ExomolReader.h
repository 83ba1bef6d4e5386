/*
 * B200ExomolReader.h — a StateReader (Readers/StateReader.h) whose parsing
 * runs on the GPU: the drop-in beside the reference's ExomolStateReader
 * (Readers/Exomol/ExomolStateReader.h), with the same constructor arguments.
 *
 * The .states file is parsed on the device at construction and Q(T) is a
 * device reduction over it (gexs_partition).  OpenFile parses the whole
 * .trans file on the device (gexs_exomol_parse_trans); ReadNextState then
 * streams the records in file order, as ExomolStateReader does
 * (ExomolStateReader.cpp:132-172), from a host copy.  device_lines() gives
 * the parsed list in device memory for callers that hand it straight to the
 * compute path (gexs_run, B200Manager) instead of streaming it through the
 * host.  Errors are kept in last_status(); no member prints or exits.
 */
#pragma once
#include <string>
#include <vector>
#ifdef GEXS_USE_REFERENCE_STATEREADER
/* compile inside the GEXS tree against its own Readers/StateReader.h (put
 * Readers/ on the include path; angle brackets skip this directory) */
#include <StateReader.h>
#else
#include "StateReader.h"
#endif
#include "../../include/gexs_b200.h"

class B200ExomolReader : public StateReader {
public:
    /* pressure is kept for signature parity and unused, as in the
     * reference; broad_mode GEXS_BROAD_DEFAULTS reproduces the reference's
     * broadening (the defaults for every line), GEXS_BROAD_BY_J the
     * intended J'' lookup; sort_by_nu orders the transitions by nu */
    B200ExomolReader(std::string pFilename = "", double partition = -1.0, double pressure = 1.0,
                     std::string broadeners = "", double default_gamma = 0.1,
                     double default_n = 0.1, int device = 0,
                     int broad_mode = GEXS_BROAD_DEFAULTS, bool sort_by_nu = false);
    /* not virtual, like ~StateReader: delete a B200ExomolReader* */
    ~B200ExomolReader();

    bool OpenFile(std::string pFilename) override;
    bool CloseFile() override;
    bool ReadNextState(double& nu, double& gns, double& e_i, double& aif, double& gam,
                       double& n) override;
    bool ReadNextState(double& nu, double& gns, double& e_i, double& aif) override;
    double ComputePartition(double temperature) override;

    /* the open file's lines in device memory (valid until CloseFile) */
    gexs_lines device_lines() const;
    int64_t num_states() const { return states_.count; }
    int64_t num_transitions() const { return lines_.count; }
    int last_status() const { return status_; }

private:
    int fail(int st) { if (!status_) status_ = st; return st; }
    gexs_ctx* ctx_ = nullptr;
    gexs_state_table states_ = {};
    gexs_line_table lines_ = {};
    std::string broad_text_;
    int broad_mode_;
    bool sort_;
    double default_gam_, default_n_;
    int status_ = GEXS_OK;
    /* host copy streamed by ReadNextState */
    std::vector<double> h_nu_, h_e_, h_a_, h_gam_, h_n_;
    std::vector<int32_t> h_g_;
    size_t cursor_ = 0;
};
