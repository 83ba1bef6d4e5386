/*
 * boundary_factory.cpp — constructs the drop-ins for boundary_driver.cpp.
 * TEST INFRASTRUCTURE ONLY: the product never links or runs it.
 *
 * Built on gexs_b200/host/'s re-declared headers (the binary drop-in: the
 * classes come from libgexs_b200.so), or with GEXS_USE_REFERENCE_BASEMANAGER
 * and GEXS_USE_REFERENCE_STATEREADER against the reference's own headers
 * together with the drop-in sources (the source drop-in).  Objects are
 * created and destroyed through their own classes (neither base class has
 * a virtual destructor, Readers/StateReader.h:12, Managers/BaseManager.h:16).
 */
#include "B200ExomolReader.h"
#include "B200Manager.h"

StateReader* boundary_make_reader(const char* states_path, int device)
{
    /* default broadening 0.07 / 0.5 for every line, lines sorted by nu as
     * BaseProfile requires */
    return new B200ExomolReader(states_path, -1.0, 1.0, "", 0.07, 0.5, device,
                                GEXS_BROAD_DEFAULTS, true);
}

void boundary_free_reader(StateReader* r) { delete static_cast<B200ExomolReader*>(r); }

BaseManager* boundary_make_manager(int profile, int device, size_t memory_bytes)
{
    return new B200Manager((ProfileType)profile, device, GEXS_CONV_REF_GPU, GEXS_FP64,
                           memory_bytes);
}

void boundary_free_manager(BaseManager* m) { delete static_cast<B200Manager*>(m); }
