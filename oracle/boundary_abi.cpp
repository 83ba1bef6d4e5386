/*
 * boundary_abi.cpp — layout probe of the two plug-in base classes.
 * TEST INFRASTRUCTURE ONLY: the product never links or runs it.
 *
 * Prints, for StateReader (Readers/StateReader.h:6-19) and BaseManager
 * (Managers/BaseManager.h:6-38) as declared by whichever headers it is
 * compiled against, the vtable byte offset of every virtual function (the
 * Itanium C++ ABI stores a pointer to a virtual member function as 1 +
 * that offset), the byte offset of every member it can name, and the
 * class sizes.  oracle/Makefile builds it twice, against the reference's
 * own headers and against gexs_b200/host/; a drop-in built on the second
 * is usable through the first when the two outputs are equal.
 *
 *   boundary_abi   -> one JSON object on stdout
 */
#include <cstdio>
#include <cstring>
#include "StateReader.h"
#include "BaseManager.h"

namespace {

template <typename M>
long first_word(M m)
{
    long w[2] = {0, 0};
    static_assert(sizeof(M) <= sizeof(w), "member pointer larger than two words");
    std::memcpy(w, &m, sizeof(M));
    return w[0];
}

/* vtable offset of a virtual member function */
template <typename M>
long slot(M m) { return first_word(m) - 1; }

/* protected data members, named through a derived class */
struct SR : StateReader {
    static long filename() { return first_word(&SR::m_filename); }
    static long part() { return first_word(&SR::partition); }
    static long open() { return first_word(&SR::open_file); }
};
struct BM : BaseManager {
    static long ntrans() { return first_word(&BM::N_trans); }
    static long prof() { return first_word(&BM::profile); }
};

}  // namespace

int main()
{
    typedef bool (StateReader::*Next6)(double&, double&, double&, double&, double&, double&);
    typedef bool (StateReader::*Next4)(double&, double&, double&, double&);
    typedef void (BaseManager::*IV1)(int);
    typedef void (BaseManager::*IV2)(int, int);
    typedef void (BaseManager::*EX3)(int, int, int);
    typedef void (BaseManager::*EX6)(int, int, int, double, double, double);
    typedef void (BaseManager::*TR3)(double*, double*, int);
    typedef void (BaseManager::*TR4)(double*, double*, int, int);
    std::printf("{\"StateReader\": {\"OpenFile\": %ld, \"CloseFile\": %ld, \"ReadNextState6\": %ld, "
                "\"ReadNextState4\": %ld, \"ComputePartition\": %ld, \"m_filename\": %ld, "
                "\"partition\": %ld, \"open_file\": %ld, \"sizeof\": %ld}, ",
                slot(&StateReader::OpenFile), slot(&StateReader::CloseFile),
                slot(static_cast<Next6>(&StateReader::ReadNextState)),
                slot(static_cast<Next4>(&StateReader::ReadNextState)),
                slot(&StateReader::ComputePartition), SR::filename(), SR::part(), SR::open(),
                (long)sizeof(StateReader));
    std::printf("\"BaseManager\": {\"InitializeVectors1\": %ld, \"InitializeVectors2\": %ld, "
                "\"InitializeConstants\": %ld, \"TransferVectors\": %ld, \"TransferFreq\": %ld, "
                "\"ExecuteCrossSection3\": %ld, \"ExecuteCrossSection6\": %ld, "
                "\"TransferResults3\": %ld, \"TransferResults4\": %ld, \"Cleanup\": %ld, "
                "\"ReadyForWork\": %ld, \"N_trans\": %ld, \"profile\": %ld, \"sizeof\": %ld}}\n",
                slot(static_cast<IV1>(&BaseManager::InitializeVectors)),
                slot(static_cast<IV2>(&BaseManager::InitializeVectors)),
                slot(&BaseManager::InitializeConstants), slot(&BaseManager::TransferVectors),
                slot(&BaseManager::TransferFreq),
                slot(static_cast<EX3>(&BaseManager::ExecuteCrossSection)),
                slot(static_cast<EX6>(&BaseManager::ExecuteCrossSection)),
                slot(static_cast<TR3>(&BaseManager::TransferResults)),
                slot(static_cast<TR4>(&BaseManager::TransferResults)),
                slot(&BaseManager::Cleanup), slot(&BaseManager::ReadyForWork), BM::ntrans(),
                BM::prof(), (long)sizeof(BaseManager));
    return 0;
}
