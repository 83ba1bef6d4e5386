/*
 * boundary_driver.cpp — drives the two drop-ins through the reference's
 * own base-class pointers, the way Profiles/BaseProfile.cpp does.
 * TEST INFRASTRUCTURE ONLY: the product never links or runs it.
 *
 * Compiled against the reference's headers alone (Readers/StateReader.h,
 * Managers/BaseManager.h); the objects come from boundary_factory.cpp,
 * built either on gexs_b200/host/'s headers with the product library's
 * classes (binary drop-in) or from the drop-in sources compiled against
 * the reference's headers (source drop-in).  Every virtual of both
 * interfaces is called through StateReader* / BaseManager*:
 *   reader  ComputePartition (BaseProfile.cpp:71,95), OpenFile (:144),
 *           ReadNextState 6 args (:148), CloseFile (:234), ReadNextState
 *           4 args (Doppler/DopplerProfile.cpp:57)
 *   manager InitializeVectors (:65), TransferFreq (:67), InitializeConstants
 *           (:71), TransferVectors + ExecuteCrossSection per (T, P) pair
 *           (:100-116), ReadyForWork, TransferResults (:279-281), Cleanup,
 *           and the deprecated 3-argument ExecuteCrossSection /
 *           TransferResults and 1-argument InitializeVectors.
 *
 *   boundary_<so|src> states trans outdir T1 P1 T2 P2 mass nu0 dnu G device
 * writes outdir/records.bin (n x {nu, gns, e_i, aif, gam, n} doubles in read
 * order), outdir/sigma0.bin and sigma1.bin (G doubles, pairs 1 and 2), and
 * prints one JSON line with the scalar results.
 */
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "StateReader.h"
#include "BaseManager.h"

StateReader* boundary_make_reader(const char* states_path, int device);
void boundary_free_reader(StateReader* r);
BaseManager* boundary_make_manager(int profile, int device, size_t memory_bytes);
void boundary_free_manager(BaseManager* m);

namespace {
bool write_doubles(const std::string& path, const std::vector<double>& v)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(v.data(), sizeof(double), v.size(), f) == v.size();
    return std::fclose(f) == 0 && ok;
}
}  // namespace

int main(int argc, char** argv)
{
    if (argc != 13) {
        std::fprintf(stderr, "usage: %s states trans outdir T1 P1 T2 P2 mass nu0 dnu G device\n", argv[0]);
        return 2;
    }
    const std::string outdir = argv[3];
    const double T1 = std::atof(argv[4]), P1 = std::atof(argv[5]);
    const double T2 = std::atof(argv[6]), P2 = std::atof(argv[7]);
    const double mass = std::atof(argv[8]), nu0 = std::atof(argv[9]), dnu = std::atof(argv[10]);
    const int G = std::atoi(argv[11]), device = std::atoi(argv[12]);

    /* ------------------------------------------------------------ reader */
    StateReader* reader = boundary_make_reader(argv[1], device);
    const double q1 = reader->ComputePartition(T1);
    const double q2 = reader->ComputePartition(T2);
    const bool opened = reader->OpenFile(argv[2]);
    std::vector<double> rec, e, nu, aif, gam, nn;
    std::vector<int> gns;
    double a, b, c, d, g, n;
    while (reader->ReadNextState(a, b, c, d, g, n)) {
        rec.push_back(a); rec.push_back(b); rec.push_back(c);
        rec.push_back(d); rec.push_back(g); rec.push_back(n);
        nu.push_back(a); gns.push_back((int)b); e.push_back(c); aif.push_back(d);
        gam.push_back(g); nn.push_back(n);
    }
    const bool closed = reader->CloseFile();
    /* the 4-argument form on a second pass: the first record again */
    const bool reopened = reader->OpenFile(argv[2]);
    double f4[4] = {0, 0, 0, 0};
    const bool got4 = reader->ReadNextState(f4[0], f4[1], f4[2], f4[3]);
    const bool closed2 = reader->CloseFile();
    const bool match4 = got4 && !rec.empty() && f4[0] == rec[0] && f4[1] == rec[1] &&
                        f4[2] == rec[2] && f4[3] == rec[3];
    boundary_free_reader(reader);
    write_doubles(outdir + "/records.bin", rec);

    /* ----------------------------------------------------------- manager */
    std::vector<double> freq(G), intens(G, 0.0), s0(G, 0.0), s1(G, 0.0);
    for (int j = 0; j < G; ++j) freq[j] = nu0 + j * dnu;
    const size_t ntr = nu.size();
    BaseManager* m = boundary_make_manager(VOIGT, device, (size_t)1 << 28);
    m->InitializeVectors(G, 2);
    m->TransferFreq(freq.data(), intens.data(), G);
    m->InitializeConstants(0.0, T1, q1, dnu, mass, P1, 296.0, 1.0);
    const size_t cap = m->GetNtrans();
    m->TransferVectors(ntr, e.data(), nu.data(), aif.data(), gns.data(), gam.data(), nn.data());
    m->ExecuteCrossSection(G, (int)ntr, 0, T1, P1, q1);
    /* one of two result slots used: ready for the next pair */
    const bool ready = m->ReadyForWork();
    m->ExecuteCrossSection(G, (int)ntr, 0, T2, P2, q2);
    m->TransferResults(freq.data(), s0.data(), G, 0);
    m->TransferResults(freq.data(), s1.data(), G, 1);
    m->Cleanup();
    boundary_free_manager(m);
    write_doubles(outdir + "/sigma0.bin", s0);
    write_doubles(outdir + "/sigma1.bin", s1);

    /* the deprecated entry points on a second manager: the 1-argument
     * InitializeVectors, then the 3-argument ExecuteCrossSection and
     * TransferResults, which the drop-in rejects (its state records the
     * error) without touching the caller's buffer */
    BaseManager* m2 = boundary_make_manager(VOIGT, device, (size_t)1 << 24);
    m2->InitializeVectors(G);
    const size_t cap2 = m2->GetNtrans();
    m2->ExecuteCrossSection(G, 0, 0);
    std::vector<double> untouched(G, 7.0);
    m2->TransferResults(freq.data(), untouched.data(), G);
    const bool kept = untouched[0] == 7.0 && untouched[G - 1] == 7.0;
    m2->Cleanup();
    boundary_free_manager(m2);

    std::printf("{\"q1\": %.17g, \"q2\": %.17g, \"opened\": %d, \"records\": %zu, \"closed\": %d, "
                "\"reopened\": %d, \"got4\": %d, \"match4\": %d, \"closed2\": %d, "
                "\"ntrans_capacity\": %zu, \"ready\": %d, \"ntrans_capacity2\": %zu, "
                "\"deprecated_left_buffer\": %d}\n",
                q1, q2, (int)opened, ntr, (int)closed, (int)reopened, (int)got4, (int)match4,
                (int)closed2, cap, (int)ready, cap2, (int)kept);
    return 0;
}
