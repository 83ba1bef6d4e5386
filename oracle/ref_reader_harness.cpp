/*
 * ref_reader_harness.cpp — drives the reference's own ExoMol reader,
 * compiled unmodified from the GEXS sources (Readers/StateReader.cpp,
 * Readers/Exomol/ExomolStateReader.cpp, Readers/Exomol/exomol_functions.cpp,
 * common/Util.cpp), to pin the CPU restatement in ingest_oracle.cpp.
 *
 * TEST INFRASTRUCTURE ONLY (built by oracle/Makefile into oracle/_ref/ as the
 * executable gexsref_reader, so the reference's C++ runtime never shares a
 * process with the caller's):
 *     gexsref_reader STATES TRANS BROAD|- DEFAULT_GAMMA DEFAULT_N OUT
 *     gexsref_reader hitran PAR PRESSURE MIXTURE QREF296 OUT
 * writes the count (int64) and then six float64 arrays of that length (nu,
 * gns, e_i, aif, gamma, n, in file order) to OUT.
 *
 * HITRAN (Readers/HITRAN/HITRANStateReader.cpp): Q(T) comes from the
 * TIPS-2011 Fortran routine bd_tips_2011_, which cannot be compiled here (no
 * Fortran compiler); the harness defines that symbol itself and returns
 * QREF296 for every call, which is the value the reference uses to rebuild
 * A from S (:222-247).  CloseFile ends without a return statement, so the
 * harness never closes or destroys the reader (it leaks one per call), and
 * builds it in zeroed memory (see ref_hitran_read).
 *
 * The bz2 transition reader (Readers/Exomol/bz2_compression) needs libbz2
 * sources this tree does not ship; the three entry points it exports are
 * stubbed here and never reached, since only uncompressed files are read.
 * ReadNextState (ExomolStateReader.cpp:132-172) leaves gamma and n untouched
 * when no broadener file was loaded; the harness passes NaN in for them.
 *
 * OpenFile, CloseFile and the 4-argument ReadNextState end without a return
 * statement (:122, :131, :176), which g++ compiles to a trap.  The harness
 * therefore opens and closes the reader's stream itself (the same access
 * shim as ref_harness.cpp) and never runs the reader's destructor, which
 * calls CloseFile: each call leaks one reader (test code only).
 */
#include <cmath>
#include <cstdlib>
#include <new>
#include <cstdint>
#include <cstdio>
#include <fcntl.h>
#include <unistd.h>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#define private public
#define protected public
#include "ExomolStateReader.h"
#include "HITRANStateReader.h"
#undef private
#undef protected

namespace {
struct Quiet {
    int saved;
    Quiet() {
        fflush(stdout);
        saved = dup(1);
        int dn = open("/dev/null", O_WRONLY);
        if (dn >= 0) { dup2(dn, 1); close(dn); }
    }
    ~Quiet() {
        fflush(stdout);
        if (saved >= 0) { dup2(saved, 1); close(saved); }
    }
};
}  // namespace

extern "C" {

static double g_tips_q = 1.0;
void bd_tips_2011_(int*, double*, int*, double* gi, double* q) { *gi = 1.0; *q = g_tips_q; }

void open_transition_file_bz2_(const char*) {}
void read_trans_lines_bz2_(int*, int*, double*, int* error) { *error = 1; }
void close_transition_file_bz2_() {}

/* every transition the reference reader yields, in file order (at most cap
 * are written); returns the count */
int64_t ref_exomol_read(const char* states_path, const char* trans_path, const char* broad_path,
                        double default_gamma, double default_n, double* nu, double* gns,
                        double* e_i, double* aif, double* gam, double* nexp, int64_t cap)
{
    Quiet q;
    std::cout.flush();
    ExomolStateReader* r = new ExomolStateReader(states_path, -1.0, 1.0,
                                                 broad_path ? broad_path : "", default_gamma,
                                                 default_n);
    r->use_compression = false;            /* what OpenFile sets for a .trans name */
    r->stream.open(trans_path);
    int64_t k = 0;
    for (;;) {
        double a = 0, b = 0, c = 0, d = 0, e = NAN, f = NAN;
        if (!r->ReadNextState(a, b, c, d, e, f)) break;
        if (k < cap) { nu[k] = a; gns[k] = b; e_i[k] = c; aif[k] = d; gam[k] = e; nexp[k] = f; }
        ++k;
    }
    r->stream.close();
    std::cout.flush();
    return k;
}

}  // extern "C"

int64_t ref_hitran_read(const char* path, double pressure, double mixture, double qref,
                        double* nu, double* gns, double* e_i, double* aif, double* gam,
                        double* nexp, int64_t cap)
{
    Quiet q;
    g_tips_q = qref;
    /* partition > 0 skips the constructor's TIPS call; OpenFile asks it for
     * Q(296).  The reader is built in zeroed memory: no constructor sets
     * StateReader::open_file, and OpenFile closes the file again when that
     * member happens to read true (the constructor has already closed it). */
    void* mem = std::calloc(1, sizeof(HITRANStateReader));
    HITRANStateReader* r = new (mem) HITRANStateReader(path, 1.0, pressure, 296.0, mixture);
    r->OpenFile(path);
    int64_t k = 0;
    for (;;) {
        double a = 0, b = 0, c = 0, d = 0, e = 0, f = 0;
        if (!r->ReadNextState(a, b, c, d, e, f)) break;
        if (k < cap) { nu[k] = a; gns[k] = b; e_i[k] = c; aif[k] = d; gam[k] = e; nexp[k] = f; }
        ++k;
    }
    if (r->hitran_file) std::fclose(r->hitran_file);
    r->open_file = false;
    return k;
}

int main(int argc, char** argv)
{
    if (argc == 7 && std::string(argv[1]) == "hitran") {
        const double P = std::atof(argv[3]), mix = std::atof(argv[4]), qr = std::atof(argv[5]);
        const int64_t n = ref_hitran_read(argv[2], P, mix, qr, 0, 0, 0, 0, 0, 0, 0);
        std::vector<double> a(n > 0 ? n : 1), b(a.size()), c(a.size()), d(a.size()), e(a.size()), f(a.size());
        ref_hitran_read(argv[2], P, mix, qr, a.data(), b.data(), c.data(), d.data(), e.data(), f.data(), n);
        FILE* out = std::fopen(argv[6], "wb");
        if (!out) return 3;
        std::fwrite(&n, sizeof(n), 1, out);
        for (std::vector<double>* v : {&a, &b, &c, &d, &e, &f}) std::fwrite(v->data(), sizeof(double), n, out);
        std::fclose(out);
        return 0;
    }
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s STATES TRANS BROAD|- DEFAULT_GAMMA DEFAULT_N OUT\n", argv[0]);
        return 2;
    }
    const char* broad = std::string(argv[3]) == "-" ? "" : argv[3];
    const double dg = std::atof(argv[4]), dn = std::atof(argv[5]);
    const int64_t n = ref_exomol_read(argv[1], argv[2], broad, dg, dn, 0, 0, 0, 0, 0, 0, 0);
    std::vector<double> a(n > 0 ? n : 1), b(a.size()), c(a.size()), d(a.size()), e(a.size()), f(a.size());
    ref_exomol_read(argv[1], argv[2], broad, dg, dn, a.data(), b.data(), c.data(), d.data(),
                    e.data(), f.data(), n);
    FILE* out = std::fopen(argv[6], "wb");
    if (!out) return 3;
    std::fwrite(&n, sizeof(n), 1, out);
    for (std::vector<double>* v : {&a, &b, &c, &d, &e, &f}) std::fwrite(v->data(), sizeof(double), n, out);
    std::fclose(out);
    return 0;
}
