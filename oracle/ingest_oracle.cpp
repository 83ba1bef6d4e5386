/*
 * ingest_oracle.cpp — CPU restatement of the reference's ExoMol reader
 * (TEST INFRASTRUCTURE ONLY: the checker of gexs_b200's GPU ingest; the
 * product path never links or calls it).
 *
 *   orc_exomol_states  Readers/Exomol/exomol_functions.cpp:8-48: fgets into
 *                      a 1024-byte buffer (a longer line is split), then
 *                      id = strtol(.., 0) - 1, energy = strtod, gns and J by
 *                      strtol(.., 0); states indexed by line number.
 *   orc_exomol_trans   Readers/Exomol/ExomolStateReader.cpp:132-172: the file
 *                      as one token stream `>> id_f >> id_i >> aif` (stops at
 *                      the first failed extraction); nu = E[id_f-1] -
 *                      E[id_i-1], e_i = E[id_i-1], gns = g[id_f-1].
 *                      Broadening (:7-37, :39-75): mode 0 gives the
 *                      defaults, which is what the reference's lookup yields
 *                      (the key keeps the failed "a1" text after
 *                      key.clear(), :21); mode 1 the intended rule: "a1"
 *                      (J'', J'), then "a0" (J''), then the defaults.
 *   orc_hitran         Readers/HITRAN/HITRANStateReader.cpp:137-250 (see
 *                      the function).
 * Pinned by tests/test_ingest_pin.py against the reference readers compiled
 * from its own sources (oracle/_ref/gexsref_reader).  Written with libc
 * only (no iostreams): `>> int` is restated as whitespace, sign, decimal
 * digits (failing on none or on int overflow) and `>> double` as the
 * longest [sign]digits[.digits][e[sign]digits] text given to strtod, which
 * is what libstdc++'s num_get extracts for such input.
 */
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace {

/* fgets(buf, 1024, f) over a memory buffer: next chunk of at most 1023
 * bytes, ending after a newline if one comes first */
bool next_fgets(const char* text, int64_t n, int64_t& pos, std::string& out)
{
    if (pos >= n) return false;
    int64_t e = pos;
    while (e < n && e - pos < 1023) {
        if (text[e++] == '\n') break;
    }
    out.assign(text + pos, text + e);
    pos = e;
    return true;
}

struct BroadTables {
    std::map<int, std::pair<double, double>> a0;
    std::map<std::pair<int, int>, std::pair<double, double>> a1;
};

bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

/* "code gamma n J'' [J']" per line; a later entry of a key replaces an
 * earlier one (a std::map assignment in the reference) */
void parse_broad(const char* text, int64_t n, BroadTables& bt)
{
    int64_t i = 0;
    while (i < n) {
        int64_t j = i;
        while (j < n && text[j] != '\n') ++j;
        std::vector<std::string> tok;
        int64_t k = i;
        while (k < j) {
            while (k < j && is_ws(text[k])) ++k;
            int64_t e = k;
            while (e < j && !is_ws(text[e])) ++e;
            if (e > k) tok.emplace_back(text + k, text + e);
            k = e;
        }
        i = j + 1;
        if (tok.size() < 4) continue;
        const double g = std::atof(tok[1].c_str()), x = std::atof(tok[2].c_str());
        const int J1 = std::atoi(tok[3].c_str());
        if (tok[0] == "a0") bt.a0[J1] = {g, x};
        else if (tok[0] == "a1" && tok.size() >= 5) bt.a1[{J1, std::atoi(tok[4].c_str())}] = {g, x};
    }
}

/* `>> int` over [p, end) */
bool get_int(const char*& p, const char* end, int* out)
{
    while (p < end && is_ws(*p)) ++p;
    const char* s = p;
    bool neg = false;
    if (s < end && (*s == '+' || *s == '-')) { neg = *s == '-'; ++s; }
    const char* d = s;
    long long v = 0;
    while (s < end && *s >= '0' && *s <= '9') {
        v = v * 10 + (*s - '0');
        if (v > 2147483648ll) return false;
        ++s;
    }
    if (s == d) return false;
    if (neg) v = -v;
    if (v > 2147483647ll || v < -2147483648ll) return false;
    *out = (int)v;
    p = s;
    return true;
}

/* `>> double` over [p, end) */
bool get_double(const char*& p, const char* end, double* out)
{
    while (p < end && is_ws(*p)) ++p;
    const char* s = p;
    if (s < end && (*s == '+' || *s == '-')) ++s;
    bool any = false;
    while (s < end && *s >= '0' && *s <= '9') { ++s; any = true; }
    if (s < end && *s == '.') { ++s; while (s < end && *s >= '0' && *s <= '9') { ++s; any = true; } }
    if (!any) return false;
    if (s < end && (*s == 'e' || *s == 'E')) {
        const char* q = s + 1;
        if (q < end && (*q == '+' || *q == '-')) ++q;
        if (q < end && *q >= '0' && *q <= '9') { while (q < end && *q >= '0' && *q <= '9') ++q; s = q; }
    }
    const std::string tok(p, s);
    *out = std::strtod(tok.c_str(), nullptr);
    p = s;
    return true;
}

}  // namespace

extern "C" {

/* returns the number of states; writes at most cap of them */
int64_t orc_exomol_states(const char* text, int64_t n, double* energy, int32_t* g, int32_t* J,
                          int64_t cap)
{
    int64_t pos = 0, k = 0;
    std::string buf;
    while (next_fgets(text, n, pos, buf)) {
        char* p = nullptr;
        const char* s = buf.c_str();
        (void)std::strtol(s, &p, 0);
        const double e = std::strtod(p, &p);
        const long gv = std::strtol(p, &p, 0);
        const long jv = std::strtol(p, &p, 0);
        if (k < cap) { energy[k] = e; g[k] = (int32_t)gv; J[k] = (int32_t)jv; }
        ++k;
    }
    return k;
}

/* returns the number of transitions (-1 if a state id is out of range);
 * writes at most cap of them, in file order */
int64_t orc_exomol_trans(const char* text, int64_t n, const double* sE, const int32_t* sg,
                         const int32_t* sJ, int64_t nstates, const char* broad, int64_t nbroad,
                         int mode, double dgam, double dn, double* nu, double* elow, double* aif,
                         int32_t* gns, double* gam, double* nexp, int64_t cap)
{
    BroadTables bt;
    if (mode == 1 && broad && nbroad > 0) parse_broad(broad, nbroad, bt);
    const char* p = text;
    const char* end = text + n;
    int idf, idi;
    double A;
    int64_t k = 0;
    while (get_int(p, end, &idf) && get_int(p, end, &idi) && get_double(p, end, &A)) {
        if (idf < 1 || idi < 1 || idf > nstates || idi > nstates) return -1;
        const int64_t f = idf - 1, l = idi - 1;
        double gv = dgam, xv = dn;
        if (mode == 1) {
            auto i1 = bt.a1.find({sJ[l], sJ[f]});
            if (i1 != bt.a1.end()) { gv = i1->second.first; xv = i1->second.second; }
            else {
                auto i0 = bt.a0.find(sJ[l]);
                if (i0 != bt.a0.end()) { gv = i0->second.first; xv = i0->second.second; }
            }
        }
        if (k < cap) {
            nu[k] = sE[f] - sE[l];
            elow[k] = sE[l];
            aif[k] = A;
            gns[k] = sg[f];
            gam[k] = gv;
            nexp[k] = xv;
        }
        ++k;
    }
    return k;
}

/* Readers/HITRAN/HITRANStateReader.cpp:137-250 restated: one record per
 * non-empty line; fields by atof of their columns (:21-29, widths
 * {2,1,12,10,10,5,5,10,4,8,15,15,15,15,6,12,1,7,7}); gamma = (gamma_air*mix
 * + gamma_self*(1-mix))*P; where A == 0 it is rebuilt from S with Q(296)
 * = ref_q and g' = 1.  Columns past the end of a short line are treated as
 * absent (the reference reads stale buffer bytes there). */
static double col_atof(const char* line, int64_t len, int off, int w)
{
    char f[13] = {0};
    const int64_t n = std::min<int64_t>(w, std::max<int64_t>(0, len - off));
    if (n > 0) std::memcpy(f, line + off, (size_t)n);
    return std::atof(f);
}

int64_t orc_hitran(const char* text, int64_t n, double pressure, double mixture, double ref_q,
                   double* nu, double* elow, double* aif, int32_t* gns, double* gam,
                   double* nexp, int64_t cap)
{
    int64_t i = 0, k = 0;
    while (i < n) {
        int64_t j = i;
        while (j < n && text[j] != '\n') ++j;
        const char* line = text + i;
        const int64_t len = j - i;
        i = j + 1;
        bool blank = true;
        for (int64_t t = 0; t < len; ++t) if (!is_ws(line[t])) { blank = false; break; }
        if (blank) continue;
        const double v_nu = col_atof(line, len, 3, 12), v_S = col_atof(line, len, 15, 10);
        double v_A = col_atof(line, len, 25, 10);
        const double g_air = col_atof(line, len, 35, 5), g_self = col_atof(line, len, 40, 5);
        const double v_E = col_atof(line, len, 45, 10), v_n = col_atof(line, len, 55, 4);
        double v_g = col_atof(line, len, 146, 7);
        const double gv = (g_air * mixture + g_self * (1.0 - mixture)) * pressure;
        if (v_A == 0.0) {
            const double planck = 6.6260693e-27, vellgt = 2.99792458e10, boltz = 1.380658e-16;
            const double pi = std::acos(-1.0);
            const double beta = planck * vellgt / (boltz * 296.0);
            v_A = v_S * 8.0 * pi * vellgt * ref_q * v_nu * v_nu /
                  (std::exp(-beta * v_E) * (1.0 - std::exp(-beta * v_nu)));
            v_g = 1.0;
        }
        if (k < cap) {
            nu[k] = v_nu; elow[k] = v_E; aif[k] = v_A; gns[k] = (int32_t)v_g;
            gam[k] = gv; nexp[k] = v_n;
        }
        ++k;
    }
    return k;
}

/* stable order of the indices by nu */
void orc_sort_by_nu(const double* nu, int64_t n, int64_t* perm)
{
    for (int64_t i = 0; i < n; ++i) perm[i] = i;
    std::stable_sort(perm, perm + n, [&](int64_t a, int64_t b) { return nu[a] < nu[b]; });
}

/* glibc strtod, for the parser tests */
double orc_strtod(const char* s)
{
    return std::strtod(s, nullptr);
}

}  // extern "C"
