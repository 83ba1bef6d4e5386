/*
 * gexs_tips.cpp — TIPS-2011 total internal partition sums Q(T) of the
 * HITRAN molecules, the source of every HITRAN Q(T) in the reference
 * (Readers/HITRAN/HITRANStateReader.cpp:62 at the run's temperature, :95 at
 * 296 K for the A coefficients rebuilt from S, :128 per (T, P) pair).
 *
 * Restated from BD_TIPS_2011 (Readers/HITRAN/BD_TIPS_2011_v1p0.for:5-345):
 * molecule -> table of its isotopologue; temperatures outside 70-3000 K
 * give Q = -1 (e.g. QT_H2O, :547-551); molecules 34 and 39 give gi = 0,
 * Q = 0.  Interpolation as AtoB (:5830-5920): I = the first index (1-based,
 * from 2) whose grid temperature is >= T; Lagrange through 3 points ending
 * at max(I, 3) when I < 3 or I is the last point, else through the 4
 * points I-2 .. I+1, each weight a product of differences divided by the
 * product of node differences, evaluated in that order in FP64.  The
 * tables (tips2011_data.h) are generated from the DATA statements by
 * gen_tips2011.py.  Host code: one scalar per temperature, no device work.
 */
#include <string>
#include "../../include/gexs_b200.h"
#include "../csrc/gexs_internal.h"
#include "tips2011_data.h"

namespace {

using namespace gexs_tips;

/* Tdat(i), 1-based: 60, 85, ..., 3010 K (exact in binary) */
double tdat(int i) { return 60.0 + 25.0 * (double)(i - 1); }

/* AtoB over Tdat and one table row (B(i) = row[i - 1]) */
double atob(double aa, const float* row)
{
    const int npt = kNT;
    auto A = [](int i) { return tdat(i); };
    auto B = [&](int i) { return (double)row[i - 1]; };
    int I = 2;
    while (I < npt && A(I) < aa) ++I;
    /* the node differences never vanish on this grid (AtoB guards zeros) */
    if (I < 3 || I == npt) {
        const int J = I < 3 ? 3 : npt;
        const double a0 = ((aa - A(J - 1)) * (aa - A(J))) / ((A(J - 2) - A(J - 1)) * (A(J - 2) - A(J)));
        const double a1 = ((aa - A(J - 2)) * (aa - A(J))) / ((A(J - 1) - A(J - 2)) * (A(J - 1) - A(J)));
        const double a2 = ((aa - A(J - 2)) * (aa - A(J - 1))) / ((A(J) - A(J - 2)) * (A(J) - A(J - 1)));
        return (a0 * B(J - 2) + a1 * B(J - 1)) + a2 * B(J);
    }
    const int J = I;
    const double d0 = ((A(J - 2) - A(J - 1)) * (A(J - 2) - A(J))) * (A(J - 2) - A(J + 1));
    const double d1 = ((A(J - 1) - A(J - 2)) * (A(J - 1) - A(J))) * (A(J - 1) - A(J + 1));
    const double d2 = ((A(J) - A(J - 2)) * (A(J) - A(J - 1))) * (A(J) - A(J + 1));
    const double d3 = ((A(J + 1) - A(J - 2)) * (A(J + 1) - A(J - 1))) * (A(J + 1) - A(J));
    const double a0 = (((aa - A(J - 1)) * (aa - A(J))) * (aa - A(J + 1))) / d0;
    const double a1 = (((aa - A(J - 2)) * (aa - A(J))) * (aa - A(J + 1))) / d1;
    const double a2 = (((aa - A(J - 2)) * (aa - A(J - 1))) * (aa - A(J + 1))) / d2;
    const double a3 = (((aa - A(J - 2)) * (aa - A(J - 1))) * (aa - A(J))) / d3;
    return ((a0 * B(J - 2) + a1 * B(J - 1)) + a2 * B(J)) + a3 * B(J + 1);
}

}  // namespace

extern "C" int gexs_tips_2011(int molecule, int isotopologue, double temperature, double* gi,
                              double* q)
{
    if (!gi || !q) return gexs::set_error(GEXS_ERR_INVALID, "gexs_tips_2011: NULL output");
    *gi = 0.0;
    *q = 0.0;
    if (molecule < 1 || molecule > kMolecules)
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_tips_2011: molecule " +
                                                     std::to_string(molecule) + " not in TIPS-2011");
    const int n = kCount[molecule - 1];
    if (n == 0) return GEXS_OK;                   /* molecules 34, 39: gi = 0, Q = 0 */
    if (isotopologue < 1 || isotopologue > n)
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_tips_2011: isotopologue " +
                                                     std::to_string(isotopologue) + " of molecule " +
                                                     std::to_string(molecule) + " not in TIPS-2011");
    const int row = kFirst[molecule - 1] + isotopologue - 1;
    *gi = (double)kGi[row];
    if (temperature < 70.0 || temperature > 3000.0) {
        *q = -1.0;
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_tips_2011: temperature outside 70-3000 K");
    }
    *q = atob(temperature, kQ[row]);
    return GEXS_OK;
}
