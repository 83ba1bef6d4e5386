/*
 * gexs_shard.cpp — split one cross-section's bins over several devices.
 *
 * A bin's value depends only on the lines within the cutoff of it, so
 * disjoint bin ranges are computed independently, each from the sub-list of
 * lines that can reach it, and the full grid is their concatenation: no
 * data-path exchange between devices.  (The reference's multi-GPU manager
 * instead gives whole line chunks to GPUs and sums full-size grids on the
 * host, Managers/Accel/GPU/MultiGPUManager.cpp:59-63,104-126.)
 *
 * The cuts equalise the (line, bin) evaluations: the work of bin j is the
 * number of lines within `reach` of it, sampled every 256th bin from the
 * sorted centres; interior cuts fall on multiples of `align` bins from
 * start_idx, so the tiles of every shard are tiles of the unsplit launch
 * (tile widths divide 4096) and a shard computes exactly the sums that the
 * single launch computes for its bins.
 */
#include <algorithm>
#include <cmath>
#include <vector>
#include "../../include/gexs_b200.h"
#include "../csrc/gexs_internal.h"

extern "C" int gexs_shard_plan(const double* h_nu, int64_t nlines, double nu_start, double dnu,
                               int64_t start_idx, int64_t n_points, double reach, int align,
                               int nshards, int64_t* bounds, int64_t* line_lo, int64_t* line_hi)
{
    if (nlines < 0 || (nlines > 0 && !h_nu) || !(dnu > 0.0) || start_idx < 0 || n_points < 0 ||
        !(reach >= 0.0) || align < 1 || nshards < 1 || !bounds || !line_lo || !line_hi)
        return gexs::set_error(GEXS_ERR_INVALID, "gexs_shard_plan: arguments");
    const double* nb = h_nu;
    const double* ne = h_nu + nlines;
    auto f = [&](int64_t j) { return nu_start + (double)j * dnu; };
    /* work per sampled bin: lines within reach (sorted centres) */
    const int64_t sample = 256;
    std::vector<double> cum(1, 0.0);
    std::vector<int64_t> at(1, start_idx);
    for (int64_t j = start_idx; j < start_idx + n_points; j += sample) {
        const double w = (double)(std::upper_bound(nb, ne, f(j) + reach) -
                                  std::lower_bound(nb, ne, f(j) - reach)) + 1e-9;
        cum.push_back(cum.back() + w * (double)std::min(sample, start_idx + n_points - j));
        at.push_back(std::min(j + sample, start_idx + n_points));
    }
    const double tot = cum.back();
    bounds[0] = start_idx;
    for (int r = 1; r < nshards; ++r) {
        const double want = tot * (double)r / (double)nshards;
        const size_t k = (size_t)(std::lower_bound(cum.begin(), cum.end(), want) - cum.begin());
        int64_t b = at[std::min(k, at.size() - 1)];
        /* round to the alignment from start_idx, keep the cuts ordered */
        b = start_idx + (int64_t)std::llround((double)(b - start_idx) / (double)align) * align;
        b = std::min(std::max(b, bounds[r - 1]), start_idx + n_points);
        bounds[r] = b;
    }
    bounds[nshards] = start_idx + n_points;
    for (int r = 0; r < nshards; ++r) {
        if (bounds[r + 1] <= bounds[r] || nlines == 0) {
            line_lo[r] = line_hi[r] = 0;
            continue;
        }
        const double fa = f(bounds[r]), fb = f(bounds[r + 1] - 1);
        line_lo[r] = (int64_t)(std::lower_bound(nb, ne, fa - reach) - nb);
        line_hi[r] = (int64_t)(std::upper_bound(nb, ne, fb + reach) - nb);
    }
    return GEXS_OK;
}
