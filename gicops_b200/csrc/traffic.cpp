// Algorithmic traffic of the query path, for the roofline figure.
//
// Per spectrum and per length with a non-empty precursor window:
//   8 B per distinct probed fragment bin (its bA pair) and 4 B per ion id of such a
//   bin whose entry lies inside the window (each distinct bin counted once, even
//   when several peaks probe it).
// Plus 8 B per peak (m/z + intensity), 8 B per length (window bounds) and the
// result record, added by the caller.  Window and bin rules are those of the
// search (source/core/dslim_query.cpp:844-877).

#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/gicops_b200.h"
#include "gx_internal.h"

namespace {

void window(const gx_length_desc &d, float prec, double dM, int64_t &lo, int64_t &hi)
{
    lo = 1;
    hi = 0;
    const int64_t N = d.npep;
    if (dM < 0.0 || N == 0) return;
    const float p1 = (float)((double)prec - dM), p2 = (float)((double)prec + dM);
    if (p1 != p1 || p2 != p2 || p1 > d.mass[N - 1] || p2 < d.mass[0]) return;
    lo = std::lower_bound(d.mass, d.mass + N, p1) - d.mass;
    hi = (std::upper_bound(d.mass, d.mass + N, p2) - d.mass) - 1;
}

}  // namespace

extern "C" gx_status gx_traffic_host(const gx_length_desc *lens, int32_t nlen, const gx_queries *q, const gx_params *p,
                                     int64_t *ids_out, int64_t *bins_out, int32_t threads)
{
    if (!lens || !q || !p || !ids_out || !bins_out) return gx::fail(GX_ERR_INVLD_PTR, "gx_traffic_host: null argument");
    const double upper = (p->max_mass * (double)p->scale) - 1.0 - (double)p->dF;
    const int T = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for num_threads(T) schedule(dynamic, 8)
    for (int64_t s = 0; s < (int64_t)q->nspec; s++) {
        std::vector<uint32_t> bins;
        for (uint32_t k = q->idx[s]; k < q->idx[s + 1]; k++) {
            const int32_t m = q->moz[k];
            if (m > (int32_t)p->dF && (double)m < upper)
                for (int32_t b = m - (int32_t)p->dF; b <= m + (int32_t)p->dF; b++) bins.push_back((uint32_t)b);
        }
        std::sort(bins.begin(), bins.end());
        bins.erase(std::unique(bins.begin(), bins.end()), bins.end());
        int64_t ni = 0, nb = 0;
        const double dM = q->dM ? q->dM[s] : p->dM;
        for (int32_t l = 0; l < nlen; l++) {
            const gx_length_desc &d = lens[l];
            int64_t lo, hi;
            window(d, q->prec[s], dM, lo, hi);
            if (hi < lo) continue;
            const uint32_t a_id = (uint32_t)lo * d.speclen, b_id = (uint32_t)(hi + 1) * d.speclen;
            nb += (int64_t)bins.size();
            for (uint32_t b : bins) {
                const uint32_t *s0 = d.iA + d.bA[b], *s1 = d.iA + d.bA[b + 1];
                ni += std::lower_bound(s0, s1, b_id) - std::lower_bound(s0, s1, a_id);
            }
        }
        ids_out[s] = ni;
        bins_out[s] = nb;
    }
    return GX_SUCCESS;
}
