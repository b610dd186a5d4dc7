// ljprune.cuh -- the device-side decision of the pruned LJ rows (ljprune.cu).
#pragma once
#include <cmath>

namespace fmd {

// 1 when the pruned rows may miss a pair now within the cutoff: the cell is
// not diagonal (now or at the prune), or k (rc + delta) + 2u >= delta less a
// rounding margin, u the largest displacement since the last prune (bits in
// *words, raised by the drift; a list build stores a huge value) and k the
// largest relative change of a cell edge since then.  Every block of the
// gather and the step's reduction evaluate it on the same, unchanged inputs.
__device__ __forceinline__ bool lj_prune_needed(const unsigned long long* words, const double* hh, const double* hb,
                                                double delta, double rc) {
    const double u = __longlong_as_double((long long)*words);
    double k = 0.0;
    for (int a = 0; a < 3; a++) k = fmax(k, fabs(hh[4 * a] - hb[4 * a]) / fabs(hb[4 * a]));
    const bool diag = hh[1] == 0.0 && hh[2] == 0.0 && hh[3] == 0.0 && hh[5] == 0.0 && hh[6] == 0.0 &&
                      hh[7] == 0.0 && hb[1] == 0.0 && hb[2] == 0.0 && hb[3] == 0.0 && hb[5] == 0.0 &&
                      hb[6] == 0.0 && hb[7] == 0.0;
    return !(diag && k * (rc + delta) + 2.0 * u < delta - 1e-6);
}

}  // namespace fmd
