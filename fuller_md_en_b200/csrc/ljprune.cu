// ljprune.cu -- dynamic pruning of the LJ gather's full rows.
//
// The reference takes a listed pair when r <= LJ_RCUT at the current step
// (AI:441, MM:745); its list holds pairs within LJ_RCUT + 2 at the last build,
// rows cut after MAX_LJ_NEIGH entries (AI:263-272, MM:337-346).  The gather's
// full rows (airebo.cu) hold exactly those pairs.  A pruning gather walks them,
// and besides the forces writes each row's entries with r <= LJ_RCUT + delta
// now, in row order, so the pruned rows are a sub-sequence of the full rows
// and keep their truncation.  Later steps gather the pruned rows.
//
// Exactness.  With a diagonal cell at the prune and now, the reference's
// minimum image is the nearest image per axis.  For fractional positions s,
// prune cell h_p, current cell h, u = max_i |h (s_i - s_i,p)| (nearest image)
// and k = max_a |h_aa - h_p,aa| / h_p,aa, an entry at distance > rc + delta at
// the prune is now farther than (1 - k)(rc + delta) - 2u.  While
// k (rc + delta) + 2u < delta (less a rounding margin) every entry dropped by
// the prune is still beyond the cutoff, so the pruned rows yield exactly the
// pairs of the full rows and the same pair terms; only the lanes that add
// them, and so the rounding of the sums, change.  The drift raises u
// (kick_body); each block of the gather evaluates the condition
// (lj_prune_needed) and walks either the full rows, writing pruned ones, or
// the pruned rows; the step's reduction kernel then restarts the bound when
// the evaluation pruned.  A list build marks the next evaluation as a prune.
#include <cmath>

#include "ljprune.h"

namespace fmd {
namespace {

__global__ void k_prune_mark(unsigned long long* words) { *words = kPruneMark; }

}  // namespace

cudaError_t lj_prune_clear(const LJPrune& p, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(p.cnt, 0, sizeof(int) * p.n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p.sb, 0, sizeof(double) * 3 * p.n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p.hb, 0, sizeof(double) * 9, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p.stats, 0, sizeof(unsigned long long) * 2, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p.words, 0x7F, sizeof(unsigned long long), st);
    return e;
}

cudaError_t lj_prune_mark(const LJPrune& p, cudaStream_t st) {
    k_prune_mark<<<1, 1, 0, st>>>(p.words);
    return cudaGetLastError();
}

LJPruneOut lj_prune_out(const LJPrune& p) {
    LJPruneOut o;
    o.cnt = p.cnt;
    o.list = p.list;
    o.sb = p.sb;
    const double r = p.rc + p.delta;
    o.r2 = r * r;
    o.words = p.words;
    o.hb = p.hb;
    o.delta = p.delta;
    o.rc = p.rc;
    return o;
}

}  // namespace fmd
