// sg_step.cu -- the learned REBO term inside a device-resident AIREBO step,
// with the plain REBO kernel as judge and fallback.
//
// Every step runs the learned pass (rows, descriptors, tensor-core network,
// force assembly) and a gated plain REBO launch; a device flag S->sg_off
// decides which of the two does any work, so the step stays one fixed CUDA
// graph whether or not the plain kernel has taken over.  On a judge step the
// plain kernel also evaluates the same positions into a side buffer and one
// block computes the force RMSE between the two; above the threshold it
// copies the plain forces and partials over the learned ones and sets the
// flag, so from that step on the trajectory follows the plain kernel.
#include <cmath>

#include "sg_host.h"
#include "step.h"

namespace fmd {
namespace {

constexpr int kJudgeThreads = 1024;

// Force RMSE sqrt(mean over the 3n components of (F_learned - F_plain)^2),
// the definition fmd_sg_eval uses.  One block; fixed summation order.
__global__ void __launch_bounds__(kJudgeThreads)
k_sg_judge(SysScal* __restrict__ S, double* __restrict__ Facc, const double* __restrict__ Fj,
           const double* __restrict__ part_j, double* __restrict__ part, int n3, int nrec, double rmse_max) {
    __shared__ double sm[kJudgeThreads / 32];
    __shared__ int take;
    if (S->sg_off) return;                       // uniform: the plain kernel already runs
    double s = 0.0;
    for (int k = threadIdx.x; k < n3; k += kJudgeThreads) {
        const double d = Facc[k] - Fj[k];
        s += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kJudgeThreads / 32; w++) t += sm[w];
        const double rmse = sqrt(t / (n3 > 0 ? n3 : 1));
        S->sg_judged += 1;
        S->sg_rmse_last = rmse;
        if (rmse > S->sg_rmse_max) S->sg_rmse_max = rmse;
        take = !(rmse <= rmse_max);              // NaN also hands over
        if (take) {
            S->sg_off = 1;
            S->sg_takeover = S->gstep;
        }
    }
    __syncthreads();
    if (!take) return;
    for (int k = threadIdx.x; k < n3; k += kJudgeThreads) Facc[k] = Fj[k];
    for (int k = threadIdx.x; k < nrec * kNV; k += kJudgeThreads) part[k] = part_j[k];
}

}  // namespace

cudaError_t sg_enqueue_rebo(SgStep& g, const StepArrays& a, bool judge, cudaStream_t st) {
    const double* hh = a.S->h;
    const int* off = &a.S->sg_off;
    cudaError_t e = sg::rebo_forces(g.work, g.img, g.vec, a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.Facc,
                                    a.part_f1, st, off);
    if (e != cudaSuccess) return e;
    e = rebo_slots_launch(a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.rebo_slots, a.Facc, a.part_f1,
                          sg::kRowBlocks, off, 1, st, a.rebo_ids);
    if (e != cudaSuccess || !judge) return e;
    if ((e = cudaMemsetAsync(g.Fj, 0, sizeof(double) * 3 * (size_t)a.n, st)) != cudaSuccess) return e;
    e = rebo_slots_launch(a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.rebo_slots, g.Fj, g.part_j, sg::kRowBlocks,
                          off, 0, st, a.rebo_ids);
    if (e != cudaSuccess) return e;
    k_sg_judge<<<1, kJudgeThreads, 0, st>>>(a.S, a.Facc, g.Fj, g.part_j, a.part_f1, 3 * a.n, sg::kRowBlocks,
                                            g.rmse_max);
    return cudaGetLastError();
}

}  // namespace fmd
