// step.h -- the velocity-Verlet NPT step as a sequence of device kernels.
#pragma once
#include "kernels.h"

namespace fmd {

// Device-resident scalars of one system.  h[9] and hi[9] are adjacent so
// &h[0] is the {h, hi} block every force and list kernel reads.
struct SysScal {
    double h[9], hi[9];
    double hi_old[9];        // inverse cell used by the drift (before the cell update)
    fmd_npt npt;
    double sc_v, sc_nh, sc_v2;
    double KE, kt, kr;       // current kinetic energies (kt, kr: rigid only)
    double W9[9];            // virial of the last force call
    double E[8];             // energies of the last force call (program grouping)
    double Tn, Pn, an;
    double scale;
    int do_rescale;
    int gstep;
    fmd_obs obs;
    fmd_avg avg;
    // Learned REBO term (AIREBO systems with a model attached): the plain
    // kernel judges it every few steps and takes over above a force RMSE.
    int sg_off;              // 1: the plain REBO kernel has taken over
    int sg_judged;           // judge evaluations so far
    int sg_takeover;         // global step of the takeover (0: none)
    double sg_rmse_last, sg_rmse_max;
    unsigned int kick2_done; // blocks of the fused second kick done this step (the last one reduces)
    unsigned int kick_done;  // blocks of the fused first kick done this step (the last one writes back)
};

struct SgStep;   // learned REBO term of a system (sg_host.h)
struct LJPrune;  // pruned LJ rows of a system (ljprune.h)

// Device pointers and sizes of one step.
struct StepArrays {
    int kind = FMD_SYS_AIREBO;
    int n = 0;               // particles: molecules (rigid) or atoms
    int natom = 0;           // sites per rigid molecule
    double* pos = nullptr; double* vel = nullptr; double* F = nullptr; double* Facc = nullptr;
    double* omg = nullptr; double* qv = nullptr; double* T = nullptr;
    const double* mass = nullptr;     // AIREBO per-atom masses; nullptr: constant carbon mass
    const double* body = nullptr;
    const int* mol_id = nullptr;
    const double* charge = nullptr;
    int has_charge = 0;
    SysScal* S = nullptr;
    const int* cnt_a = nullptr; const int* list_a = nullptr; int cap_a = 0;     // LJ half / rigid
    const int* in_cnt = nullptr; const int* in_list = nullptr; int in_cap = 0;  // LJ full rows (incoming + own)
    const int* cnt_b = nullptr; const int* list_b = nullptr; int cap_b = 0;     // REBO
    double* rebo_slots = nullptr;   // [n * cap_b * kReboSlotDoubles] REBO slot records (fast path)
    const int* rebo_ids = nullptr;  // occupied REBO slots (warp-aligned) and partner slots of the last build
    double* part_f1 = nullptr;  // REBO / rigid / bonded partials
    double* part_f2 = nullptr;  // LJ partials
    double* part_f3 = nullptr;  // Coulomb partials
    double* part_ke = nullptr;  // kinetic partials
    MMTopoDev topo{};
    double rmcut2 = 0, Mmol = 0, I0 = 0;
    double* rigid_lab = nullptr;   // [n * natom * kRigidLabDoubles] lab-frame sites (rigid)
    int rigid_shape = 0;           // launch shape of the rigid pair kernel (rigid_launch)
    int precision = FMD_PREC_FP64;
    int quat_left = 0;              // FMD_PHYS_QUAT: the rotation increment multiplies q on the left
    int rebo_phys = 0;              // FMD_PHYS_REBO: bond-order gradient instead of the reference's three-body forces
    LJShape lj_shape{};            // launch shape of the atomistic LJ gather over the full rows
    LJShape lj_shape_p{};          // ... and over the pruned rows
    DevErr* err = nullptr;         // device error word (bounded waits of staged kernels)
    int lj_blocks = 0;             // partial records in part_f2: the larger grid of the two gathers
    SgStep* sg = nullptr;          // AIREBO: learned REBO term instead of the plain kernel
    int rebo_blocks = kForceBlocks;  // partial records the REBO term writes into part_f1
    // REBO-II extension (fmd_system_set_rebo2): FMD_REBO2_* flags, the device
    // tables, and the switched-LJ correction's partials (kForceBlocks records)
    int rebo2_flags = 0;
    Rebo2Dev rebo2{};
    double* part_sw = nullptr;
    // Pruned LJ rows (AIREBO, MM): host descriptor (nullptr: full rows every
    // step), and the fractional positions of the last prune and the
    // displacement word the drift raises.
    const LJPrune* prune = nullptr;
    const double* prune_sb = nullptr;
    unsigned long long* prune_umax = nullptr;
    double* prune_hb = nullptr;                 // cell of the last prune
    unsigned long long* prune_stats = nullptr;  // {evaluations, prunes}
    double prune_delta = 0.0, prune_rc = 0.0;   // buffer (0: off) and LJ cutoff
};

struct StepParams {
    double dt = 1.0, T = 300.0, T_cold = 4.0;
    int coldstart = 0, warmup = 0, gavg_from = 1, gavg_to = 0, nc = 1, nmol = 1;
    int schedule = 0;        // 1: driver schedule, observables and averages (system runs)
};

// Force evaluation of the step's kind; fills partials and F (and T).
// judge: AIREBO with a learned REBO term also runs the plain REBO kernel and
// compares the two (sg_step.cu).
cudaError_t enqueue_forces(const StepArrays& a, cudaStream_t st, bool judge = false);
// The LJ term alone (ff: FMD_FF_AIREBO / FMD_FF_MM): F = Facc + LJ, Facc zeroed.
cudaError_t enqueue_lj(const StepArrays& a, int ff, cudaStream_t st);
// Reduces the force partials into S->W9 / S->E (one small kernel).
cudaError_t enqueue_force_reduce(const StepArrays& a, cudaStream_t st);
// Recomputes S->KE (and kt, kr) from the velocities.
cudaError_t enqueue_ke(const StepArrays& a, cudaStream_t st);
// One step_npt (+ driver schedule if p.schedule); rescale_phase selects the
// cold/warm velocity rescale kernels.
cudaError_t enqueue_step(const StepArrays& a, const StepParams& p, bool rescale_phase, cudaStream_t st,
                         bool judge = false);
// Observables / averages for the pre-loop state (not a step).
int force_partial_blocks(const StepArrays& a);

// ------------------------------------------------------- replica batches --
// A batched launch covers R replicas: block b belongs to replica r with
// off[r] <= b < off[r + 1] and acts as block b - off[r] of a grid of
// off[r + 1] - off[r] blocks for that replica alone, so each replica keeps
// its own grid size (and partial-record count) inside one launch.
__device__ __forceinline__ int batch_rep(const int* __restrict__ off, int R, int b) {
    int lo = 0, hi = R - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Device tables of a batch: per-replica arrays and parameters, and the block
// offsets of each launch class (R + 1 entries each).
struct BatchDev {
    int R = 0;
    const StepArrays* A = nullptr;
    const StepParams* P = nullptr;
    const int* off_atom = nullptr;   // per-particle kernels (kicks, rescale)
    const int* off_lj = nullptr;     // LJ gather (part_f2 records)
    const int* off_f1 = nullptr;     // bonded terms (part_f1 records)
    int nblk_atom = 0, nblk_lj = 0, nblk_f1 = 0;   // totals (off[R])
    int lj_threads = 256, lj_unroll = 4, f1_threads = 128;
    int lj_staged_in_cap = 0;        // > 0: LJ rows staged in shared memory
    int kind = FMD_SYS_MM, ff = FMD_FF_MM, precision = FMD_PREC_FP64;
};
// LJ gather / MM bonded terms over all replicas in one launch each.
// staged_in_cap > 0: rows staged in shared memory (all replicas' row stride).
cudaError_t batch_lj_launch(const StepArrays* As, const int* off, int R, int nblocks, int ff, int precision,
                            int threads, int unroll, cudaStream_t st, int staged_in_cap = 0);
cudaError_t batch_mm_bonded_launch(const StepArrays* As, const int* off, int R, int nblocks, int threads,
                                   cudaStream_t st);
// One step of every replica (the single-system step's launches, each once
// for the whole batch); rescale_phase as in enqueue_step.
cudaError_t enqueue_batch_step(const BatchDev& b, bool rescale_phase, cudaStream_t st);

}  // namespace fmd
