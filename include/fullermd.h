/*
 * fullermd.h -- C-ABI of libfullermd_cuda.so, the B200 (sm_100a) implementation
 * of fuller_md's per-step force-and-integrate path.
 *
 * Plain pointers and sizes only.  All arrays use the reference layouts: flat
 * row-major double, positions pos[3*i+c], quaternions qv[4*i+c] (w,x,y,z),
 * cell matrix h[3*r+c] whose COLUMNS are the lattice vectors, 9-component
 * virials W[3*a+b], neighbour lists list[i*max_neigh+k] with counts cnt[i].
 *
 * Two families of entry points:
 *  - host-pointer kernels (fmd_nlist_*, fmd_*_forces, fmd_*_step): each
 *    replaces one reference routine, takes and returns host arrays, copies
 *    them to and from the device, and is synchronous.  They are the parity
 *    boundary the tests check against the reference.
 *  - device-resident systems (fmd_system_*): own all state in HBM, run many
 *    steps with no host round trip (lists rebuilt on the device, the step
 *    replayed as a CUDA graph) and return observables.  The C++ drivers
 *    fuller_*_gpu are built on these.
 *
 * Every function returns an fmd_status; fmd_ctx_last_error() explains a
 * failure.  A context is bound to one device and one stream and is not
 * thread-safe.  Reference citations are to focusnishikawa/fuller_md_en src/:
 *   LJ = fuller_LJ_npt_md_serial_omp_acc.cpp, CORE = fuller_LJ_npt_md_core_serial.cpp,
 *   AI = fuller_airebo_npt_md_serial_omp_acc.cpp, MM = fuller_LJ_npt_mmmd_serial_omp_acc.cpp
 */
#ifndef FULLERMD_H
#define FULLERMD_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum fmd_status {
    FMD_OK = 0,
    FMD_ERR_ARG = 1,        /* bad argument (null pointer, size out of range) */
    FMD_ERR_CUDA = 2,       /* CUDA runtime error or extension not usable */
    FMD_ERR_CAPACITY = 3,   /* a fixed-size buffer would overflow */
    FMD_ERR_NONFINITE = 4,  /* NaN/Inf detected in the state */
    FMD_ERR_STATE = 5       /* call out of order (e.g. run before init) */
};

enum fmd_precision {
    FMD_PREC_FP64 = 0,      /* all pair arithmetic in FP64 */
    FMD_PREC_FP32_PAIR = 1  /* pair arithmetic in FP32; minimum image, cutoff tests
                               and force/energy/virial sums in FP64 */
};

/* Opt-in physics corrections (no reference counterpart; off by default, so a
 * system computes the reference's forces).  FMD_PHYS_MM_BONDED: every MM
 * bonded force is -grad E of the MM energy: bond and angle forces negated
 * (the reference's equal +grad E, MM:389-398, MM:468-491) and the dihedral
 * and improper forces on the two middle atoms taken from the gradient (the
 * reference's projection terms have the opposite sign, MM:500-709).
 * FMD_PHYS_REBO: REBO forces are -grad E of the REBO energy: the bond-order
 * term's gradient replaces the reference's three-body forces (opposite sign
 * on the neighbours, no term on the bond partner, AI:361-419).  The learned
 * REBO term, when attached, is not affected.  FMD_PHYS_QUAT (rigid): the
 * quaternion's rotation increment from the lab-frame angular velocity
 * multiplies q on the left (the reference's on the right applies it as a
 * body-frame one, LJ:166-174, LJ:503-508). */
enum fmd_physics { FMD_PHYS_MM_BONDED = 1, FMD_PHYS_REBO = 2, FMD_PHYS_QUAT = 4 };

enum fmd_forcefield { FMD_FF_AIREBO = 0, FMD_FF_MM = 1 };
enum fmd_kind { FMD_SYS_RIGID = 0, FMD_SYS_AIREBO = 1, FMD_SYS_MM = 2 };

typedef struct fmd_ctx fmd_ctx;

/* NPT thermostat/barostat state, field for field as NPTState
 * (LJ:425, AI:511, MM:804). */
typedef struct {
    double xi, Q, Vg[9], W, Pe, Tt;
    int Nf;
} fmd_npt;

/* Flat MM topology, as FlatTopology (MM:226-237) without mol_id. */
typedef struct {
    int nb;   const int *b_i0, *b_i1; const double *b_kb, *b_r0;
    int nang; const int *ang_i0, *ang_i1, *ang_i2; const double *ang_kth, *ang_th0;
    int ndih; const int *dih_i0, *dih_i1, *dih_i2, *dih_i3; const double *dih_vn;
              const int *dih_mult; const double *dih_gamma;
    int nimp; const int *imp_i0, *imp_i1, *imp_i2, *imp_i3; const double *imp_ki, *imp_gamma;
} fmd_mm_topology;

/* ------------------------------------------------------------------ context */
int fmd_version(void);
int fmd_ctx_create(fmd_ctx **out, int device);
int fmd_ctx_destroy(fmd_ctx *ctx);
/* Use the caller's CUDA stream (a cudaStream_t) instead of the context's own. */
int fmd_ctx_set_stream(fmd_ctx *ctx, void *cuda_stream);
void *fmd_ctx_get_stream(fmd_ctx *ctx);
int fmd_ctx_synchronize(fmd_ctx *ctx);
/* Pair arithmetic of the atomistic LJ term (AIREBO and MM) in this context's
 * host-pointer calls (fmd_precision; default FMD_PREC_FP64, the reference's
 * arithmetic).  No counterpart in the reference. */
int fmd_ctx_set_precision(fmd_ctx *ctx, int precision);
const char *fmd_ctx_last_error(const fmd_ctx *ctx);
const char *fmd_status_string(int code);
/* Device name and total memory in GiB (the drivers' banner; replaces the
 * OpenACC device queries acc_get_num_devices/acc_get_property, LJ:726-739). */
int fmd_device_info(int device, char *name, int name_cap, double *total_gib);

/* ------------------------------------------------------- host-pointer kernels */
/* mat_inv9 (LJ:120-124), evaluated on the device. */
int fmd_mat_inv9(fmd_ctx *ctx, const double *h, double *hi);
/* apply_pbc (LJ:137-151, AI:149-161). */
int fmd_apply_pbc(fmd_ctx *ctx, double *pos, const double *h, const double *hi, int n);

/* nlist_build_sym (LJ:257-268, CORE:280-301): symmetric molecule list, pair
 * test |mimg(r_j-r_i)|^2 < (rmcut+3)^2, rows ascending, first max_neigh kept.
 * *dropped (may be NULL) receives the number of entries that did not fit. */
int fmd_nlist_rigid(fmd_ctx *ctx, const double *pos, const double *h, const double *hi, int n,
                    double rmcut, int max_neigh, int *nl_count, int *nl_list, int *dropped);
/* build_nlist_lj (AI:263-272, MM:337-346): intermolecular half list, j>i
 * ascending, |d|^2 < rc_list^2, first max_neigh kept. */
int fmd_nlist_lj_half(fmd_ctx *ctx, const double *pos, const double *h, const double *hi, int na,
                      const int *mol_id, double rc_list, int max_neigh, int *nlc, int *nll,
                      int *dropped);
/* build_nlist_rebo (AI:251-261): intramolecular symmetric list, |d|^2 < rc^2. */
int fmd_nlist_rebo(fmd_ctx *ctx, const double *pos, const double *h, const double *hi, int na,
                   const int *mol_id, double rc, int max_neigh, int *nlc, int *nll, int *dropped);

/* forces (LJ:271-400, CORE:346-444): lab-frame sites from quaternions, then
 * site-site shifted LJ over the symmetric list.  Overwrites Fv, Tv, Wm9;
 * *Ep = potential energy. */
int fmd_lj_rigid_forces(fmd_ctx *ctx, const double *pos, const double *qv, const double *body,
                        const double *h, const double *hi, const int *nl_count, const int *nl_list,
                        int max_neigh, int n, int natom, double rmcut2, int precision,
                        double *Fv, double *Tv, double *Wm9, double *Ep);
/* compute_rebo (AI:275-421): ADDS into F and vir9 like the reference; *E = energy. */
int fmd_rebo_forces(fmd_ctx *ctx, const double *pos, const double *h, const double *hi,
                    const int *nlc, const int *nll, int max_neigh, int na,
                    double *F, double *vir9, double *E);
/* No counterpart in the reference.  The REBO force of fmd_rebo_forces for
 * callers that cannot allocate device memory: programs whose memory pool or
 * allocator owns all device memory and forbids side allocations, and drivers
 * that must not touch the allocator after start-up.  It needs no fmd_ctx and
 * calls no cudaMalloc/cudaFree or any allocating routine.  All arrays are
 * DEVICE pointers except h and hi (9 doubles each, host, read during the
 * call and passed to the GPU by value): d_pos[3*na], the REBO list
 * d_nlc[na], d_nll[na*max_neigh] (entries must be valid atom indices, as
 * fmd_nlist_rebo produces them); d_F[3*na] and d_vir9[9] are ADDED into like
 * compute_rebo (AI:275-421) does; *d_E receives the REBO energy.  The device
 * is the one holding d_pos; the caller's current device is unchanged on
 * return.  Work is enqueued on `stream` (a cudaStream_t, NULL = default
 * stream) and the call returns without synchronising.  Scratch is a fixed
 * file-scope device array (82 KB on every GPU that loads the library, held
 * until exit) for the cell matrix and 1,024 partial {E, W} records: na is
 * limited to 131,072; larger na returns FMD_ERR_CAPACITY and does nothing.
 * Every call shares that array and it keeps the last call's contents (each
 * call rewrites all it reads), so calls that overlap on the GPU -- on
 * different streams, or from several host threads -- race and must be
 * serialised by the caller.  The first call on a device looks up the
 * array's device address; make that first call before any stream capture. */
int fmd_rebo_forces_noalloc(const double *d_pos, const double *h, const double *hi,
                            const int *d_nlc, const int *d_nll, int max_neigh, int na,
                            double *d_F, double *d_vir9, double *d_E, void *stream);
/* compute_lj (AI:424-473) for ff=FMD_FF_AIREBO, MM LJ block (MM:711-764) for
 * ff=FMD_FF_MM: ADDS into F and vir9; *E = energy. */
int fmd_lj_half_forces(fmd_ctx *ctx, int ff, const double *pos, const double *h, const double *hi,
                       const int *nlc, const int *nll, int max_neigh, int na,
                       double *F, double *vir9, double *E);
/* compute_forces (AI:477-495): zeroes F, vir9; E3 = {Ep, Ep_rebo, Ep_lj}.
 * Lists use the reference widths 12 (REBO) and 400 (LJ). */
int fmd_airebo_forces(fmd_ctx *ctx, const double *pos, const double *h, const double *hi,
                      const int *nlc_r, const int *nll_r, const int *nlc_l, const int *nll_l,
                      int na, double *F, double *vir9, double *E3);
/* ---- REBO-II extension (no counterpart in the reference) ----
 * The reference's REBO bond order is b = (1 + sum f_c G)^-1/2 (AI:301-323).
 * The extension adds, for carbon-only systems, the terms of Brenner et al.,
 * J. Phys.: Condens. Matter 14 (2002) 783:
 *   bbar = (p_ij + p_ji)/2 + pi^rc + pi^dh,
 *   p_ij = (1 + sum_k f_c G + P_CC(N_ij))^-1/2,  pi^rc = F_CC(N_ij, N_ji, N_conj),
 *   pi^dh = T_CC(N_ij, N_ji, N_conj) sum_kl (1 - cos^2 w_kijl) f_c(r_ik) f_c(r_jl)
 *           tau(cos theta_jik) tau(cos theta_ijl)
 * (N_ij = sum_{k != j} f_c(r_ik); N_conj = 1 + A_ij^2 + A_ji^2 with
 * A_ij = sum_{k != j} f_c(r_ik) F(N_k - f_c(r_ik)); tau = 1 for |cos| <= 0.995,
 * cubic switch to 0 at |cos| = 1), and AIREBO's switched LJ (Stuart, Tutein,
 * Harrison, J. Chem. Phys. 112 (2000) 6472) over the reference's LJ pairs:
 * V(r) [1 - S(t_r) (1 - S(t_b(b*)))], t_r = (r - sigma)/(2^(1/6) sigma - sigma),
 * t_b = (b* - 0.77)/0.04, b* the bond order of the pair's own direction.
 * f_c, V_R, V_A, G and the LJ V are the reference's (AI:119-124, 164-191).
 * Forces are -grad E and the virial is the full virial of every term.  The
 * spline tables are the caller's: cubic Hermite in each variable through
 * values and derivatives given at integer knots (with every knot zero the
 * bond order is the reference's). */
typedef struct fmd_rebo2_knots {
    double pcc[5][2];           /* P_CC(N, N_H = 0) at N = 0..4: {P, dP/dN} */
    double pirc[5][5][10][8];   /* pi^rc_CC at N_ij, N_ji = 0..4, N_conj = 0..9:
                                   {f, f_x, f_y, f_z, f_xy, f_xz, f_yz, f_xyz} */
    double tcc[5][5][10][8];    /* T_CC, same layout */
} fmd_rebo2_knots;
enum fmd_rebo2_flags { FMD_REBO2_BOND_ORDER = 1, FMD_REBO2_LJ_SWITCH = 2 };
/* Host only (no GPU needed): the splines' per-cell polynomial coefficients
 * that the kernels evaluate, out[16 + 2 * 9216]: P_CC as out[4 n + a] (u^a on
 * cell [n, n+1)), then pi^rc_CC and T_CC as [((x * 4 + y) * 9 + z) * 64 +
 * a + 4 b + 16 c] (u^a v^b w^c on the cell at (x, y, z)), u, v, w the
 * offsets from the cell's lower knots.  Arguments beyond the knots are
 * clamped to them. */
int fmd_rebo2_coeffs(const fmd_rebo2_knots *kn, double *out);
/* REBO-II energy over the bonds i < j of the REBO rows (the enumeration of
 * AI:286-290): ADDS -grad E into F and the virial into vir9; *E = energy. */
int fmd_rebo2_forces(fmd_ctx *ctx, const double *pos, const double *h, const double *hi,
                     const int *nlc, const int *nll, int max_neigh, int na, const fmd_rebo2_knots *kn,
                     double *F, double *vir9, double *E);
/* The switched-LJ correction over the LJ half rows (nlc_l, nll_l): *E = sum of
 * -V S(t_r) (1 - S(t_b(b*))); ADDS its -grad into F and its virial into vir9.
 * The switched LJ term is fmd_lj_half_forces (FMD_FF_AIREBO) plus this. */
int fmd_lj_switch_forces(fmd_ctx *ctx, const double *pos, const double *h, const double *hi,
                         const int *nlc_r, const int *nll_r, int max_neigh_r,
                         const int *nlc_l, const int *nll_l, int max_neigh_l, int na,
                         const fmd_rebo2_knots *kn, double *F, double *vir9, double *E);

/* compute_forces (MM:351-788): zeroes F, vir9;
 * E7 = {Eb, Ea, Ed, Ei, Elj, Ecoul, Etot}.  LJ list width 400. */
int fmd_mm_forces(fmd_ctx *ctx, const fmd_mm_topology *t, const double *pos, const double *h,
                  const double *hi, const int *nlc, const int *nll, const double *charge,
                  const int *mol_id, int has_charge, int na, double *F, double *vir9, double *E7);

/* step_npt (LJ:434-538): one rigid NPT step on host state; out2 = {Ep, KE}. */
int fmd_rigid_step(fmd_ctx *ctx, double *pos, double *vel, double *qv, double *omg,
                   double *Fv, double *Tv, double *Wm9, double *h, double *hi,
                   const double *body, double I0, double Mmol, int n, int natom, double rmcut2,
                   double dt, fmd_npt *npt, const int *nl_count, const int *nl_list,
                   int max_neigh, int precision, double *out2);
/* step_npt (AI:518-590); out4 = {Ep, Ep_rebo, Ep_lj, KE}. */
int fmd_airebo_step(fmd_ctx *ctx, double *pos, double *vel, double *F, double *vir9,
                    double *h, double *hi, const double *mass, int na, double dt, fmd_npt *npt,
                    const int *nlc_r, const int *nll_r, const int *nlc_l, const int *nll_l,
                    double *out4);
/* step_npt (MM:811-890); out8 = {Eb, Ea, Ed, Ei, Elj, Ecoul, Etot, KE}. */
int fmd_mm_step(fmd_ctx *ctx, double *pos, double *vel, double *F, double *vir9, double *h,
                double *hi, int na, double dt, fmd_npt *npt, const fmd_mm_topology *t,
                const int *nlc, const int *nll, const double *charge, const int *mol_id,
                int has_charge, double *out8);

/* ------------------------------------------------------ device-resident systems */
typedef struct fmd_system fmd_system;

/* Run schedule of a driver (LJ:830-897, AI:855-912, MM:1174-1236). */
typedef struct {
    double dt, T, Pe, T_cold;
    int coldstart, warmup, nsteps;   /* total steps = coldstart + warmup + nsteps */
    int nlup;                        /* list rebuild cadence (25 rigid, 20 atomistic) */
    int gavg_from, gavg_to;          /* global-step averaging window */
    int nc;                          /* lattice repeats, for a = h[0]/nc */
    int nmol;                        /* energies are reported per molecule */
    int precision;                   /* fmd_precision of the pair kernel (rigid site-site
                                        LJ, atomistic LJ of AIREBO and MM) */
    int use_graphs;                  /* 1: replay steps as CUDA graphs */
} fmd_run_params;

/* Observables of one step, as the reference monitor line computes them. */
typedef struct {
    int step;
    double T, P, a, KE;
    double E[8];   /* rigid: {Ep}; AIREBO: {Ep, Ep_rebo, Ep_lj};
                      MM: {Eb, Ea, Ed, Ei, Elj, Ecoul, Etot} -- totals, not per molecule */
} fmd_obs;

/* Running averages over the window (the reference's sT, sP, sa, sE... sums). */
typedef struct {
    int n;
    double sT, sP, sa;
    double sE[8];  /* per-molecule energy sums in the program's own grouping */
} fmd_avg;

/* Rigid LJ system (LJ main, LJ:742-944).  pos/vel/qv/omg: n molecules. */
int fmd_system_create_rigid(fmd_ctx *ctx, const fmd_run_params *p, int n, int natom,
                            const double *body, double I0, double Mmol, double rmcut,
                            int max_neigh, const double *pos, const double *vel, const double *qv,
                            const double *omg, const double *h, const fmd_npt *npt,
                            fmd_system **out);
/* AIREBO system (AI main, AI:771-955). */
int fmd_system_create_airebo(fmd_ctx *ctx, const fmd_run_params *p, int na, const double *pos,
                             const double *vel, const double *mass, const int *mol_id,
                             const double *h, const fmd_npt *npt, fmd_system **out);
/* MM system (MM main, MM:1094-1279). */
int fmd_system_create_mm(fmd_ctx *ctx, const fmd_run_params *p, int na, const double *pos,
                         const double *vel, const int *mol_id, const fmd_mm_topology *t,
                         const double *charge, const double *h, const fmd_npt *npt,
                         fmd_system **out);
/* MM system of nmol molecules of natom_mol atoms each (atoms of molecule m
 * at m*natom_mol .. (m+1)*natom_mol-1), no charges (the reference's are all
 * zero, MM:1098-1111), built from ONE molecule's topology t1 (indices
 * 0..natom_mol-1): the copies of build_flat_topology's replication
 * (MM:254-334) are made on the device, term k of molecule m being t1's term
 * k with every index offset by m*natom_mol, each term kind molecule-major --
 * the arrays fmd_system_create_mm receives from a full flat topology. */
int fmd_system_create_mm_replicated(fmd_ctx *ctx, const fmd_run_params *p, int nmol, int natom_mol,
                                    const double *pos, const double *vel, const fmd_mm_topology *t1,
                                    const double *h, const fmd_npt *npt, fmd_system **out);
/* The reference's pre-loop work: apply_pbc, neighbour lists, first forces
 * (LJ:813-828, AI:830-853, MM:1152-1172). */
int fmd_system_init(fmd_system *s);
/* Advances global steps first..last inclusive (driver loop body of
 * LJ:847-897 etc., including list rebuilds, the temperature schedule,
 * cold/warm rescaling and window averages).  *last receives the observables
 * of step `last` (may be NULL). */
int fmd_system_run(fmd_system *s, int first, int last, fmd_obs *obs);
/* As fmd_system_run but only enqueues the steps on the context stream and
 * returns without synchronising (errors surface at the next synchronising
 * call). */
int fmd_system_enqueue(fmd_system *s, int first, int last);
/* As fmd_system_enqueue, then an asynchronous copy of the observables of
 * step `last` into *obs (host memory; page-locked for the copy to run without
 * a host round trip), so a caller can enqueue the next steps before it reads
 * these: the copy is complete once fmd_system_wait_obs(s, last) returns.  The
 * completion marks alternate by the parity of `last`: at most two copies may
 * be waited for at once.  Errors surface at the next synchronising call. */
int fmd_system_enqueue_obs(fmd_system *s, int first, int last, fmd_obs *obs);
int fmd_system_wait_obs(fmd_system *s, int step);
int fmd_system_averages(fmd_system *s, fmd_avg *avg);
/* Copies the state to host arrays (any may be NULL). */
int fmd_system_download(fmd_system *s, double *pos, double *vel, double *qv, double *omg,
                        double *h, fmd_npt *npt);
/* Forces (3 n doubles; rigid systems: centre-of-mass forces) of the last force
 * evaluation, torques (rigid only, 3 n) and its energies E[8] in the program's
 * grouping (AIREBO: total, REBO, LJ; MM: bond, angle, dihedral, improper, LJ,
 * Coulomb, total; rigid: LJ); any pointer may be null. */
int fmd_system_forces(fmd_system *s, double *F, double *T, double *E);
/* Virial tensor W9 of the last force evaluation and the current kinetic
 * energy (eV; rigid: translational + rotational); either may be NULL. */
int fmd_system_virial(fmd_system *s, double *W9, double *KE);
/* Current neighbour lists (reference layout) for inspection. */
int fmd_system_lists(fmd_system *s, int *cnt_a, int *list_a, int *cnt_b, int *list_b);
/* Row lengths of the atomistic LJ gather (n ints each, either may be NULL):
 * the full rows (incoming entries + the reference row) of the last list build
 * and the pruned rows of the last prune (see fmd_system_set_lj_prune). */
int fmd_system_lj_rows(fmd_system *s, int *full_cnt, int *pruned_cnt);
/* The full rows themselves: *stride = the row stride (0 for a system without
 * them, e.g. the rigid model); cnt (n ints) and list (n * stride ints), when
 * not NULL, receive the row lengths and rows -- row j holds the atoms i < j
 * whose reference row lists j, ascending, then j's own reference row. */
int fmd_system_lj_full_rows(fmd_system *s, int *cnt, int *list, int *stride);
/* Physics corrections (fmd_physics bits) of a system; before fmd_system_init.
 * A bit the system's force field lacks is an FMD_ERR_ARG. */
int fmd_system_set_physics(fmd_system *s, int flags);
/* REBO-II extension in an AIREBO system (see fmd_rebo2_knots): flags
 * FMD_REBO2_BOND_ORDER replaces the REBO term, FMD_REBO2_LJ_SWITCH switches the
 * LJ term; 0 turns both off.  Call before fmd_system_init; not with a learned
 * REBO term.  The system's energies and virial then hold the extended terms
 * (E[1] REBO-II, E[2] the switched LJ). */
int fmd_system_set_rebo2(fmd_system *s, const fmd_rebo2_knots *kn, int flags);
int fmd_system_destroy(fmd_system *s);

/* Measurement helpers (no reference counterpart).  fmd_system_kernel_ms
 * launches one stage `reps` times on the context stream between CUDA events
 * and returns the mean duration per launch in milliseconds; stages:
 *   0 the pair kernel (rigid site-site LJ, or the atomistic LJ gather),
 *   1 the second force kernel (REBO -- REBO-II when the system uses it --,
 *     or MM bonded), 2 a full list rebuild,
 *   3 the whole force evaluation of a step (eager launches),
 *   4 the atomistic LJ gather over the pruned rows of the last prune (see
 *     fmd_system_set_lj_prune),
 *   5 the switched-LJ correction (systems with FMD_REBO2_LJ_SWITCH).
 * The force stages leave F in place (they recompute the current forces).
 * fmd_system_step_kernels returns the number of kernel launches of one step
 * of each variant (list rebuild or not; phase bit 0: cold/warm phase, bit 1:
 * a judge step of the learned REBO term). */
int fmd_system_kernel_ms(fmd_system *s, int stage, int reps, double *ms_per_launch);
/* Launch shape of the atomistic LJ gather that fmd_system_init's autotuner
 * chose (threads per block 128/256, list entries in flight per lane 2/4,
 * row feed 0 loads as used / 1 software-pipelined / 2 rows staged in shared
 * memory by bulk asynchronous copies, plus 4 when each block walks its own
 * contiguous run of atoms instead of atoms strided over the grid; grid
 * blocks); any pointer may be NULL.
 * fmd_system_set_lj_shape pins a shape (for reproducible runs; results then
 * do not depend on timing), after fmd_system_init. */
int fmd_system_lj_shape(fmd_system *s, int *threads, int *unroll, int *pipelined, int *blocks);
/* Launch shape of the gather over the pruned rows, tuned separately on those
 * rows at set-up (the same shape when pinned by FMD_LJ_SHAPE or set_lj_shape). */
int fmd_system_lj_shape_pruned(fmd_system *s, int *threads, int *unroll, int *feed);
/* Pruned rows of the atomistic LJ gather (AIREBO, MM; the reference walks
 * its whole list every step, AI:435-470, MM:729-760).  After each list build,
 * and whenever the largest atom displacement u and the largest relative
 * cell-edge change k since the last prune reach k (rc + delta) + 2 u >= delta,
 * the gather walks the full rows and keeps each row's entries within
 * rc + delta, in row order; other steps walk those rows.  Every pair within
 * the cutoff stays in them, so the pairs and pair terms are the full rows'
 * (on non-diagonal cells every step prunes).  delta in A: 0 = off, default
 * 0.5.  fmd_system_lj_prune reports delta and the numbers of force
 * evaluations and of prunes among them since set-up. */
int fmd_system_set_lj_prune(fmd_system *s, double delta);
int fmd_system_lj_prune(fmd_system *s, double *delta, long long *evaluations, long long *prunes);
int fmd_system_set_lj_shape(fmd_system *s, int threads, int unroll, int feed);
int fmd_system_step_kernels(fmd_system *s, int rebuild, int phase, int *nkernels);
/* Rigid systems: the number of site pairs within the LJ cutoff in the
 * current state (the reference's FP64 test, LJ:320-336; each molecule pair
 * once): the work count of the site-pair kernel.  Overwrites the system's
 * lab-frame site scratch (the next force evaluation rebuilds it). */
int fmd_system_site_pairs(fmd_system *s, long long *pairs);

/* ------------------------------------------------------- replica batches --
 * No counterpart in the reference (its programs run one system each).  A
 * batch advances R MM systems of one context together -- different sizes,
 * cells, temperatures and pressures -- with every phase of the step one
 * launch over all replicas and each step one CUDA graph; every replica gets
 * the results of its own kernels run alone.  The systems stay owned by the
 * caller (they must outlive the batch) and keep serving fmd_system_download,
 * fmd_system_averages and fmd_system_lists; they must share nlup, coldstart,
 * warmup and precision, carry no charges and no learned REBO term, and are
 * initialised here if they are not yet.  autotune != 0 times the LJ gather
 * and bonded kernels over candidate launch shapes on the batch itself and
 * keeps the fastest (cached per device, replica count and atom count; the
 * forces of the current state are recomputed afterwards). */
typedef struct fmd_batch fmd_batch;
typedef struct {
    int lj_threads;               /* threads per block of the LJ gather */
    int lj_unroll;                /* list entries in flight per lane (neighbours per warp / 32) */
    int lj_atoms_per_block;       /* sites per block of the LJ gather */
    int lj_staged;                /* 1: LJ rows staged in shared memory by bulk asynchronous copies */
    int bonded_threads;           /* threads per block of the bonded terms */
    int bonded_terms_per_block;
    double lj_ms, bonded_ms;      /* timed duration of the chosen shapes, ms per launch */
    int blocks_lj, blocks_bonded, blocks_atom;   /* launch sizes over the whole batch */
} fmd_batch_tuning;
int fmd_batch_create(fmd_ctx *ctx, int nrep, fmd_system *const *systems, int autotune, fmd_batch **out);
/* Global steps first..last of every replica (as fmd_system_run); _run
 * synchronises, _enqueue does not. */
int fmd_batch_run(fmd_batch *b, int first, int last);
int fmd_batch_enqueue(fmd_batch *b, int first, int last);
/* Observables of the last step of each replica: obs[nrep]. */
int fmd_batch_observables(fmd_batch *b, fmd_obs *obs);
int fmd_batch_get_tuning(fmd_batch *b, fmd_batch_tuning *t);
/* Kernel launches of one batch step (rebuild or not, cold/warm phase or not):
 * the kernels of the step's graph that run on every replay.  A rebuild step
 * of a batch whose replicas all use the molecule-wise list builder also
 * holds a conditional node whose kernels (every replica's cell-grid
 * fallback, counted by fmd_batch_step_kernels_conditional) run only when
 * some replica's molecule path is rejected for that build. */
int fmd_batch_step_kernels(fmd_batch *b, int rebuild, int phase, int *nkernels);
int fmd_batch_step_kernels_conditional(fmd_batch *b, int rebuild, int phase, int *nkernels);
int fmd_batch_destroy(fmd_batch *b);


/* ------------------------------------------- learned bond-order potential --
 * No counterpart in the reference.  A network stands in for the bond order
 * b_ij of compute_rebo (AI:275-421); the pair functions, b_bar and the
 * reference's force construction are kept.  Row = directed bond i->j of the
 * REBO list with r_ij <= 2.0; its 32 descriptors are sums over i's other
 * bonded neighbours k of fc(r_ik) T_a((r_ik-1.55)/0.45) T_b(cos theta_jik)
 * (Chebyshev T, a<4, b<8; descriptor 31 is a constant bias input).  Network:
 * three 128-wide SiLU layers (unit 127 of each is a constant bias unit),
 * linear output y, b = b0 + bs*y, evaluated with BF16 operands and FP32
 * accumulation on the tensor cores.
 * Parameter vector (doubles, fmd_sg_nparams() of them):
 *   W1[32][128] W2[128][128] W3[128][128] w4[128] m[32] s[32] b0 bs
 * (W[in][out]; descriptors are normalised as (x-m)/s before the network). */
typedef struct fmd_sg fmd_sg;
int fmd_sg_nparams(void);
int fmd_sg_create(fmd_ctx *ctx, const double *params, fmd_sg **out);
int fmd_sg_set_params(fmd_sg *s, const double *params);
int fmd_sg_get_params(fmd_sg *s, double *params);
int fmd_sg_destroy(fmd_sg *s);
/* As fmd_rebo_forces with the learned bond order: ADDS into F and vir9,
 * *E = energy.  The REBO list must be symmetric (as fmd_nlist_rebo makes it). */
int fmd_sg_rebo_forces(fmd_sg *s, const double *pos, const double *h, const double *hi, const int *nlc,
                       const int *nll, int max_neigh, int na, double *F, double *vir9, double *E);
/* Rows of the last fmd_sg_rebo_forces call: *nrows, and (each may be NULL)
 * row_i, row_j, normalised BF16 descriptors xn[rows*32] as floats, b[rows],
 * gx[rows*32] = db/dxn.  cap_rows = capacity of the arrays. */
int fmd_sg_last_rows(fmd_sg *s, int cap_rows, int *nrows, int *row_i, int *row_j, float *xn, float *b, float *gx);

/* Training data: snapshots whose reference REBO energy, forces and virial are
 * computed on the device by the plain REBO kernel (fmd_rebo_forces). */
typedef struct fmd_sg_data fmd_sg_data;
int fmd_sg_data_create(fmd_ctx *ctx, fmd_sg_data **out);
int fmd_sg_data_destroy(fmd_sg_data *d);
int fmd_sg_data_count(const fmd_sg_data *d);
int fmd_sg_data_add(fmd_sg_data *d, const double *pos, const double *h, const double *hi, const int *nlc,
                    const int *nll, int max_neigh, int na);
/* Current state of a running AIREBO system (device to device). */
int fmd_sg_data_add_system(fmd_sg_data *d, fmd_system *sys);
/* Reference values of snapshot k: *na, *E, W9[9], F[3*na] (any may be NULL but na). */
int fmd_sg_data_get(fmd_sg_data *d, int k, int *na, double *E, double *W9, double *F);

/* Mean and standard deviation of the raw descriptors over the rows of
 * snapshots [first, first+n): the normalisation m, s of a new model. */
int fmd_sg_feature_stats(fmd_sg *s, fmd_sg_data *d, int first, int n, double *mean, double *stdev);

/* Loss L = wF mean(dF^2) + wE (dE/na)^2 + wW mean((dW/na)^2) of the REBO
 * term against given reference values, and dL/dparams (the layout of the
 * parameter vector; zeros for m, s, b0, bs, which do not train). */
int fmd_sg_loss_grad(fmd_sg *s, const double *pos, const double *h, const double *hi, const int *nlc,
                     const int *nll, int max_neigh, int na, const double *F_ref, double E_ref,
                     const double *W_ref, double wE, double wF, double wW, double *loss, double *grad);

typedef struct {
    int steps;          /* Adam updates */
    int batch;          /* snapshots per update (drawn uniformly with `seed`) */
    int n_train;        /* draw from snapshots [0, n_train); <= 0: all */
    int seed;
    double lr, lr_final;  /* cosine schedule from lr to lr_final */
    double wE, wF, wW;  /* loss weights */
    double clip;        /* per-component gradient clip (<= 0: none) */
} fmd_sg_train_args;
/* Adam training with the tensor-core forward/backward kernels.
 * history[2*k] = mean loss of step k, history[2*k+1] = force RMSE of step k
 * (eV/A, over the step's batch, before the update); may be NULL. */
int fmd_sg_train(fmd_sg *s, fmd_sg_data *d, const fmd_sg_train_args *a, double *history);
/* Force RMSE (eV/A) against the reference REBO forces of snapshots
 * [first, first+n): rmse[n]. */
int fmd_sg_eval(fmd_sg *s, fmd_sg_data *d, int first, int n, double *rmse);

/* Learned REBO term inside a device-resident AIREBO system (no counterpart
 * in the reference).  From the next step on, the system's REBO term comes
 * from `model`; the plain REBO kernel stays beside it as judge and fallback:
 * on every global step divisible by judge_every (0: never) it evaluates the
 * same positions, the force RMSE sqrt(mean_k (F_learned,k - F_plain,k)^2)
 * over the 3n components is recorded, and if it exceeds rmse_max (eV/A) the
 * plain result replaces the learned one for that step and the plain kernel
 * takes over for the rest of the run.  Everything stays on the device and
 * inside the step's CUDA graph.  model == NULL returns to the plain kernel.
 * Each call resets the judge record; if the system is initialised, the
 * current forces are recomputed with the new term.  The model must outlive
 * its use by the system; fmd_sg_set_params takes effect at the next step. */
typedef struct {
    int attached;        /* a model is attached */
    int active;          /* the learned term is in use (no takeover yet) */
    int judged;          /* judge evaluations so far */
    int takeover_step;   /* global step of the takeover, 0: none */
    double rmse_last;    /* force RMSE of the last judge step, eV/A */
    double rmse_max;     /* largest judged force RMSE, eV/A */
} fmd_sg_status;
int fmd_system_use_surrogate(fmd_system *s, fmd_sg *model, int judge_every, double rmse_max);
int fmd_system_surrogate_status(fmd_system *s, fmd_sg_status *st);

#ifdef __cplusplus
}
#endif
#endif
