/*
 * fmd_oracle.h -- CPU restatement of fuller_md's per-step force-and-integrate
 * path, used ONLY as the checker by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py.  It is test infrastructure: nothing in the
 * product (the CUDA library, the C++ drivers, the Python package) links,
 * loads or calls it.
 *
 * Every function restates one reference routine in plain C99 with the same
 * floating-point operation order where the result feeds a discrete decision
 * (neighbour tests, cutoffs), so that neighbour sets are bit-exact.  The
 * restatement is pinned against the reference itself: oracle/Makefile
 * compiles the reference translation units unchanged into oracle/_ref/, and
 * tests/golden/gen_golden.py records their outputs as fixtures that
 * tests/test_oracle_golden.py checks this file against.
 *
 * Citations are to focusnishikawa/fuller_md_en, src/ directory:
 *   LJ   = fuller_LJ_npt_md_serial_omp_acc.cpp
 *   CORE = fuller_LJ_npt_md_core_serial.cpp
 *   AI   = fuller_airebo_npt_md_serial_omp_acc.cpp
 *   MM   = fuller_LJ_npt_mmmd_serial_omp_acc.cpp
 */
#ifndef FMD_ORACLE_H
#define FMD_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* NPT state, field for field as NPTState (LJ:425, AI:511, MM:804). */
typedef struct {
    double xi, Q, Vg[9], W, Pe, Tt;
    int Nf;
} fmo_npt;

/* ---- a4: cell geometry (LJ:113-151, AI:132-161) ---- */
double fmo_mat_det9(const double *h);
void fmo_mat_inv9(const double *h, double *hi);
void fmo_mimg(double *dx, double *dy, double *dz, const double *hi, const double *h);
void fmo_apply_pbc(double *pos, const double *h, const double *hi, int n);

/* ---- a1-a3: neighbour lists; each returns the number of dropped entries ---- */
int fmo_nlist_sym(const double *pos, const double *h, const double *hi, int n,
                  double rmcut, int max_neigh, int *cnt, int *list);          /* LJ:257 */
int fmo_nlist_half(const double *pos, const double *h, const double *hi, int na,
                   const int *mol_id, double rc_list, int max_neigh,
                   int *cnt, int *list);                                      /* AI:263, MM:337 */
int fmo_nlist_half_rows(const double *pos, const double *h, const double *hi, int na,
                        const int *mol_id, double rc_list, int max_neigh, int i0, int i1,
                        int *cnt, int *list);                                 /* rows [i0, i1) only */
int fmo_nlist_intra(const double *pos, const double *h, const double *hi, int na,
                    const int *mol_id, double rc, int max_neigh,
                    int *cnt, int *list);                                     /* AI:251 */

/* ---- a5-a6: rigid-body site-site LJ (LJ:271-400) ---- */
void fmo_lab_frame(const double *qv, const double *body, int n, int natom, double *lab);
double fmo_rigid_forces(double *F, double *T, double *W9,
                        const double *pos, const double *qv, const double *body,
                        const double *h, const double *hi,
                        const int *cnt, const int *list, int max_neigh,
                        int n, int natom, double rmcut2, double *lab);

/* ---- a7-a9: simplified AIREBO (AI:275-495) ---- */
double fmo_rebo(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                const int *cnt, const int *list, int max_neigh, int na);
/* Not the reference: fmo_rebo's energy with forces -grad E (its three-body
 * forces replaced by the bond-order gradient); adds into F, returns E. */
double fmo_rebo_grad(double *F, const double *pos, const double *h, const double *hi,
                     const int *cnt, const int *list, int max_neigh, int na);
/* Half-list shifted LJ.  full_virial=1: 9 components (AI:465-472);
 * full_virial=0: diagonal only (MM:751-763). */
typedef struct { double sig2, eps, rc2, vshift; int full_virial; } fmo_lj_params;
fmo_lj_params fmo_lj_params_airebo(void);   /* AI:119-124 */
fmo_lj_params fmo_lj_params_mm(void);       /* MM:113-116 */
double fmo_lj_half(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                   const int *cnt, const int *list, int max_neigh, int na,
                   const fmo_lj_params *p);
/* E[0]=total E[1]=rebo E[2]=lj; zeroes F and vir9 first (AI:477-495). */
void fmo_airebo_forces(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                       const int *cnt_r, const int *list_r, const int *cnt_l, const int *list_l,
                       int na, double *E);

/* ---- f4: REBO-II extension (rebo2_oracle.c; no reference counterpart) ----
 * Spline knots of the carbon-only terms, field for field as fmd_rebo2_knots
 * in include/fullermd.h: P_CC(N, 0) at N = 0..4 (value, dP/dN); pi^rc_CC and
 * T_CC on the integer knots N_ij, N_ji in 0..4, N_conj in 0..9 with
 * f, f_x, f_y, f_z, f_xy, f_xz, f_yz, f_xyz per knot. */
typedef struct {
    double pcc[5][2];
    double pirc[5][5][10][8];
    double tcc[5][5][10][8];
} fmo_rebo2_knots;
/* N_k = sum of f_c over k's REBO row. */
void fmo_rebo2_coordination(const double *pos, const double *h, const double *hi, const int *cnt,
                            const int *list, int max_neigh, int na, double *ncoord);
/* bbar_ij = (p_ij + p_ji)/2 + pi^rc + T sum(1 - cos^2) ... for bond vector dij = r_j - r_i. */
double fmo_rebo2_bond_order(const double *pos, const double *h, const double *hi, const int *cnt,
                            const int *list, int max_neigh, const fmo_rebo2_knots *kn, const double *ncoord,
                            int i, int j, const double *dij);
/* REBO-II energy over the bonds i < j of the REBO rows. */
double fmo_rebo2_energy(const double *pos, const double *h, const double *hi, const int *cnt, const int *list,
                        int max_neigh, int na, const fmo_rebo2_knots *kn);
/* Switched-LJ correction over the LJ half rows: sum of -V S(t_r) (1 - S(t_b(b*))). */
double fmo_lj_switch_energy(const double *pos, const double *h, const double *hi, const int *cnt_r,
                            const int *list_r, int max_neigh_r, const int *cnt_l, const int *list_l,
                            int max_neigh_l, int na, const fmo_rebo2_knots *kn);
double fmo_rebo2_spline3(const fmo_rebo2_knots *kn, int which, double x, double y, double z);
double fmo_rebo2_spline_p(const fmo_rebo2_knots *kn, double x);

/* ---- a10-a16: molecular mechanics (MM:226-788) ---- */
typedef struct {
    int nb;   const int *b_i0, *b_i1; const double *b_kb, *b_r0;
    int nang; const int *a_i0, *a_i1, *a_i2; const double *a_kth, *a_th0;
    int ndih; const int *d_i0, *d_i1, *d_i2, *d_i3; const double *d_vn; const int *d_mult; const double *d_gamma;
    int nimp; const int *m_i0, *m_i1, *m_i2, *m_i3; const double *m_ki, *m_gamma;
} fmo_mm_topo;
/* E[0..6] = Eb, Ea, Ed, Ei, Elj, Ecoul, Etot (ForceResult MM:349). */
void fmo_mm_forces(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                   const fmo_mm_topo *t, const int *cnt, const int *list,
                   const double *charge, const int *mol_id, int has_charge, int na, double *E);
/* Per-molecule topology from a bond list (MM:240-334).  Counts are returned
 * in counts[4] = {nb, nang, ndih, nimp}; arrays must hold at least
 * 4*nbond (bonds), 12*nbond (angles), 36*nbond (dihedrals), natom (impropers). */
double fmo_dihedral_angle(const double *c, int i, int j, int k, int l);
void fmo_mm_topology_mol(const double *coords, int natom, const int *bonds, int nbond,
                         int *counts,
                         int *b_idx, double *b_r0,
                         int *a_idx, double *a_th0,
                         int *d_idx, double *d_gamma,
                         int *m_idx, double *m_gamma);

/* ---- a17-a18: NPT velocity-Verlet steps ---- */
fmo_npt fmo_make_npt_rigid(double T, double Pe, int n);     /* LJ:426 */
fmo_npt fmo_make_npt_atom(double T, double Pe, int na);     /* AI:512, MM:805 */
double fmo_ke_trans(const double *vel, int n, double mmol); /* LJ:403 */
double fmo_ke_rot(const double *omg, int n, double i0);     /* LJ:412 */
double fmo_ke_atoms(const double *vel, const double *mass, int na); /* AI:498 */
double fmo_inst_T(double ke, int nf);
double fmo_inst_P(const double *W, double ke, double V);
/* Rigid step (LJ:434-538).  out[0]=Ep, out[1]=KE. */
void fmo_rigid_step(double *pos, double *vel, double *qv, double *omg,
                    double *F, double *T, double *W9, double *h, double *hi,
                    const double *body, double i0, double mmol,
                    int n, int natom, double rmcut2, double dt, fmo_npt *npt,
                    const int *cnt, const int *list, int max_neigh, double *lab, double *out);
/* AIREBO step (AI:518-590).  out = {Ep, Ep_rebo, Ep_lj, KE}. */
void fmo_airebo_step(double *pos, double *vel, double *F, double *vir9, double *h, double *hi,
                     const double *mass, int na, double dt, fmo_npt *npt,
                     const int *cnt_r, const int *list_r, const int *cnt_l, const int *list_l,
                     double *out);
/* MM step (MM:811-890).  out = {Eb, Ea, Ed, Ei, Elj, Ecoul, Etot, KE}. */
void fmo_mm_step(double *pos, double *vel, double *F, double *vir9, double *h, double *hi,
                 int na, double dt, fmo_npt *npt, const fmo_mm_topo *t,
                 const int *cnt, const int *list, const double *charge, const int *mol_id,
                 int has_charge, double *out);

#ifdef __cplusplus
}
#endif
#endif
