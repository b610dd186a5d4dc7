/*
 * fmd_oracle.c -- CPU restatement of fuller_md's force-and-integrate path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the checker.
 * The product path (fuller_md_en_b200/) never links or calls it.
 *
 * Parity pin: tests/test_oracle_golden.py checks every function here against
 * fixtures recorded from the unmodified reference (oracle/_ref, built by
 * oracle/Makefile from the reference sources) -- except fmo_rebo_grad, which
 * is not the reference's arithmetic (the gradient of its REBO energy, for the
 * opt-in physics tests) and is checked by finite differences instead.
 *
 * Build: gcc -std=c99 -O2 -ffp-contract=off (no FMA contraction), so that the
 * distance tests round exactly like the reference built by g++ -O3 on x86-64.
 * Citations: LJ/CORE/AI/MM as listed in fmd_oracle.h.
 */
#include "fmd_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Units and constants (LJ:101-107, AI:105-124, MM:109-119). */
#define CONV 9.64853321e-3
#define KB 8.617333262e-5
#define EV2GPA 160.21766208
#define PI_D 3.14159265358979323846

/* ------------------------------------------------------------------ a4 */

/* LJ:114-117 (cofactor expansion along the first row). */
double fmo_mat_det9(const double *h)
{
    return h[0] * (h[4] * h[8] - h[5] * h[7])
         - h[1] * (h[3] * h[8] - h[5] * h[6])
         + h[2] * (h[3] * h[7] - h[4] * h[6]);
}

/* LJ:120-124: adjugate scaled by 1/det. */
void fmo_mat_inv9(const double *h, double *hi)
{
    double id = 1.0 / fmo_mat_det9(h);
    hi[0] = id * (h[4] * h[8] - h[5] * h[7]);
    hi[1] = id * (h[2] * h[7] - h[1] * h[8]);
    hi[2] = id * (h[1] * h[5] - h[2] * h[4]);
    hi[3] = id * (h[5] * h[6] - h[3] * h[8]);
    hi[4] = id * (h[0] * h[8] - h[2] * h[6]);
    hi[5] = id * (h[2] * h[3] - h[0] * h[5]);
    hi[6] = id * (h[3] * h[7] - h[4] * h[6]);
    hi[7] = id * (h[1] * h[6] - h[0] * h[7]);
    hi[8] = id * (h[0] * h[4] - h[1] * h[3]);
}

/* LJ:128-135 / AI:144-147: one image per pair, chosen by round() of each
 * fractional component. */
void fmo_mimg(double *dx, double *dy, double *dz, const double *hi, const double *h)
{
    double x = *dx, y = *dy, z = *dz;
    double s0 = hi[0] * x + hi[1] * y + hi[2] * z;
    double s1 = hi[3] * x + hi[4] * y + hi[5] * z;
    double s2 = hi[6] * x + hi[7] * y + hi[8] * z;
    s0 -= round(s0);
    s1 -= round(s1);
    s2 -= round(s2);
    *dx = h[0] * s0 + h[1] * s1 + h[2] * s2;
    *dy = h[3] * s0 + h[4] * s1 + h[5] * s2;
    *dz = h[6] * s0 + h[7] * s1 + h[8] * s2;
}

/* LJ:137-151: wrap into the cell with floor() in fractional coordinates. */
void fmo_apply_pbc(double *pos, const double *h, const double *hi, int n)
{
    for (int i = 0; i < n; i++) {
        double *p = pos + 3 * i;
        double s0 = hi[0] * p[0] + hi[1] * p[1] + hi[2] * p[2];
        double s1 = hi[3] * p[0] + hi[4] * p[1] + hi[5] * p[2];
        double s2 = hi[6] * p[0] + hi[7] * p[1] + hi[8] * p[2];
        s0 -= floor(s0);
        s1 -= floor(s1);
        s2 -= floor(s2);
        p[0] = h[0] * s0 + h[1] * s1 + h[2] * s2;
        p[1] = h[3] * s0 + h[4] * s1 + h[5] * s2;
        p[2] = h[6] * s0 + h[7] * s1 + h[8] * s2;
    }
}

static double pair_r2(const double *pos, int i, int j, const double *h, const double *hi)
{
    double dx = pos[3 * j] - pos[3 * i];
    double dy = pos[3 * j + 1] - pos[3 * i + 1];
    double dz = pos[3 * j + 2] - pos[3 * i + 2];
    fmo_mimg(&dx, &dy, &dz, hi, h);
    return dx * dx + dy * dy + dz * dz;
}

/* ------------------------------------------------------------------ a1-a3 */

/* LJ:257-268 (and CORE:280-301): symmetric molecule list, pair (i<j) tested
 * once with d = r_j - r_i, appended to both rows while a row has room.  Rows
 * come out ascending because j<i partners arrive from earlier outer
 * iterations. */
int fmo_nlist_sym(const double *pos, const double *h, const double *hi, int n,
                  double rmcut, int max_neigh, int *cnt, int *list)
{
    double rc2 = (rmcut + 3.0) * (rmcut + 3.0);
    int dropped = 0;
    for (int i = 0; i < n; i++) cnt[i] = 0;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            if (pair_r2(pos, i, j, h, hi) < rc2) {
                if (cnt[i] < max_neigh) list[i * max_neigh + cnt[i]++] = j; else dropped++;
                if (cnt[j] < max_neigh) list[j * max_neigh + cnt[j]++] = i; else dropped++;
            }
        }
    return dropped;
}

/* AI:263-272, MM:337-346: intermolecular half list, j>i ascending, first
 * max_neigh kept, the rest dropped silently in the reference.  Row i depends
 * only on atom i and the atoms after it, so rows [i0, i1) can be built on
 * their own (the large-system tests split the rows over host threads). */
int fmo_nlist_half_rows(const double *pos, const double *h, const double *hi, int na,
                        const int *mol_id, double rc_list, int max_neigh, int i0, int i1,
                        int *cnt, int *list)
{
    double rc2 = rc_list * rc_list;
    int dropped = 0;
    if (i1 > na - 1) i1 = na - 1;
    for (int i = i0; i < i1; i++) {
        int mi = mol_id[i];
        cnt[i] = 0;
        for (int j = i + 1; j < na; j++) {
            if (mol_id[j] == mi) continue;
            if (pair_r2(pos, i, j, h, hi) < rc2) {
                if (cnt[i] < max_neigh) list[(size_t)i * max_neigh + cnt[i]++] = j; else dropped++;
            }
        }
    }
    return dropped;
}

int fmo_nlist_half(const double *pos, const double *h, const double *hi, int na,
                   const int *mol_id, double rc_list, int max_neigh, int *cnt, int *list)
{
    for (int i = 0; i < na; i++) cnt[i] = 0;
    return fmo_nlist_half_rows(pos, h, hi, na, mol_id, rc_list, max_neigh, 0, na - 1, cnt, list);
}

/* AI:251-261: intramolecular symmetric list for the bond-order term. */
int fmo_nlist_intra(const double *pos, const double *h, const double *hi, int na,
                    const int *mol_id, double rc, int max_neigh, int *cnt, int *list)
{
    double rc2 = rc * rc;
    int dropped = 0;
    for (int i = 0; i < na; i++) cnt[i] = 0;
    for (int i = 0; i < na - 1; i++) {
        int mi = mol_id[i];
        for (int j = i + 1; j < na; j++) {
            if (mol_id[j] != mi) continue;
            if (pair_r2(pos, i, j, h, hi) < rc2) {
                if (cnt[i] < max_neigh) list[i * max_neigh + cnt[i]++] = j; else dropped++;
                if (cnt[j] < max_neigh) list[j * max_neigh + cnt[j]++] = i; else dropped++;
            }
        }
    }
    return dropped;
}

/* ------------------------------------------------------------------ a5-a6 */

/* LJ:155-159: rotation matrix of a unit quaternion (w,x,y,z). */
static void quat_to_rot(const double *q, double *R)
{
    double w = q[0], x = q[1], y = q[2], z = q[3];
    R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z);     R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);     R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);     R[7] = 2 * (y * z + w * x);     R[8] = 1 - 2 * (x * x + y * y);
}

/* LJ:276-291: lab-frame site offsets R(q_i) * body_a. */
void fmo_lab_frame(const double *qv, const double *body, int n, int natom, double *lab)
{
    for (int i = 0; i < n; i++) {
        double R[9];
        quat_to_rot(qv + 4 * i, R);
        for (int a = 0; a < natom; a++) {
            const double *b = body + 3 * a;
            double *o = lab + ((size_t)i * natom + a) * 3;
            o[0] = R[0] * b[0] + R[1] * b[1] + R[2] * b[2];
            o[1] = R[3] * b[0] + R[4] * b[1] + R[5] * b[2];
            o[2] = R[6] * b[0] + R[7] * b[1] + R[8] * b[2];
        }
    }
}

/* Site-site LJ constants of the rigid model (LJ:103-107). */
#define RIG_SIGMA 3.431
#define RIG_EPS 2.635e-3

/* LJ:271-400: per molecule i, every listed j whose COM image lies within
 * rmcut2, all site pairs with r^2 < RCUT^2; r^2 clamped at 0.25; energy and
 * virial halved because the list is symmetric. */
double fmo_rigid_forces(double *F, double *T, double *W9,
                        const double *pos, const double *qv, const double *body,
                        const double *h, const double *hi,
                        const int *cnt, const int *list, int max_neigh,
                        int n, int natom, double rmcut2, double *lab)
{
    const double rcut = 3.0 * RIG_SIGMA, rcut2 = rcut * rcut, sig2 = RIG_SIGMA * RIG_SIGMA;
    const double sr = 1.0 / 3.0, sr2v = sr * sr, sr6v = sr2v * sr2v * sr2v;
    const double vshift = 4.0 * RIG_EPS * (sr6v * sr6v - sr6v);
    int own = (lab == NULL);
    if (own) lab = (double *)malloc(sizeof(double) * (size_t)n * natom * 3);
    fmo_lab_frame(qv, body, n, natom, lab);
    for (int k = 0; k < 9; k++) W9[k] = 0;
    double Ep = 0;
    for (int i = 0; i < n; i++) {
        double f[3] = {0, 0, 0}, t[3] = {0, 0, 0}, w[9] = {0}, e = 0;
        for (int k = 0; k < cnt[i]; k++) {
            int j = list[i * max_neigh + k];
            double mx = pos[3 * j] - pos[3 * i], my = pos[3 * j + 1] - pos[3 * i + 1],
                   mz = pos[3 * j + 2] - pos[3 * i + 2];
            fmo_mimg(&mx, &my, &mz, hi, h);
            if (mx * mx + my * my + mz * mz > rmcut2) continue;
            for (int a = 0; a < natom; a++) {
                const double *ra = lab + ((size_t)i * natom + a) * 3;
                for (int b = 0; b < natom; b++) {
                    const double *rb = lab + ((size_t)j * natom + b) * 3;
                    double ddx = mx + rb[0] - ra[0], ddy = my + rb[1] - ra[1], ddz = mz + rb[2] - ra[2];
                    double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    if (!(r2 < rcut2)) continue;
                    if (r2 < 0.25) r2 = 0.25;
                    double ri2 = 1.0 / r2, s2 = sig2 * ri2, s6 = s2 * s2 * s2, s12 = s6 * s6;
                    double fm = 24.0 * RIG_EPS * (2.0 * s12 - s6) * ri2;
                    double fx = fm * ddx, fy = fm * ddy, fz = fm * ddz;
                    f[0] -= fx; f[1] -= fy; f[2] -= fz;
                    t[0] -= (ra[1] * fz - ra[2] * fy);
                    t[1] -= (ra[2] * fx - ra[0] * fz);
                    t[2] -= (ra[0] * fy - ra[1] * fx);
                    e += 0.5 * (4.0 * RIG_EPS * (s12 - s6) - vshift);
                    w[0] += 0.5 * ddx * fx; w[1] += 0.5 * ddx * fy; w[2] += 0.5 * ddx * fz;
                    w[3] += 0.5 * ddy * fx; w[4] += 0.5 * ddy * fy; w[5] += 0.5 * ddy * fz;
                    w[6] += 0.5 * ddz * fx; w[7] += 0.5 * ddz * fy; w[8] += 0.5 * ddz * fz;
                }
            }
        }
        for (int c = 0; c < 3; c++) { F[3 * i + c] = f[c]; T[3 * i + c] = t[c]; }
        for (int c = 0; c < 9; c++) W9[c] += w[c];
        Ep += e;
    }
    if (own) free(lab);
    return Ep;
}

/* ------------------------------------------------------------------ a7-a9 */

/* REBO C-C parameters (AI:110-116). */
#define Q_CC 0.3134602960833
#define A_CC 10953.544162170
#define ALPHA_CC 4.7465390606595
#define B1_CC 12388.79197798
#define BETA1_CC 4.7204523127
#define B2_CC 17.56740646509
#define BETA2_CC 1.4332132499
#define B3_CC 30.71493208065
#define BETA3_CC 1.3826912506
#define DMIN_CC 1.7
#define DMAX_CC 2.0
#define BO_DELTA 0.5
#define G_A0 0.00020813
#define G_C0 330.0
#define G_D0 3.5

/* Cutoff switch and radial/angular pieces (AI:164-191). */
static double sw_fc(double r)
{
    if (r <= DMIN_CC) return 1.0;
    if (r >= DMAX_CC) return 0.0;
    return 0.5 * (1.0 + cos(PI_D * (r - DMIN_CC) / (DMAX_CC - DMIN_CC)));
}
static double sw_dfc(double r)
{
    if (r <= DMIN_CC || r >= DMAX_CC) return 0.0;
    return -0.5 * PI_D / (DMAX_CC - DMIN_CC) * sin(PI_D * (r - DMIN_CC) / (DMAX_CC - DMIN_CC));
}
static double rep_v(double r) { return (1.0 + Q_CC / r) * A_CC * exp(-ALPHA_CC * r); }
static double rep_dv(double r)
{
    double ex = A_CC * exp(-ALPHA_CC * r);
    return (-Q_CC / (r * r)) * ex + (1.0 + Q_CC / r) * (-ALPHA_CC) * ex;
}
static double att_v(double r)
{
    return B1_CC * exp(-BETA1_CC * r) + B2_CC * exp(-BETA2_CC * r) + B3_CC * exp(-BETA3_CC * r);
}
static double att_dv(double r)
{
    return -BETA1_CC * B1_CC * exp(-BETA1_CC * r) - BETA2_CC * B2_CC * exp(-BETA2_CC * r)
           - BETA3_CC * B3_CC * exp(-BETA3_CC * r);
}
static double ang_g(double x)
{
    double c2 = G_C0 * G_C0, d2 = G_D0 * G_D0, hh = 1.0 + x;
    return G_A0 * (1.0 + c2 / d2 - c2 / (d2 + hh * hh));
}
static double ang_dg(double x)
{
    double c2 = G_C0 * G_C0, d2 = G_D0 * G_D0, hh = 1.0 + x, dn = d2 + hh * hh;
    return G_A0 * 2.0 * c2 * hh / (dn * dn);
}

static double clamp1(double c)
{
    if (c < -1.0) c = -1.0;
    if (c > 1.0) c = 1.0;
    return c;
}

/* The C-C pair pieces above for other files of the oracle (rebo2_oracle.c). */
void fmo_rebo_pair_fns(double r, double *fc, double *dfc, double *vr, double *dvr, double *va, double *dva)
{
    *fc = sw_fc(r); *dfc = sw_dfc(r);
    *vr = rep_v(r); *dvr = rep_dv(r);
    *va = att_v(r); *dva = att_dv(r);
}
double fmo_rebo_ang_g(double c) { return ang_g(c); }

/* Bond-order sum of the centre atom c around its bond to `skip`, whose bond
 * vector from c is (bx,by,bz) with length rb (AI:301-309, 313-322). */
static double bo_sum(const double *pos, const double *h, const double *hi, const int *cnt,
                     const int *list, int max_neigh, int c, int skip,
                     double bx, double by, double bz, double rb)
{
    double gs = 0;
    for (int kn = 0; kn < cnt[c]; kn++) {
        int k = list[c * max_neigh + kn];
        if (k == skip) continue;
        double kx = pos[3 * k] - pos[3 * c], ky = pos[3 * k + 1] - pos[3 * c + 1],
               kz = pos[3 * k + 2] - pos[3 * c + 2];
        fmo_mimg(&kx, &ky, &kz, hi, h);
        double rk = sqrt(kx * kx + ky * ky + kz * kz);
        if (rk > DMAX_CC) continue;
        double fk = sw_fc(rk);
        if (fk < 1e-15) continue;
        double ct = clamp1((bx * kx + by * ky + bz * kz) / (rb * rk));
        gs += fk * ang_g(ct);
    }
    return gs;
}

/* The reference's three-body force on the neighbours k of centre c
 * (AI:361-386 with c=i, AI:389-419 with c=j).  (ux,uy,uz) is the unit bond
 * vector pointing away from c along the bond; force on k is added, the same
 * amount subtracted from c. */
static void bo_three_body(double *F, const double *pos, const double *h, const double *hi,
                          const int *cnt, const int *list, int max_neigh, int c, int skip,
                          double bx, double by, double bz, double rb,
                          double ux, double uy, double uz, double gs, double fcut, double va)
{
    if (!(fabs(gs) > 1e-20 && va > 1e-20)) return;
    double dbp = -BO_DELTA * pow(1.0 + gs, -BO_DELTA - 1.0);
    double vh = 0.5 * fcut * va;
    for (int kn = 0; kn < cnt[c]; kn++) {
        int k = list[c * max_neigh + kn];
        if (k == skip) continue;
        double kx = pos[3 * k] - pos[3 * c], ky = pos[3 * k + 1] - pos[3 * c + 1],
               kz = pos[3 * k + 2] - pos[3 * c + 2];
        fmo_mimg(&kx, &ky, &kz, hi, h);
        double rk = sqrt(kx * kx + ky * ky + kz * kz);
        if (rk > DMAX_CC) continue;
        double fck = sw_fc(rk);
        if (fck < 1e-15) continue;
        double dfck = sw_dfc(rk);
        double rki = 1.0 / rk;
        double rkv[3] = {kx * rki, ky * rki, kz * rki};
        double uv[3] = {ux, uy, uz};
        double ct = clamp1((bx * kx + by * ky + bz * kz) / (rb * rk));
        double gv = ang_g(ct), dgv = ang_dg(ct), coeff = -vh * dbp;
        for (int a = 0; a < 3; a++) {
            double f1 = coeff * dfck * gv * rkv[a];
            double dc = (uv[a] - ct * rkv[a]) * rki;
            double fk = f1 + coeff * fck * dgv * dc;
            F[3 * k + a] += fk;
            F[3 * c + a] -= fk;
        }
    }
}

/* AI:275-421: bonds i<j with r<=Dmax; V = fc [V_R - bbar V_A]. */
double fmo_rebo(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                const int *cnt, const int *list, int max_neigh, int na)
{
    double Ep = 0;
    for (int i = 0; i < na; i++) {
        for (int jn = 0; jn < cnt[i]; jn++) {
            int j = list[i * max_neigh + jn];
            if (j <= i) continue;
            double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
                   dz = pos[3 * j + 2] - pos[3 * i + 2];
            fmo_mimg(&dx, &dy, &dz, hi, h);
            double rij = sqrt(dx * dx + dy * dy + dz * dz);
            if (rij > DMAX_CC) continue;
            double fcut = sw_fc(rij), dfcut = sw_dfc(rij);
            if (fcut < 1e-15 && dfcut == 0) continue;
            double vr = rep_v(rij), dvr = rep_dv(rij), va = att_v(rij), dva = att_dv(rij);
            double rinv = 1.0 / rij;
            double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            double gij = bo_sum(pos, h, hi, cnt, list, max_neigh, i, j, dx, dy, dz, rij);
            double bij = pow(1.0 + gij, -BO_DELTA);
            double gji = bo_sum(pos, h, hi, cnt, list, max_neigh, j, i, -dx, -dy, -dz, rij);
            double bji = pow(1.0 + gji, -BO_DELTA);
            double bbar = 0.5 * (bij + bji);
            Ep += fcut * (vr - bbar * va);
            double fpair = (dfcut * (vr - bbar * va) + fcut * (dvr - bbar * dva)) * rinv;
            F[3 * i] += fpair * dx; F[3 * i + 1] += fpair * dy; F[3 * i + 2] += fpair * dz;
            F[3 * j] -= fpair * dx; F[3 * j + 1] -= fpair * dy; F[3 * j + 2] -= fpair * dz;
            double d[3] = {dx, dy, dz};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) vir9[a * 3 + b] -= d[a] * fpair * d[b];
            bo_three_body(F, pos, h, hi, cnt, list, max_neigh, i, j, dx, dy, dz, rij,
                          ux, uy, uz, gij, fcut, va);
            bo_three_body(F, pos, h, hi, cnt, list, max_neigh, j, i, -dx, -dy, -dz, rij,
                          -ux, -uy, -uz, gji, fcut, va);
        }
    }
    return Ep;
}

/* NOT a restatement of the reference: the gradient of fmo_rebo's energy (the
 * forces of the FMD_PHYS_REBO option).  The reference's three-body force on a
 * neighbour k of centre c is +coeff dG/dr_k; the gradient's is -coeff dG/dr_k,
 * and the bond partner b gets -coeff dG/dr_b = -coeff sum_k fc_k g'(cos)
 * (u_k - cos u_b) / r_b.  Checked by finite differences of fmo_rebo's energy
 * (tests/test_force_gradients.py), not against the reference. */
static void bo_three_body_grad(double *F, const double *pos, const double *h, const double *hi,
                               const int *cnt, const int *list, int max_neigh, int c, int b,
                               double bx, double by, double bz, double rb,
                               double ux, double uy, double uz, double gs, double fcut, double va)
{
    if (!(fabs(gs) > 1e-20 && va > 1e-20)) return;
    double coeff = 0.5 * fcut * va * BO_DELTA * pow(1.0 + gs, -BO_DELTA - 1.0);   /* dE/dG */
    double fb[3] = {0.0, 0.0, 0.0};
    for (int kn = 0; kn < cnt[c]; kn++) {
        int k = list[c * max_neigh + kn];
        if (k == b) continue;
        double kx = pos[3 * k] - pos[3 * c], ky = pos[3 * k + 1] - pos[3 * c + 1],
               kz = pos[3 * k + 2] - pos[3 * c + 2];
        fmo_mimg(&kx, &ky, &kz, hi, h);
        double rk = sqrt(kx * kx + ky * ky + kz * kz);
        if (rk > DMAX_CC) continue;
        double fck = sw_fc(rk);
        if (fck < 1e-15) continue;
        double dfck = sw_dfc(rk), rki = 1.0 / rk;
        double rkv[3] = {kx * rki, ky * rki, kz * rki}, uv[3] = {ux, uy, uz};
        double ct = clamp1((bx * kx + by * ky + bz * kz) / (rb * rk));
        double gv = ang_g(ct), dgv = ang_dg(ct);
        for (int a = 0; a < 3; a++) {
            double fk = -coeff * (dfck * gv * rkv[a] + fck * dgv * (uv[a] - ct * rkv[a]) * rki);
            F[3 * k + a] += fk;
            F[3 * c + a] -= fk;
            fb[a] += -coeff * fck * dgv * (rkv[a] - ct * uv[a]) / rb;
        }
    }
    for (int a = 0; a < 3; a++) {
        F[3 * b + a] += fb[a];
        F[3 * c + a] -= fb[a];
    }
}

double fmo_rebo_grad(double *F, const double *pos, const double *h, const double *hi,
                     const int *cnt, const int *list, int max_neigh, int na)
{
    double Ep = 0;
    for (int i = 0; i < na; i++) {
        for (int jn = 0; jn < cnt[i]; jn++) {
            int j = list[i * max_neigh + jn];
            if (j <= i) continue;
            double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
                   dz = pos[3 * j + 2] - pos[3 * i + 2];
            fmo_mimg(&dx, &dy, &dz, hi, h);
            double rij = sqrt(dx * dx + dy * dy + dz * dz);
            if (rij > DMAX_CC) continue;
            double fcut = sw_fc(rij), dfcut = sw_dfc(rij);
            if (fcut < 1e-15 && dfcut == 0) continue;
            double vr = rep_v(rij), dvr = rep_dv(rij), va = att_v(rij), dva = att_dv(rij);
            double rinv = 1.0 / rij;
            double gij = bo_sum(pos, h, hi, cnt, list, max_neigh, i, j, dx, dy, dz, rij);
            double gji = bo_sum(pos, h, hi, cnt, list, max_neigh, j, i, -dx, -dy, -dz, rij);
            double bbar = 0.5 * (pow(1.0 + gij, -BO_DELTA) + pow(1.0 + gji, -BO_DELTA));
            Ep += fcut * (vr - bbar * va);
            double fpair = (dfcut * (vr - bbar * va) + fcut * (dvr - bbar * dva)) * rinv;
            F[3 * i] += fpair * dx; F[3 * i + 1] += fpair * dy; F[3 * i + 2] += fpair * dz;
            F[3 * j] -= fpair * dx; F[3 * j + 1] -= fpair * dy; F[3 * j + 2] -= fpair * dz;
            bo_three_body_grad(F, pos, h, hi, cnt, list, max_neigh, i, j, dx, dy, dz, rij,
                               dx * rinv, dy * rinv, dz * rinv, gij, fcut, va);
            bo_three_body_grad(F, pos, h, hi, cnt, list, max_neigh, j, i, -dx, -dy, -dz, rij,
                               -dx * rinv, -dy * rinv, -dz * rinv, gji, fcut, va);
        }
    }
    return Ep;
}

/* AI:119-124: sigma 3.40, eps 2.84 meV, rc = 3 sigma, V shifted by V(rc). */
fmo_lj_params fmo_lj_params_airebo(void)
{
    fmo_lj_params p;
    double sig = 3.40, rc = 3.0 * sig, sr = sig / rc, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2;
    p.sig2 = sig * sig; p.eps = 2.84e-3; p.rc2 = rc * rc;
    p.vshift = 4 * p.eps * (sr6 * sr6 - sr6);
    p.full_virial = 1;
    return p;
}

/* MM:113-116: sigma 3.431, eps 2.635 meV, rc = 3 sigma, sigma/rc = 1/3. */
fmo_lj_params fmo_lj_params_mm(void)
{
    fmo_lj_params p;
    double sig = 3.431, rc = 3.0 * sig, sr = 1.0 / 3.0, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2;
    p.sig2 = sig * sig; p.eps = 2.635e-3; p.rc2 = rc * rc;
    p.vshift = 4.0 * p.eps * (sr6 * sr6 - sr6);
    p.full_virial = 0;
    return p;
}

/* AI:424-473 and MM:711-764: half-list shifted LJ with r^2 clamp 0.25. */
double fmo_lj_half(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                   const int *cnt, const int *list, int max_neigh, int na, const fmo_lj_params *p)
{
    double Ep = 0;
    for (int i = 0; i < na; i++) {
        for (int jn = 0; jn < cnt[i]; jn++) {
            int j = list[i * max_neigh + jn];
            double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
                   dz = pos[3 * j + 2] - pos[3 * i + 2];
            fmo_mimg(&dx, &dy, &dz, hi, h);
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > p->rc2) continue;
            if (r2 < 0.25) r2 = 0.25;
            double ri2 = 1.0 / r2, s2 = p->sig2 * ri2, s6 = s2 * s2 * s2, s12 = s6 * s6;
            double fm = 24 * p->eps * (2 * s12 - s6) * ri2;
            Ep += 4 * p->eps * (s12 - s6) - p->vshift;
            F[3 * i] -= fm * dx; F[3 * i + 1] -= fm * dy; F[3 * i + 2] -= fm * dz;
            F[3 * j] += fm * dx; F[3 * j + 1] += fm * dy; F[3 * j + 2] += fm * dz;
            if (p->full_virial) {
                double d[3] = {dx, dy, dz};
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) vir9[a * 3 + b] += d[a] * fm * d[b];
            } else {
                vir9[0] += dx * fm * dx;
                vir9[4] += dy * fm * dy;
                vir9[8] += dz * fm * dz;
            }
        }
    }
    return Ep;
}

/* AI:477-495. */
void fmo_airebo_forces(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                       const int *cnt_r, const int *list_r, const int *cnt_l, const int *list_l,
                       int na, double *E)
{
    fmo_lj_params p = fmo_lj_params_airebo();
    memset(F, 0, sizeof(double) * 3 * (size_t)na);
    memset(vir9, 0, sizeof(double) * 9);
    double er = fmo_rebo(F, vir9, pos, h, hi, cnt_r, list_r, 12, na);
    double el = fmo_lj_half(F, vir9, pos, h, hi, cnt_l, list_l, 400, na, &p);
    E[0] = er + el; E[1] = er; E[2] = el;
}

/* ------------------------------------------------------------------ a10-a16 */

static void mm_add(double *F, int i, double x, double y, double z)
{
    F[3 * i] += x; F[3 * i + 1] += y; F[3 * i + 2] += z;
}

/* Torsion force pattern shared by dihedrals and impropers (MM:503-529,
 * MM:613-672).  Atoms a1..a4 receive f1..f4; returns the energy. */
static double torsion(double *F, const double *pos, const double *h, const double *hi,
                      int a1, int a2, int a3, int a4, int mult, double vn, double gamma)
{
    double b1x = pos[3 * a2] - pos[3 * a1], b1y = pos[3 * a2 + 1] - pos[3 * a1 + 1],
           b1z = pos[3 * a2 + 2] - pos[3 * a1 + 2];
    double b2x = pos[3 * a3] - pos[3 * a2], b2y = pos[3 * a3 + 1] - pos[3 * a2 + 1],
           b2z = pos[3 * a3 + 2] - pos[3 * a2 + 2];
    double b3x = pos[3 * a4] - pos[3 * a3], b3y = pos[3 * a4 + 1] - pos[3 * a3 + 1],
           b3z = pos[3 * a4 + 2] - pos[3 * a3 + 2];
    fmo_mimg(&b1x, &b1y, &b1z, hi, h);
    fmo_mimg(&b2x, &b2y, &b2z, hi, h);
    fmo_mimg(&b3x, &b3y, &b3z, hi, h);
    double mx = b1y * b2z - b1z * b2y, my = b1z * b2x - b1x * b2z, mz = b1x * b2y - b1y * b2x;
    double nx = b2y * b3z - b2z * b3y, ny = b2z * b3x - b2x * b3z, nz = b2x * b3y - b2y * b3x;
    double mm = mx * mx + my * my + mz * mz, nn = nx * nx + ny * ny + nz * nz;
    if (mm < 1e-20 || nn < 1e-20) return 0.0;
    double imm = 1.0 / mm, inn = 1.0 / nn;
    double b2len = sqrt(b2x * b2x + b2y * b2y + b2z * b2z);
    double cosphi = clamp1((mx * nx + my * ny + mz * nz) / sqrt(mm * nn));
    double b1b2 = b1x * b2x + b1y * b2y + b1z * b2z;
    double b2b3 = b2x * b3x + b2y * b3y + b2z * b3z;
    double sinphi = (mx * b3x + my * b3y + mz * b3z) * b2len / sqrt(mm * nn);
    double phi = atan2(sinphi, cosphi);
    double e = 0.5 * vn * (1.0 + cos(mult * phi - gamma));
    double dphi = -0.5 * vn * mult * sin(mult * phi - gamma);
    double f1x = dphi * b2len * imm * mx, f1y = dphi * b2len * imm * my, f1z = dphi * b2len * imm * mz;
    double f4x = -dphi * b2len * inn * nx, f4y = -dphi * b2len * inn * ny, f4z = -dphi * b2len * inn * nz;
    double ci = b1b2 / (b2len * b2len), ck = b2b3 / (b2len * b2len);
    mm_add(F, a1, f1x, f1y, f1z);
    mm_add(F, a2, -f1x + ci * f1x - ck * f4x, -f1y + ci * f1y - ck * f4y, -f1z + ci * f1z - ck * f4z);
    mm_add(F, a3, -f4x - ci * f1x + ck * f4x, -f4y - ci * f1y + ck * f4y, -f4z - ci * f1z + ck * f4z);
    mm_add(F, a4, f4x, f4y, f4z);
    return e;
}

/* MM:351-788.  Forces follow the reference's sign conventions exactly,
 * including the bond/angle terms that equal +grad E. */
void fmo_mm_forces(double *F, double *vir9, const double *pos, const double *h, const double *hi,
                   const fmo_mm_topo *t, const int *cnt, const int *list,
                   const double *charge, const int *mol_id, int has_charge, int na, double *E)
{
    memset(F, 0, sizeof(double) * 3 * (size_t)na);
    memset(vir9, 0, sizeof(double) * 9);
    double eb = 0, ea = 0, ed = 0, ei = 0, elj = 0, ec = 0;
    for (int b = 0; b < t->nb; b++) {                      /* MM:384-447 */
        int i = t->b_i0[b], j = t->b_i1[b];
        double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
               dz = pos[3 * j + 2] - pos[3 * i + 2];
        fmo_mimg(&dx, &dy, &dz, hi, h);
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (r < 1e-10) continue;
        double dr = r - t->b_r0[b];
        eb += 0.5 * t->b_kb[b] * dr * dr;
        double fm = -t->b_kb[b] * dr / r;
        double fx = fm * dx, fy = fm * dy, fz = fm * dz;
        mm_add(F, i, fx, fy, fz);
        mm_add(F, j, -fx, -fy, -fz);
        vir9[0] += dx * fx; vir9[4] += dy * fy; vir9[8] += dz * fz;
    }
    for (int a = 0; a < t->nang; a++) {                    /* MM:455-492 */
        int i = t->a_i0[a], j = t->a_i1[a], k = t->a_i2[a];
        double u0 = pos[3 * i] - pos[3 * j], u1 = pos[3 * i + 1] - pos[3 * j + 1],
               u2 = pos[3 * i + 2] - pos[3 * j + 2];
        double v0 = pos[3 * k] - pos[3 * j], v1 = pos[3 * k + 1] - pos[3 * j + 1],
               v2 = pos[3 * k + 2] - pos[3 * j + 2];
        fmo_mimg(&u0, &u1, &u2, hi, h);
        fmo_mimg(&v0, &v1, &v2, hi, h);
        double du = sqrt(u0 * u0 + u1 * u1 + u2 * u2), dv = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        if (du < 1e-10 || dv < 1e-10) continue;
        double c = (u0 * v0 + u1 * v1 + u2 * v2) / (du * dv);
        if (c > 0.999999) c = 0.999999;
        if (c < -0.999999) c = -0.999999;
        double th = acos(c), dth = th - t->a_th0[a];
        ea += 0.5 * t->a_kth[a] * dth * dth;
        double s = sqrt(1.0 - c * c + 1e-30);
        double dV = -t->a_kth[a] * dth / s;
        double uu[3] = {u0, u1, u2}, vv[3] = {v0, v1, v2};
        for (int q = 0; q < 3; q++) {
            double fi = dV * (vv[q] / (du * dv) - c * uu[q] / (du * du));
            double fk = dV * (uu[q] / (du * dv) - c * vv[q] / (dv * dv));
            F[3 * i + q] += fi;
            F[3 * k + q] += fk;
            F[3 * j + q] -= fi + fk;
        }
    }
    for (int d = 0; d < t->ndih; d++)                      /* MM:500-602 */
        ed += torsion(F, pos, h, hi, t->d_i0[d], t->d_i1[d], t->d_i2[d], t->d_i3[d],
                      t->d_mult[d], t->d_vn[d], t->d_gamma[d]);
    for (int q = 0; q < t->nimp; q++)                      /* MM:610-709: order c1,c0,c2,c3 */
        ei += torsion(F, pos, h, hi, t->m_i1[q], t->m_i0[q], t->m_i2[q], t->m_i3[q],
                      2, t->m_ki[q], t->m_gamma[q]);
    fmo_lj_params p = fmo_lj_params_mm();
    elj = fmo_lj_half(F, vir9, pos, h, hi, cnt, list, 400, na, &p);
    if (has_charge) {                                      /* MM:766-786 */
        const double kc = 14.3996, rc = 3.0 * 3.431, rc2 = rc * rc;
        for (int i = 0; i < na - 1; i++)
            for (int j = i + 1; j < na; j++) {
                if (mol_id[i] == mol_id[j]) continue;
                double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
                       dz = pos[3 * j + 2] - pos[3 * i + 2];
                fmo_mimg(&dx, &dy, &dz, hi, h);
                double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > rc2) continue;
                double r = sqrt(r2), qi = charge[i], qj = charge[j];
                ec += kc * qi * qj / r - kc * qi * qj / rc;
                double fm = kc * qi * qj / (r2 * r);
                mm_add(F, i, -fm * dx, -fm * dy, -fm * dz);
                mm_add(F, j, fm * dx, fm * dy, fm * dz);
            }
    }
    E[0] = eb; E[1] = ea; E[2] = ed; E[3] = ei; E[4] = elj; E[5] = ec;
    E[6] = eb + ea + ed + ei + elj + ec;
}

/* MM:240-252: signed dihedral angle i-j-k-l of a reference geometry. */
double fmo_dihedral_angle(const double *c, int i, int j, int k, int l)
{
    double b1x = c[3 * j] - c[3 * i], b1y = c[3 * j + 1] - c[3 * i + 1], b1z = c[3 * j + 2] - c[3 * i + 2];
    double b2x = c[3 * k] - c[3 * j], b2y = c[3 * k + 1] - c[3 * j + 1], b2z = c[3 * k + 2] - c[3 * j + 2];
    double b3x = c[3 * l] - c[3 * k], b3y = c[3 * l + 1] - c[3 * k + 1], b3z = c[3 * l + 2] - c[3 * k + 2];
    double mx = b1y * b2z - b1z * b2y, my = b1z * b2x - b1x * b2z, mz = b1x * b2y - b1y * b2x;
    double nx = b2y * b3z - b2z * b3y, ny = b2z * b3x - b2x * b3z, nz = b2x * b3y - b2y * b3x;
    double mm = mx * mx + my * my + mz * mz, nn = nx * nx + ny * ny + nz * nz;
    if (mm < 1e-20 || nn < 1e-20) return 0;
    double b2len = sqrt(b2x * b2x + b2y * b2y + b2z * b2z);
    double cp = clamp1((mx * nx + my * ny + mz * nz) / sqrt(mm * nn));
    double sp = (mx * b3x + my * b3y + mz * b3z) * b2len / sqrt(mm * nn);
    return atan2(sp, cp);
}

/* MM:254-334 for one molecule.  `bonds` is the sorted unique (lo,hi) list
 * that load_cc1 builds from the adjacency columns (MM:180-182); the
 * adjacency used for angles/dihedrals/impropers is rebuilt from it in bond
 * order (MM:256-257). */
void fmo_mm_topology_mol(const double *coords, int natom, const int *bonds, int nbond,
                         int *counts, int *b_idx, double *b_r0, int *a_idx, double *a_th0,
                         int *d_idx, double *d_gamma, int *m_idx, double *m_gamma)
{
    int *deg = (int *)calloc((size_t)natom, sizeof(int));
    int *adj = (int *)malloc(sizeof(int) * (size_t)natom * 2 * (nbond > 0 ? nbond : 1));
    int stride = 2 * (nbond > 0 ? nbond : 1);
    for (int b = 0; b < nbond; b++) {
        int bi = bonds[2 * b], bj = bonds[2 * b + 1];
        adj[bi * stride + deg[bi]++] = bj;
        adj[bj * stride + deg[bj]++] = bi;
    }
    int nb = 0, nang = 0, ndih = 0, nimp = 0;
    for (int b = 0; b < nbond; b++) {
        int bi = bonds[2 * b], bj = bonds[2 * b + 1];
        double dx = coords[3 * bi] - coords[3 * bj], dy = coords[3 * bi + 1] - coords[3 * bj + 1],
               dz = coords[3 * bi + 2] - coords[3 * bj + 2];
        b_idx[2 * nb] = bi; b_idx[2 * nb + 1] = bj;
        b_r0[nb++] = sqrt(dx * dx + dy * dy + dz * dz);
    }
    for (int j = 0; j < natom; j++)
        for (int ii = 0; ii < deg[j]; ii++)
            for (int kk = ii + 1; kk < deg[j]; kk++) {
                int i = adj[j * stride + ii], k = adj[j * stride + kk];
                double u[3], v[3];
                for (int a = 0; a < 3; a++) {
                    u[a] = coords[3 * i + a] - coords[3 * j + a];
                    v[a] = coords[3 * k + a] - coords[3 * j + a];
                }
                double du = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                double dv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                double c = clamp1((u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) / (du * dv));
                a_idx[3 * nang] = i; a_idx[3 * nang + 1] = j; a_idx[3 * nang + 2] = k;
                a_th0[nang++] = acos(c);
            }
    for (int b = 0; b < nbond; b++) {
        int bj = bonds[2 * b], bk = bonds[2 * b + 1];
        for (int ii = 0; ii < deg[bj]; ii++) {
            int i = adj[bj * stride + ii];
            if (i == bk) continue;
            for (int ll = 0; ll < deg[bk]; ll++) {
                int l = adj[bk * stride + ll];
                if (l == bj || l == i) continue;
                double phi0 = fmo_dihedral_angle(coords, i, bj, bk, l);
                d_idx[4 * ndih] = i; d_idx[4 * ndih + 1] = bj;
                d_idx[4 * ndih + 2] = bk; d_idx[4 * ndih + 3] = l;
                d_gamma[ndih++] = 2 * phi0 + PI_D;
            }
        }
    }
    for (int i = 0; i < natom; i++) {
        if (deg[i] != 3) continue;
        int j = adj[i * stride], k = adj[i * stride + 1], l = adj[i * stride + 2];
        double psi0 = fmo_dihedral_angle(coords, j, i, k, l);
        m_idx[4 * nimp] = i; m_idx[4 * nimp + 1] = j; m_idx[4 * nimp + 2] = k; m_idx[4 * nimp + 3] = l;
        m_gamma[nimp++] = 2 * psi0 + PI_D;
    }
    counts[0] = nb; counts[1] = nang; counts[2] = ndih; counts[3] = nimp;
    free(deg);
    free(adj);
}

/* ------------------------------------------------------------------ a17-a18 */

static double dmax2(double a, double b) { return a > b ? a : b; }
static double dclamp(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* LJ:426-431: Nf = 6N-3, Q and W with the reference's 1e4/1e6 factors. */
fmo_npt fmo_make_npt_rigid(double T, double Pe, int n)
{
    fmo_npt s;
    int nf = 6 * n - 3;
    s.xi = 0; s.Q = dmax2(nf * KB * T * 100.0 * 100.0, 1e-20);
    for (int k = 0; k < 9; k++) s.Vg[k] = 0;
    s.W = dmax2((nf + 9) * KB * T * 1000.0 * 1000.0, 1e-20);
    s.Pe = Pe; s.Tt = T; s.Nf = nf;
    return s;
}

/* AI:512-515, MM:805-808: Nf = 3Na-3. */
fmo_npt fmo_make_npt_atom(double T, double Pe, int na)
{
    fmo_npt s;
    int nf = 3 * na - 3;
    s.xi = 0; s.Q = dmax2(nf * KB * T * 100.0 * 100.0, 1e-20);
    for (int k = 0; k < 9; k++) s.Vg[k] = 0;
    s.W = dmax2((nf + 9) * KB * T * 1000.0 * 1000.0, 1e-20);
    s.Pe = Pe; s.Tt = T; s.Nf = nf;
    return s;
}

double fmo_ke_trans(const double *vel, int n, double mmol)
{
    double s = 0;
    for (int i = 0; i < n; i++)
        s += vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2];
    return 0.5 * mmol * s / CONV;
}

double fmo_ke_rot(const double *omg, int n, double i0)
{
    double s = 0;
    for (int i = 0; i < n; i++)
        s += omg[3 * i] * omg[3 * i] + omg[3 * i + 1] * omg[3 * i + 1] + omg[3 * i + 2] * omg[3 * i + 2];
    return 0.5 * i0 * s / CONV;
}

double fmo_ke_atoms(const double *vel, const double *mass, int na)
{
    double s = 0;
    for (int i = 0; i < na; i++)
        s += mass[i] * (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]);
    return 0.5 * s / CONV;
}

double fmo_inst_T(double ke, int nf) { return 2 * ke / (nf * KB); }
double fmo_inst_P(const double *W, double ke, double V)
{
    return (2 * ke + W[0] + W[4] + W[8]) / (3 * V) * EV2GPA;
}

/* Thermostat/barostat half update shared by all programs (LJ:448-455). */
static void npt_half(fmo_npt *s, double hdt, double ke, double ke_p, const double *W, double V,
                     double xi_lim, double vg_lim)
{
    s->xi += hdt * (2 * ke - s->Nf * KB * s->Tt) / s->Q;
    s->xi = dclamp(s->xi, -xi_lim, xi_lim);
    double dP = fmo_inst_P(W, ke_p, V) - s->Pe;
    for (int a = 0; a < 3; a++) s->Vg[a * 4] += hdt * V * dP / (s->W * EV2GPA);
    for (int a = 0; a < 3; a++) s->Vg[a * 4] = dclamp(s->Vg[a * 4], -vg_lim, vg_lim);
}

/* Drift in fractional coordinates with the current inverse cell, wrap,
 * then map back with the updated cell (LJ:476-497). */
static void drift_wrap(double *pos, const double *vel, const double *hi_old, int n, double dt)
{
    for (int i = 0; i < n; i++) {
        double *p = pos + 3 * i;
        const double *v = vel + 3 * i;
        const double *q = hi_old;
        double sx = q[0] * p[0] + q[1] * p[1] + q[2] * p[2];
        double sy = q[3] * p[0] + q[4] * p[1] + q[5] * p[2];
        double sz = q[6] * p[0] + q[7] * p[1] + q[8] * p[2];
        double vx = q[0] * v[0] + q[1] * v[1] + q[2] * v[2];
        double vy = q[3] * v[0] + q[4] * v[1] + q[5] * v[2];
        double vz = q[6] * v[0] + q[7] * v[1] + q[8] * v[2];
        sx += dt * vx; sy += dt * vy; sz += dt * vz;
        sx -= floor(sx); sy -= floor(sy); sz -= floor(sz);
        p[0] = sx; p[1] = sy; p[2] = sz;
    }
}

static void frac_to_cart(double *pos, const double *h, int n)
{
    for (int i = 0; i < n; i++) {
        double *p = pos + 3 * i;
        double sx = p[0], sy = p[1], sz = p[2];
        p[0] = h[0] * sx + h[1] * sy + h[2] * sz;
        p[1] = h[3] * sx + h[4] * sy + h[5] * sz;
        p[2] = h[6] * sx + h[7] * sy + h[8] * sz;
    }
}

/* LJ:161-174: quaternion product and small-rotation increment. */
static void quat_mul(const double *a, const double *b, double *o)
{
    o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
    o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

static void omega_to_dq(double wx, double wy, double wz, double dt, double *dq)
{
    double wm = sqrt(wx * wx + wy * wy + wz * wz), th = wm * dt * 0.5;
    if (th < 1e-14) { dq[0] = 1.0; dq[1] = 0.5 * dt * wx; dq[2] = 0.5 * dt * wy; dq[3] = 0.5 * dt * wz; }
    else { double s = sin(th) / wm; dq[0] = cos(th); dq[1] = s * wx; dq[2] = s * wy; dq[3] = s * wz; }
}

void fmo_rigid_step(double *pos, double *vel, double *qv, double *omg,
                    double *F, double *T, double *W9, double *h, double *hi,
                    const double *body, double i0, double mmol,
                    int n, int natom, double rmcut2, double dt, fmo_npt *npt,
                    const int *cnt, const int *list, int max_neigh, double *lab, double *out)
{
    double hdt = 0.5 * dt;
    fmo_mat_inv9(h, hi);
    double V = fabs(fmo_mat_det9(h));
    double kt = fmo_ke_trans(vel, n, mmol), kr = fmo_ke_rot(omg, n, i0), KE = kt + kr;
    npt_half(npt, hdt, KE, kt, W9, V, 0.1, 0.01);
    double eps = npt->Vg[0] * hi[0] + npt->Vg[4] * hi[4] + npt->Vg[8] * hi[8];
    double sc_nh = exp(-hdt * npt->xi), sc_pr = exp(-hdt * eps / 3.0), sc_v = sc_nh * sc_pr;
    double cF = CONV / mmol, cT = CONV / i0;
    for (int i = 0; i < 3 * n; i++) {
        vel[i] = vel[i] * sc_v + hdt * F[i] * cF;
        omg[i] = omg[i] * sc_nh + hdt * T[i] * cT;
    }
    drift_wrap(pos, vel, hi, n, dt);
    for (int a = 0; a < 9; a++) h[a] += dt * npt->Vg[a];
    frac_to_cart(pos, h, n);
    for (int i = 0; i < n; i++) {
        double dq[4], q[4];
        omega_to_dq(omg[3 * i], omg[3 * i + 1], omg[3 * i + 2], dt, dq);
        quat_mul(qv + 4 * i, dq, q);
        double nrm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]), inv = 1.0 / nrm;
        for (int a = 0; a < 4; a++) qv[4 * i + a] = q[a] * inv;
    }
    fmo_mat_inv9(h, hi);
    double Ep = fmo_rigid_forces(F, T, W9, pos, qv, body, h, hi, cnt, list, max_neigh,
                                 n, natom, rmcut2, lab);
    double eps2 = npt->Vg[0] * hi[0] + npt->Vg[4] * hi[4] + npt->Vg[8] * hi[8];
    double sc_v2 = sc_nh * exp(-hdt * eps2 / 3.0);
    for (int i = 0; i < 3 * n; i++) {
        vel[i] = (vel[i] + hdt * F[i] * cF) * sc_v2;
        omg[i] = (omg[i] + hdt * T[i] * cT) * sc_nh;
    }
    kt = fmo_ke_trans(vel, n, mmol); kr = fmo_ke_rot(omg, n, i0); KE = kt + kr;
    double V2 = fabs(fmo_mat_det9(h));
    npt_half(npt, hdt, KE, kt, W9, V2, 0.1, 0.01);
    out[0] = Ep; out[1] = KE;
}

/* Shared atomistic velocity-Verlet skeleton (AI:518-590, MM:811-890);
 * `force` fills F, vir9 and the energy record. */
/* MM:791-799: constant carbon mass inside the sum. */
static double ke_const_mass(const double *vel, int na, double m)
{
    double s = 0;
    for (int i = 0; i < na; i++)
        s += m * (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]);
    return 0.5 * s / CONV;
}

typedef void (*atom_force_fn)(void *ctx, double *F, double *vir9, const double *pos,
                              const double *h, const double *hi, double *E);

static double atom_step(double *pos, double *vel, double *F, double *vir9, double *h, double *hi,
                        const double *mass, double mconst, int na, double dt, fmo_npt *npt,
                        atom_force_fn force, void *fctx, double *E)
{
    double hdt = 0.5 * dt, V = fabs(fmo_mat_det9(h));
    double KE = mass ? fmo_ke_atoms(vel, mass, na) : ke_const_mass(vel, na, mconst);
    npt_half(npt, hdt, KE, KE, vir9, V, 0.05, 0.005);
    double eps = npt->Vg[0] * hi[0] + npt->Vg[4] * hi[4] + npt->Vg[8] * hi[8];
    double sc_nh = exp(-hdt * npt->xi), sc_pr = exp(-hdt * eps / 3.0), sc_v = sc_nh * sc_pr;
    double mconv = CONV / mconst;
    for (int i = 0; i < na; i++) {
        double mi = mass ? CONV / mass[i] : mconv;
        for (int a = 0; a < 3; a++) vel[3 * i + a] = vel[3 * i + a] * sc_v + hdt * F[3 * i + a] * mi;
    }
    drift_wrap(pos, vel, hi, na, dt);
    for (int a = 0; a < 9; a++) h[a] += dt * npt->Vg[a];
    fmo_mat_inv9(h, hi);
    frac_to_cart(pos, h, na);
    force(fctx, F, vir9, pos, h, hi, E);
    double eps2 = npt->Vg[0] * hi[0] + npt->Vg[4] * hi[4] + npt->Vg[8] * hi[8];
    double sc_v2 = sc_nh * exp(-hdt * eps2 / 3.0);
    for (int i = 0; i < na; i++) {
        double mi = mass ? CONV / mass[i] : mconv;
        for (int a = 0; a < 3; a++) vel[3 * i + a] = (vel[3 * i + a] + hdt * F[3 * i + a] * mi) * sc_v2;
    }
    KE = mass ? fmo_ke_atoms(vel, mass, na) : ke_const_mass(vel, na, mconst);
    double V2 = fabs(fmo_mat_det9(h));
    npt_half(npt, hdt, KE, KE, vir9, V2, 0.05, 0.005);
    return KE;
}

typedef struct { const int *cr, *lr, *cl, *ll; int na; } airebo_ctx;
static void airebo_force_cb(void *c, double *F, double *vir9, const double *pos,
                            const double *h, const double *hi, double *E)
{
    airebo_ctx *a = (airebo_ctx *)c;
    fmo_airebo_forces(F, vir9, pos, h, hi, a->cr, a->lr, a->cl, a->ll, a->na, E);
}

void fmo_airebo_step(double *pos, double *vel, double *F, double *vir9, double *h, double *hi,
                     const double *mass, int na, double dt, fmo_npt *npt,
                     const int *cnt_r, const int *list_r, const int *cnt_l, const int *list_l,
                     double *out)
{
    airebo_ctx c = {cnt_r, list_r, cnt_l, list_l, na};
    double E[3];
    double KE = atom_step(pos, vel, F, vir9, h, hi, mass, 12.011, na, dt, npt, airebo_force_cb, &c, E);
    out[0] = E[0]; out[1] = E[1]; out[2] = E[2]; out[3] = KE;
}

typedef struct { const fmo_mm_topo *t; const int *cnt, *list; const double *charge;
                 const int *mol_id; int has_charge, na; } mm_ctx;
static void mm_force_cb(void *c, double *F, double *vir9, const double *pos,
                        const double *h, const double *hi, double *E)
{
    mm_ctx *m = (mm_ctx *)c;
    fmo_mm_forces(F, vir9, pos, h, hi, m->t, m->cnt, m->list, m->charge, m->mol_id,
                  m->has_charge, m->na, E);
}

void fmo_mm_step(double *pos, double *vel, double *F, double *vir9, double *h, double *hi,
                 int na, double dt, fmo_npt *npt, const fmo_mm_topo *t,
                 const int *cnt, const int *list, const double *charge, const int *mol_id,
                 int has_charge, double *out)
{
    mm_ctx c = {t, cnt, list, charge, mol_id, has_charge, na};
    double E[7];
    double KE = atom_step(pos, vel, F, vir9, h, hi, NULL, 12.011, na, dt, npt, mm_force_cb, &c, E);
    for (int k = 0; k < 7; k++) out[k] = E[k];
    out[7] = KE;
}
