/*
 * rebo2_oracle.c -- CPU restatement of the REBO-II extension for carbon-only
 * systems: the bond order with the P_CC correction, the radical/conjugation
 * term pi^rc and the dihedral term pi^dh, and AIREBO's switched LJ.
 *
 * TEST INFRASTRUCTURE ONLY, like fmd_oracle.c: only tests/ load it, as the
 * checker of the product's kernels (fuller_md_en_b200/csrc/rebo2.cu).
 *
 * The reference has none of these terms (its compute_rebo, AI:275-421, is
 * b = (1 + sum fc G)^-1/2 and nothing else), so nothing pins this file to the
 * reference beyond one limit: with every spline knot zero the bond order is
 * compute_rebo's and so is the energy (checked against the reference's own
 * recorded E_rebo).  Parity of the spline terms is unpinned: the spline
 * tables of the publications are not part of this repository, and the tests
 * use synthetic knots.  The energies follow the published forms:
 *   Brenner et al., J. Phys.: Condens. Matter 14 (2002) 783, eqs. 1-16
 *   Stuart, Tutein, Harrison, J. Chem. Phys. 112 (2000) 6472, eqs. 2-9
 * with the reference's own pair functions (AI:164-191) and G (AI:181-191).
 * Energies only: forces are checked by central differences of them.
 *
 * The splines are evaluated here from the knots by the tensor-product cubic
 * Hermite basis directly; the product library expands the same splines into
 * per-cell polynomial coefficients, so the two routes check each other.
 */
#include "fmd_oracle.h"
#include <math.h>
#include <stdlib.h>

#define DMAX_CC 2.0
#define LJ_SIG 3.40
#define LJ_EPS 2.84e-3
#define BSW_MIN 0.77
#define BSW_MAX 0.81
#define TAU_C0 0.995
#define PI_D 3.14159265358979323846

void fmo_rebo_pair_fns(double r, double *fc, double *dfc, double *vr, double *dvr, double *va, double *dva);
double fmo_rebo_ang_g(double c);

/* Cubic Hermite basis on [0,1]: h00, h10, h01, h11. */
static void herm(double u, double b[4])
{
    double u2 = u * u, u3 = u2 * u;
    b[0] = 2 * u3 - 3 * u2 + 1;
    b[1] = u3 - 2 * u2 + u;
    b[2] = -2 * u3 + 3 * u2;
    b[3] = u3 - u2;
}

/* Cell index and local coordinate on knots 0..n (argument clamped). */
static int cell(double x, int n, double *u)
{
    if (x < 0) x = 0;
    if (x > n) x = n;
    int c = (int)floor(x);
    if (c > n - 1) c = n - 1;
    *u = x - c;
    return c;
}

/* P_CC(N, N_H = 0) from its knots at N = 0..4 (value, dP/dN). */
static double spline_p(const double k[5][2], double x)
{
    double u, b[4];
    int c = cell(x, 4, &u);
    herm(u, b);
    return k[c][0] * b[0] + k[c][1] * b[1] + k[c + 1][0] * b[2] + k[c + 1][1] * b[3];
}

/* Tricubic Hermite on knots [0..4]x[0..4]x[0..9]; per knot f, fx, fy, fz,
 * fxy, fxz, fyz, fxyz. */
static double spline3(const double k[5][5][10][8], double x, double y, double z)
{
    static const int didx[2][2][2] = {{{0, 3}, {2, 6}}, {{1, 5}, {4, 7}}};
    double u, v, w, bx[4], by[4], bz[4];
    int ix = cell(x, 4, &u), iy = cell(y, 4, &v), iz = cell(z, 9, &w);
    herm(u, bx); herm(v, by); herm(w, bz);
    double f = 0;
    for (int cx = 0; cx < 2; cx++)
        for (int cy = 0; cy < 2; cy++)
            for (int cz = 0; cz < 2; cz++)
                for (int ax = 0; ax < 2; ax++)
                    for (int ay = 0; ay < 2; ay++)
                        for (int az = 0; az < 2; az++)
                            f += k[ix + cx][iy + cy][iz + cz][didx[ax][ay][az]] * bx[2 * cx + ax] *
                                 by[2 * cy + ay] * bz[2 * cz + az];
    return f;
}

/* Cubic switch: 1 for t <= 0, 0 for t >= 1 (Stuart 2000, eq. 4). */
static double sw_cubic(double t)
{
    if (t <= 0) return 1.0;
    if (t >= 1) return 0.0;
    return 1.0 - t * t * (3.0 - 2.0 * t);
}

/* Conjugation switch F(x) of N_conj (Brenner 2002, eq. 15). */
static double f_conj(double x)
{
    if (x <= 2.0) return 1.0;
    if (x >= 3.0) return 0.0;
    return 0.5 * (1.0 + cos(PI_D * (x - 2.0)));
}

/* Weight of a bond angle in the dihedral sum: 1 away from collinear, going
 * smoothly to 0 as |cos| goes from 0.995 to 1 (where the dihedral plane is
 * undefined). */
static double tau(double c)
{
    return sw_cubic((fabs(c) - TAU_C0) / (1.0 - TAU_C0));
}

static void bvec(const double *pos, const double *h, const double *hi, int a, int b, double d[3])
{
    d[0] = pos[3 * b] - pos[3 * a];
    d[1] = pos[3 * b + 1] - pos[3 * a + 1];
    d[2] = pos[3 * b + 2] - pos[3 * a + 2];
    fmo_mimg(&d[0], &d[1], &d[2], hi, h);
}
static double norm(const double d[3]) { return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]); }
static double dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross(const double a[3], const double b[3], double c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static double fcut(double r)
{
    double fc, dfc, vr, dvr, va, dva;
    if (r >= DMAX_CC) return 0.0;
    fmo_rebo_pair_fns(r, &fc, &dfc, &vr, &dvr, &va, &dva);
    return fc;
}

void fmo_rebo2_coordination(const double *pos, const double *h, const double *hi, const int *cnt,
                            const int *list, int max_neigh, int na, double *ncoord)
{
    for (int k = 0; k < na; k++) {
        double s = 0, e[3];
        for (int mn = 0; mn < cnt[k]; mn++) {
            bvec(pos, h, hi, k, list[k * max_neigh + mn], e);
            s += fcut(norm(e));
        }
        ncoord[k] = s;
    }
}

/* One end c of the bond c -> b (bond vector d from c): the sum of fc G over
 * c's other neighbours, their coordination N and the conjugation sum. */
static void side(const double *pos, const double *h, const double *hi, const int *cnt, const int *list,
                 int max_neigh, const double *ncoord, int c, int b, const double d[3], double *gs, double *nc,
                 double *ac)
{
    double r = norm(d), e[3];
    *gs = *nc = *ac = 0;
    for (int kn = 0; kn < cnt[c]; kn++) {
        int k = list[c * max_neigh + kn];
        if (k == b) continue;
        bvec(pos, h, hi, c, k, e);
        double rk = norm(e);
        if (rk >= DMAX_CC) continue;
        double fc = fcut(rk), ct = dot(d, e) / (r * rk);
        if (ct < -1) ct = -1;
        if (ct > 1) ct = 1;
        *gs += fc * fmo_rebo_ang_g(ct);
        *nc += fc;
        *ac += fc * f_conj(ncoord[k] - fc);
    }
}

double fmo_rebo2_bond_order(const double *pos, const double *h, const double *hi, const int *cnt,
                            const int *list, int max_neigh, const fmo_rebo2_knots *kn, const double *ncoord,
                            int i, int j, const double *dij)
{
    double d[3] = {dij[0], dij[1], dij[2]}, md[3] = {-dij[0], -dij[1], -dij[2]};
    double gi, ni, ai, gj, nj, aj;
    side(pos, h, hi, cnt, list, max_neigh, ncoord, i, j, d, &gi, &ni, &ai);
    side(pos, h, hi, cnt, list, max_neigh, ncoord, j, i, md, &gj, &nj, &aj);
    double pij = 1.0 / sqrt(1.0 + gi + spline_p(kn->pcc, ni));
    double pji = 1.0 / sqrt(1.0 + gj + spline_p(kn->pcc, nj));
    double nconj = 1.0 + ai * ai + aj * aj;
    double pirc = spline3(kn->pirc, ni, nj, nconj);
    double t = spline3(kn->tcc, ni, nj, nconj);
    double sdh = 0, r = norm(d);
    if (t != 0.0) {
        for (int kk = 0; kk < cnt[i]; kk++) {
            int k = list[i * max_neigh + kk];
            if (k == j) continue;
            double e1[3];
            bvec(pos, h, hi, i, k, e1);
            double r1 = norm(e1);
            if (r1 >= DMAX_CC) continue;
            double w1 = fcut(r1) * tau(dot(d, e1) / (r * r1));
            if (w1 == 0.0) continue;
            double n1[3];
            cross(d, e1, n1);
            for (int ll = 0; ll < cnt[j]; ll++) {
                int l = list[j * max_neigh + ll];
                if (l == i) continue;
                double e2[3];
                bvec(pos, h, hi, j, l, e2);
                double r2 = norm(e2);
                if (r2 >= DMAX_CC) continue;
                double w2 = fcut(r2) * tau(dot(md, e2) / (r * r2));
                if (w2 == 0.0) continue;
                double n2[3];
                cross(d, e2, n2);
                double v = dot(n1, n2) / (norm(n1) * norm(n2));
                sdh += (1.0 - v * v) * w1 * w2;
            }
        }
    }
    return 0.5 * (pij + pji) + pirc + t * sdh;
}

double fmo_rebo2_energy(const double *pos, const double *h, const double *hi, const int *cnt, const int *list,
                        int max_neigh, int na, const fmo_rebo2_knots *kn)
{
    double *nc = (double *)malloc(sizeof(double) * (na > 0 ? na : 1));
    fmo_rebo2_coordination(pos, h, hi, cnt, list, max_neigh, na, nc);
    double E = 0;
    for (int i = 0; i < na; i++)
        for (int jn = 0; jn < cnt[i]; jn++) {
            int j = list[i * max_neigh + jn];
            if (j <= i) continue;
            double d[3];
            bvec(pos, h, hi, i, j, d);
            double r = norm(d);
            if (r >= DMAX_CC) continue;
            double fc, dfc, vr, dvr, va, dva;
            fmo_rebo_pair_fns(r, &fc, &dfc, &vr, &dvr, &va, &dva);
            double b = fmo_rebo2_bond_order(pos, h, hi, cnt, list, max_neigh, kn, nc, i, j, d);
            E += fc * (vr - b * va);
        }
    free(nc);
    return E;
}

double fmo_lj_switch_energy(const double *pos, const double *h, const double *hi, const int *cnt_r,
                            const int *list_r, int max_neigh_r, const int *cnt_l, const int *list_l,
                            int max_neigh_l, int na, const fmo_rebo2_knots *kn)
{
    const double rmax = pow(2.0, 1.0 / 6.0) * LJ_SIG, rc = 3.0 * LJ_SIG;
    const double sr6 = pow(LJ_SIG / rc, 6), vshift = 4 * LJ_EPS * (sr6 * sr6 - sr6);
    double *nc = (double *)malloc(sizeof(double) * (na > 0 ? na : 1));
    fmo_rebo2_coordination(pos, h, hi, cnt_r, list_r, max_neigh_r, na, nc);
    double E = 0;
    for (int i = 0; i < na; i++)
        for (int jn = 0; jn < cnt_l[i]; jn++) {
            int j = list_l[i * max_neigh_l + jn];
            double d[3];
            bvec(pos, h, hi, i, j, d);
            double r2 = dot(d, d);
            if (r2 >= rmax * rmax) continue;
            double r = sqrt(r2), sr = sw_cubic((r - LJ_SIG) / (rmax - LJ_SIG));
            if (sr == 0.0) continue;
            double r2c = r2 < 0.25 ? 0.25 : r2;
            double s6 = pow(LJ_SIG * LJ_SIG / r2c, 3), v = 4 * LJ_EPS * (s6 * s6 - s6) - vshift;
            double b = fmo_rebo2_bond_order(pos, h, hi, cnt_r, list_r, max_neigh_r, kn, nc, i, j, d);
            double sb = sw_cubic((b - BSW_MIN) / (BSW_MAX - BSW_MIN));
            E += -v * sr * (1.0 - sb);
        }
    free(nc);
    return E;
}

double fmo_rebo2_spline3(const fmo_rebo2_knots *kn, int which, double x, double y, double z)
{
    return spline3(which ? kn->tcc : kn->pirc, x, y, z);
}
double fmo_rebo2_spline_p(const fmo_rebo2_knots *kn, double x) { return spline_p(kn->pcc, x); }
