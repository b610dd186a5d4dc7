// rebo2.cu -- REBO-II extension for carbon-only systems, no counterpart in
// the reference (whose compute_rebo, AI:275-421, has the bond order
// b = (1 + sum f_c G)^-1/2 only):
//
//   bbar_ij = (p_ij + p_ji)/2 + pi^rc_ij + pi^dh_ij                 (Brenner 2002, eq. 3)
//   p_ij    = [1 + sum_k f_c(r_ik) G(cos theta_jik) + P_CC(N_ij)]^-1/2    (eq. 8, lambda = 0 for C)
//   pi^rc   = F_CC(N_ij, N_ji, N_conj)                               (eq. 12)
//   pi^dh   = T_CC(N_ij, N_ji, N_conj) sum_kl (1 - cos^2 w_kijl) f_c(r_ik) f_c(r_jl) tau_ik tau_jl  (eq. 17)
//   N_ij    = sum_{k != j} f_c(r_ik);  N_conj = 1 + A_ij^2 + A_ji^2,
//   A_ij    = sum_{k != j} f_c(r_ik) F(N_k - f_c(r_ik))               (eqs. 14-15)
//   E_REBO  = sum over bonds i<j of f_c(r_ij) [V_R(r_ij) - bbar_ij V_A(r_ij)]
//
// with the reference's own f_c, V_R, V_A and G (AI:164-191), and AIREBO's
// switched LJ (Stuart, Tutein, Harrison 2000, eqs. 2-9) over the reference's
// LJ pair set:
//
//   E_LJ = sum V(r) [1 - S(t_r(r)) (1 - S(t_b(b*_ij)))],
//   t_r = (r - sigma)/(2^(1/6) sigma - sigma),  t_b = (b* - 0.77)/(0.81 - 0.77)
//
// where b*_ij is bbar for the pair's own direction.  The connectivity switch
// C_ij of that paper is 1 for every pair here: the LJ rows pair atoms of
// different molecules (AI:263-272) and the REBO rows only atoms of the same
// molecule (AI:251-261), so no path of REBO bonds joins an LJ pair.
//
// Carbon only: P_CC is needed on the edge N_H = 0, where the bicubic spline
// is the cubic Hermite in N_C through the edge knots.  The splines are cubic
// Hermite in each variable on integer knots (values and derivatives given at
// the knots); the caller supplies the knots (fmd_rebo2_knots), which
// rebo2_coeffs expands into per-cell polynomial coefficients.  tau(c) (the
// weight of a bond angle in the dihedral sum) is 1 for |cos| <= 0.995 and
// goes to 0 at |cos| = 1 by the cubic switch, so the dihedral term is smooth
// where its plane is undefined.
//
// Forces are -grad E of exactly this energy, and the virial is the full one:
// every term depends on bond vectors only, and each gradient g with respect to
// a bond vector e = r_b - r_a adds F_a += g, F_b -= g and W -= e (x) g (the
// reference's pair virial convention, AI:339-349, extended to every term).
// A scan compacts the work (the bonds of the REBO rows; the LJ pairs closer
// than 2^(1/6) sigma), then one thread per item, FP64 throughout, forces by
// atomics, energy and virial as per-block partial records.
#include <cmath>
#include <cstring>

#include "kernels.h"
#include "ljpair.cuh"
#include "pdl.cuh"
#include "rebo_fn.cuh"

namespace fmd {
namespace {

using namespace rebo;

constexpr double kBswMin = 0.77, kBswMax = 0.81;   // bond-order switch of the LJ term
constexpr double kTauC0 = 0.995;                   // dihedral angle weight starts to fall
constexpr double kSwitchRmaxOverSigma2 = 1.2599210498948732;   // (2^(1/6))^2: the switch ends at 2^(1/6) sigma

struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double len(V3 a) { return sqrt(dot(a, a)); }

// Cubic switch S(t): 1 for t <= 0, 0 for t >= 1, 1 - t^2 (3 - 2t) between.
__device__ __forceinline__ void sw_cubic(double t, double& s, double& ds) {
    if (t <= 0.0) { s = 1.0; ds = 0.0; return; }
    if (t >= 1.0) { s = 0.0; ds = 0.0; return; }
    s = 1.0 - t * t * (3.0 - 2.0 * t);
    ds = -6.0 * t * (1.0 - t);
}

// F(x) of the conjugation number: 1 for x <= 2, 0 for x >= 3, cosine between.
__device__ __forceinline__ void f_conj(double x, double& f, double& df) {
    if (x <= 2.0) { f = 1.0; df = 0.0; return; }
    if (x >= 3.0) { f = 0.0; df = 0.0; return; }
    f = 0.5 * (1.0 + cos(kPi * (x - 2.0)));
    df = -0.5 * kPi * sin(kPi * (x - 2.0));
}

__device__ __forceinline__ void tau_fn(double c, double& t, double& dt) {
    double s, ds;
    sw_cubic((fabs(c) - kTauC0) / (1.0 - kTauC0), s, ds);
    t = s;
    dt = ds / (1.0 - kTauC0) * (c < 0.0 ? -1.0 : 1.0);
}

// Cell and local coordinate on knots 0..n; out: the argument was clamped
// (the spline is constant beyond the table, so its derivative is zero).
__device__ __forceinline__ int knot_cell(double x, int n, double& u, bool& out) {
    out = x < 0.0 || x > (double)n;
    x = fmin(fmax(x, 0.0), (double)n);
    const int c = min((int)floor(x), n - 1);
    u = x - c;
    return c;
}

// P_CC(N, 0): coefficients q[4 * cell + a] of u^a.
__device__ __forceinline__ double spline_p(const double* __restrict__ q, double x, double& dx) {
    double u;
    bool out;
    const double* c = q + 4 * knot_cell(x, kRebo2Nx, u, out);
    const double f = c[0] + u * (c[1] + u * (c[2] + u * c[3]));
    dx = out ? 0.0 : c[1] + u * (2.0 * c[2] + 3.0 * u * c[3]);
    return f;
}

// Tricubic: coefficients c[a + 4 b + 16 cz] of u^a v^b w^cz per cell.
__device__ double spline3(const double* __restrict__ tab, double x, double y, double z, double& gx, double& gy,
                          double& gz) {
    double u, v, w;
    bool ox, oy, oz;
    const int ix = knot_cell(x, kRebo2Nx, u, ox), iy = knot_cell(y, kRebo2Ny, v, oy),
              iz = knot_cell(z, kRebo2Nz, w, oz);
    const double* c = tab + (size_t)((ix * kRebo2Ny + iy) * kRebo2Nz + iz) * 64;
    double f = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
    for (int cz = 3; cz >= 0; cz--) {
        double py = 0.0, pyx = 0.0, pyy = 0.0;
        for (int b = 3; b >= 0; b--) {
            const double* q = c + 4 * b + 16 * cz;
            const double px = q[0] + u * (q[1] + u * (q[2] + u * q[3]));
            const double dpx = q[1] + u * (2.0 * q[2] + 3.0 * u * q[3]);
            pyy = pyy * v + py;      // d/dv of the Horner sum, before py advances
            py = py * v + px;
            pyx = pyx * v + dpx;
        }
        fz = fz * w + f;
        f = f * w + py;
        fx = fx * w + pyx;
        fy = fy * w + pyy;
    }
    gx = ox ? 0.0 : fx;
    gy = oy ? 0.0 : fy;
    gz = oz ? 0.0 : fz;
    return f;
}

struct Geo {
    const double* pos;
    const int* cnt;
    const int* list;
    int cap;
    const double* h;
    const double* hi;
    const double* ncoord;
    Rebo2Dev t;
};

__device__ __forceinline__ V3 bvec(const Geo& g, int a, int b) {
    double x, y, z;
    bond_vec(g.pos, a, b, g.h, g.hi, x, y, z);
    return {x, y, z};
}

__device__ __forceinline__ void cut_fns(double r, double& fc, double& dfc) {
    fc = r >= DMAX_CC ? 0.0 : sw_fc(r);
    dfc = r >= DMAX_CC ? 0.0 : sw_dfc(r);
}

__device__ __forceinline__ void pair_fns(double r, double& vr, double& dvr, double& va, double& dva) {
    const double ea = A_CC * exp(-ALPHA_CC * r), qr = Q_CC / r;
    vr = (1.0 + qr) * ea;
    dvr = (-qr / r) * ea - ALPHA_CC * (1.0 + qr) * ea;
    const double e1 = exp(-BETA1_CC * r), e2 = exp(-BETA2_CC * r), e3 = exp(-BETA3_CC * r);
    va = B1_CC * e1 + B2_CC * e2 + B3_CC * e3;
    dva = -BETA1_CC * B1_CC * e1 - BETA2_CC * B2_CC * e2 - BETA3_CC * B3_CC * e3;
}

// F_a += g, F_b -= g, W -= e (x) g for a gradient g of E with respect to the
// bond vector e = r_b - r_a.
__device__ __forceinline__ void scatter(double* __restrict__ F, double (&w)[9], int a, int b, V3 e, V3 g) {
    atomic_add3(F, a, g.x, g.y, g.z);
    atomic_add3(F, b, -g.x, -g.y, -g.z);
    const double ev[3] = {e.x, e.y, e.z}, gv[3] = {g.x, g.y, g.z};
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
        for (int q = 0; q < 3; q++) w[3 * p + q] -= ev[p] * gv[q];
}

// Scalars of bbar for one bond (or LJ pair) i -> j.
struct BoState {
    double pi, pj, dPi, dPj, Ai, Aj;
    double prc, prc_x, prc_y, prc_z;
    double T, T_x, T_y, T_z;
    double sdh, b;
};

// Centre c's sums over its neighbours other than skip, for the bond whose
// unit vector from c is u: sum f_c G, N, A.
__device__ void side_sums(const Geo& g, int c, int skip, V3 u, double& gs, double& n, double& a) {
    gs = n = a = 0.0;
    const int m = g.cnt[c];
    for (int kn = 0; kn < m; kn++) {
        const int k = g.list[(size_t)c * g.cap + kn];
        if (k == skip) continue;
        const V3 e = bvec(g, c, k);
        const double rk = len(e);
        if (rk >= DMAX_CC) continue;
        const double fc = sw_fc(rk);
        const double ct = clamp1(dot(u, e) / rk);
        double f, df;
        f_conj(g.ncoord[k] - fc, f, df);
        gs += fc * ang_g(ct);
        n += fc;
        a += fc * f;
    }
}

// sum over k of i, l of j of (1 - cos^2 w) f_c f_c tau tau.
__device__ double dihedral_sum(const Geo& g, int i, int j, V3 d, double r) {
    const V3 u = (1.0 / r) * d;
    double s = 0.0;
    const int mi = g.cnt[i], mj = g.cnt[j];
    for (int kn = 0; kn < mi; kn++) {
        const int k = g.list[(size_t)i * g.cap + kn];
        if (k == j) continue;
        const V3 e1 = bvec(g, i, k);
        const double r1 = len(e1);
        if (r1 >= DMAX_CC) continue;
        double t1, dt1;
        tau_fn(dot(u, e1) / r1, t1, dt1);
        const double w1 = sw_fc(r1) * t1;
        if (w1 == 0.0) continue;
        const V3 n1 = cross(d, e1);
        const double l1 = len(n1);
        for (int ln = 0; ln < mj; ln++) {
            const int l = g.list[(size_t)j * g.cap + ln];
            if (l == i) continue;
            const V3 e2 = bvec(g, j, l);
            const double r2 = len(e2);
            if (r2 >= DMAX_CC) continue;
            double t2, dt2;
            tau_fn(-dot(u, e2) / r2, t2, dt2);
            const double w2 = sw_fc(r2) * t2;
            if (w2 == 0.0) continue;
            const V3 n2 = cross(d, e2);
            const double v = dot(n1, n2) / (l1 * len(n2));
            s += (1.0 - v * v) * w1 * w2;
        }
    }
    return s;
}

__device__ void bo_eval(const Geo& g, int i, int j, V3 d, double r, BoState& s) {
    const V3 u = (1.0 / r) * d;
    double gi, ni, gj, nj;
    side_sums(g, i, j, u, gi, ni, s.Ai);
    side_sums(g, j, i, -1.0 * u, gj, nj, s.Aj);
    s.pi = 1.0 / sqrt(1.0 + gi + spline_p(g.t.pcc, ni, s.dPi));
    s.pj = 1.0 / sqrt(1.0 + gj + spline_p(g.t.pcc, nj, s.dPj));
    const double nconj = 1.0 + s.Ai * s.Ai + s.Aj * s.Aj;
    s.prc = spline3(g.t.pirc, ni, nj, nconj, s.prc_x, s.prc_y, s.prc_z);
    s.T = spline3(g.t.tcc, ni, nj, nconj, s.T_x, s.T_y, s.T_z);
    const bool dh = s.T != 0.0 || s.T_x != 0.0 || s.T_y != 0.0 || s.T_z != 0.0;
    s.sdh = dh ? dihedral_sum(g, i, j, d, r) : 0.0;
    s.b = 0.5 * (s.pi + s.pj) + s.prc + s.T * s.sdh;
}

// Gradient of bbar times beta through centre c's side (c -> skip along unit
// u, bond length r): scatters the terms on c's other bonds (and, through the
// conjugation number, on those neighbours' bonds) and returns the gradient
// with respect to the bond vector c -> skip.
__device__ V3 side_grad(const Geo& g, double* __restrict__ F, double (&w)[9], int c, int skip, V3 u, double r,
                        double aS, double aN, double aA) {
    V3 gu{0.0, 0.0, 0.0};
    const int m = g.cnt[c];
    for (int kn = 0; kn < m; kn++) {
        const int k = g.list[(size_t)c * g.cap + kn];
        if (k == skip) continue;
        const V3 e = bvec(g, c, k);
        const double rk = len(e);
        if (rk >= DMAX_CC) continue;
        const V3 uk = (1.0 / rk) * e;
        double fc, dfc;
        cut_fns(rk, fc, dfc);
        const double ct = clamp1(dot(u, uk));
        const double G = ang_g(ct), dG = ang_dg(ct);
        double f, df;
        f_conj(g.ncoord[k] - fc, f, df);
        const double cr = aS * dfc * G + aN * dfc + aA * dfc * f;
        const double cc = aS * fc * dG;
        V3 ge = cr * uk + (cc / rk) * (u - ct * uk);
        gu += (cc / r) * (uk - ct * u);
        // x = N_k - f_c(r_ck) through k's own bonds
        const double q = aA * fc * df;
        if (q != 0.0) {
            bool found = false;
            const int mk = g.cnt[k];
            for (int mn = 0; mn < mk; mn++) {
                const int mm = g.list[(size_t)k * g.cap + mn];
                if (mm == c) { found = true; continue; }
                const V3 e2 = bvec(g, k, mm);
                const double r2 = len(e2);
                if (r2 >= DMAX_CC) continue;
                double fc2, dfc2;
                cut_fns(r2, fc2, dfc2);
                if (dfc2 != 0.0) scatter(F, w, k, mm, e2, (q * dfc2 / r2) * e2);
            }
            // c absent from k's row: N_k lacks f_c(r_kc), x depends on e directly
            if (!found) ge += (-q * dfc) * uk;
        }
        scatter(F, w, c, k, e, ge);
    }
    return gu;
}

// Gradient of aD * (dihedral sum); returns the part on the bond vector d.
__device__ V3 dihedral_grad(const Geo& g, double* __restrict__ F, double (&w)[9], int i, int j, V3 d, double r,
                            double aD) {
    const V3 u = (1.0 / r) * d;
    V3 gd{0.0, 0.0, 0.0};
    const int mi = g.cnt[i], mj = g.cnt[j];
    for (int kn = 0; kn < mi; kn++) {
        const int k = g.list[(size_t)i * g.cap + kn];
        if (k == j) continue;
        const V3 e1 = bvec(g, i, k);
        const double r1 = len(e1);
        if (r1 >= DMAX_CC) continue;
        const V3 u1 = (1.0 / r1) * e1;
        double fc1, dfc1, t1, dt1;
        cut_fns(r1, fc1, dfc1);
        const double c1 = clamp1(dot(u, u1));
        tau_fn(c1, t1, dt1);
        if (t1 == 0.0) continue;
        const V3 n1 = cross(d, e1);
        const double l1 = len(n1);
        const V3 h1 = (1.0 / l1) * n1;
        V3 g1{0.0, 0.0, 0.0};
        for (int ln = 0; ln < mj; ln++) {
            const int l = g.list[(size_t)j * g.cap + ln];
            if (l == i) continue;
            const V3 e2 = bvec(g, j, l);
            const double r2 = len(e2);
            if (r2 >= DMAX_CC) continue;
            const V3 u2 = (1.0 / r2) * e2;
            double fc2, dfc2, t2, dt2;
            cut_fns(r2, fc2, dfc2);
            const double c2 = clamp1(-dot(u, u2));
            tau_fn(c2, t2, dt2);
            if (t2 == 0.0) continue;
            const V3 n2 = cross(d, e2);
            const double l2 = len(n2);
            const V3 h2 = (1.0 / l2) * n2;
            const double v = dot(h1, h2), Q = 1.0 - v * v;
            // through cos w
            const double av = aD * (-2.0 * v) * fc1 * fc2 * t1 * t2;
            const V3 w1 = (1.0 / l1) * (h2 - v * h1), w2 = (1.0 / l2) * (h1 - v * h2);
            gd += av * (cross(e1, w1) + cross(e2, w2));
            g1 += av * cross(w1, d);
            V3 g2 = av * cross(w2, d);
            // through the cutoffs
            g1 += (aD * Q * fc2 * t1 * t2 * dfc1) * u1;
            g2 += (aD * Q * fc1 * t1 * t2 * dfc2) * u2;
            // through the angle weights: c1 = u.u1, c2 = -u.u2
            const double a1 = aD * Q * fc1 * fc2 * t2 * dt1, a2 = aD * Q * fc1 * fc2 * t1 * dt2;
            gd += (a1 / r) * (u1 - c1 * u);
            g1 += (a1 / r1) * (u - c1 * u1);
            gd += (-a2 / r) * (u2 + c2 * u);
            g2 += (a2 / r2) * (-1.0 * u - c2 * u2);
            scatter(F, w, j, l, e2, g2);
        }
        scatter(F, w, i, k, e1, g1);
    }
    return gd;
}

// Gradient of beta * bbar_ij: scatters every term off the bond itself and
// returns the part on the bond vector d = r_j - r_i.
__device__ V3 bo_grad(const Geo& g, double* __restrict__ F, double (&w)[9], int i, int j, V3 d, double r,
                      const BoState& s, double beta) {
    const V3 u = (1.0 / r) * d;
    const double aSi = -0.25 * beta * s.pi * s.pi * s.pi, aSj = -0.25 * beta * s.pj * s.pj * s.pj;
    const double aNi = aSi * s.dPi + beta * (s.prc_x + s.T_x * s.sdh);
    const double aNj = aSj * s.dPj + beta * (s.prc_y + s.T_y * s.sdh);
    const double aC = beta * (s.prc_z + s.T_z * s.sdh);
    V3 gd = side_grad(g, F, w, i, j, u, r, aSi, aNi, 2.0 * aC * s.Ai);
    const V3 ge = side_grad(g, F, w, j, i, -1.0 * u, r, aSj, aNj, 2.0 * aC * s.Aj);
    gd += -1.0 * ge;
    if (s.T != 0.0) gd += dihedral_grad(g, F, w, i, j, d, r, beta * s.T);
    return gd;
}

__global__ void __launch_bounds__(256)
k_rebo2_coord(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
              const int* __restrict__ list, int cap, int na, double* __restrict__ ncoord) {
    FMD_PDL_WAIT();
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < na; k += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int mn = 0; mn < cnt[k]; mn++) {
            double x, y, z;
            bond_vec(pos, k, list[(size_t)k * cap + mn], s_hh, s_hh + 9, x, y, z);
            const double r = sqrt(x * x + y * y + z * z);
            if (r < DMAX_CC) s += sw_fc(r);
        }
        ncoord[k] = s;
    }
}

// Appends (i, j) to a compacted work list from every lane of the warp that
// takes its entry (one atomic per warp); entries beyond cap are dropped and
// reported in err.  The whole warp calls it.
__device__ __forceinline__ void warp_append(bool take, int i, int j, int2* __restrict__ out, int* __restrict__ count,
                                            int cap, DevErr* err) {
    const unsigned m = __ballot_sync(kFull, take);
    if (!m) return;
    const int lane = threadIdx.x & 31, lead = __ffs(m) - 1;
    int base = 0;
    if (lane == lead) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(kFull, base, lead);
    if (!take) return;
    const int k = base + __popc(m & ((1u << lane) - 1u));
    if (k < cap) out[k] = make_int2(i, j);
    else if (err && atomicCAS(&err->code, FMD_OK, FMD_ERR_CAPACITY) == FMD_OK) {
        err->where = K_REBO2; err->index = i; err->value = k + 1;
    }
}

// The bonds of the REBO rows: slot i -> j with j > i (the enumeration of
// AI:286-290) and r < D_max, compacted (the rows are 12 wide and hold ~3).
__global__ void __launch_bounds__(256)
k_rebo2_scan(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
             const int* __restrict__ list, int cap, int na, Rebo2Dev t) {
    FMD_PDL_WAIT();
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const long long tot = (long long)na * cap, stride = (long long)gridDim.x * blockDim.x;
    for (long long b = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); b < tot; b += stride) {
        const long long s = b + (threadIdx.x & 31);
        bool take = false;
        int i = 0, j = 0;
        if (s < tot) {
            i = (int)(s / cap);
            const int jn = (int)(s - (long long)i * cap);
            if (jn < cnt[i]) {
                j = list[s];
                if (j > i) {
                    double x, y, z;
                    bond_vec(pos, i, j, s_hh, s_hh + 9, x, y, z);
                    take = sqrt(x * x + y * y + z * z) < DMAX_CC;
                }
            }
        }
        warp_append(take, i, j, t.bonds, &t.counts[0], na * cap, nullptr);
    }
}

// One thread per bond of the compacted list: the bond's energy, and forces
// and virial of its gradient.  Capped at 128 registers (4 blocks per SM; some
// spill to L1): the uncapped kernel held 254 registers at 7 warps per SM and
// took 123 us at nc = 5, the capped one 97 us.
__global__ void __launch_bounds__(128, 4)
k_rebo2_bonds(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
              const int* __restrict__ list, int cap, Rebo2Dev t, double* __restrict__ F, double* __restrict__ part) {
    FMD_PDL_WAIT();
    __shared__ double sm[32 * kNV];
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const Geo g{pos, cnt, list, cap, s_hh, s_hh + 9, t.ncoord, t};
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int nb = t.counts[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
        const int2 ij = t.bonds[k];
        const int i = ij.x, j = ij.y;
        const V3 d = bvec(g, i, j);
        const double r = len(d);
        double fc, dfc, vr, dvr, va, dva;
        cut_fns(r, fc, dfc);
        pair_fns(r, vr, dvr, va, dva);
        BoState st;
        bo_eval(g, i, j, d, r, st);
        acc[0] += fc * (vr - st.b * va);
        V3 gd = ((dfc * (vr - st.b * va) + fc * (dvr - st.b * dva)) / r) * d;
        gd += bo_grad(g, F, w, i, j, d, r, st, -fc * va);
        scatter(F, w, i, j, d, gd);
    }
#pragma unroll
    for (int q = 0; q < 9; q++) acc[1 + q] = w[q];
    block_sum_store<kNV>(acc, sm, part + (size_t)blockIdx.x * kNV);
}

// The LJ pairs closer than 2^(1/6) sigma (where the switch acts), compacted
// from the half rows.
__global__ void __launch_bounds__(256)
k_lj_switch_scan(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt_a,
                 const int* __restrict__ list_a, int cap_a, int na, Rebo2Dev t) {
    FMD_PDL_WAIT();
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const LJP lp = lj_params_dev(FMD_FF_AIREBO);
    const double rmax2 = kSwitchRmaxOverSigma2 * lp.sig2;
    const long long tot = (long long)na * cap_a, stride = (long long)gridDim.x * blockDim.x;
    for (long long b = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); b < tot; b += stride) {
        const long long s = b + (threadIdx.x & 31);
        bool take = false;
        int i = 0, j = 0;
        if (s < tot) {
            i = (int)(s / cap_a);
            const int jn = (int)(s - (long long)i * cap_a);
            if (jn < cnt_a[i]) {
                j = list_a[s];
                double x, y, z;
                bond_vec(pos, i, j, s_hh, s_hh + 9, x, y, z);
                take = x * x + y * y + z * z < rmax2;
            }
        }
        warp_append(take, i, j, t.sw_pairs, &t.counts[1], t.sw_cap, t.err);
    }
}

// One thread per compacted close LJ pair: the correction
// -V S(t_r) (1 - S(t_b(b*))) that turns the plain LJ term into the switched one.
__global__ void __launch_bounds__(128)
k_lj_switch(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt_b,
            const int* __restrict__ list_b, int cap_b, Rebo2Dev t, double* __restrict__ F, double* __restrict__ part) {
    FMD_PDL_WAIT();
    __shared__ double sm[32 * kNV];
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const Geo g{pos, cnt_b, list_b, cap_b, s_hh, s_hh + 9, t.ncoord, t};
    const LJP lp = lj_params_dev(FMD_FF_AIREBO);
    const double sig = sqrt(lp.sig2), rmax = sqrt(kSwitchRmaxOverSigma2) * sig;
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int np = min(t.counts[1], t.sw_cap);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        const int2 ij = t.sw_pairs[k];
        const int i = ij.x, j = ij.y;
        const V3 d = bvec(g, i, j);
        const double r2 = dot(d, d), r = sqrt(r2);
        double sr, dsr;
        sw_cubic((r - sig) / (rmax - sig), sr, dsr);
        if (sr == 0.0) continue;
        dsr /= (rmax - sig);
        // the plain term's V (AI:447-457, r^2 clamped at 0.25)
        const double r2c = r2 < 0.25 ? 0.25 : r2;
        const double s2 = lp.sig2 / r2c, s6 = s2 * s2 * s2, s12 = s6 * s6;
        const double v = lp.c4 * (s12 - s6) - lp.vshift;
        const double dv = r2 < 0.25 ? 0.0 : -lp.c24 * (2.0 * s12 - s6) / r;
        BoState st;
        bo_eval(g, i, j, d, r, st);
        double sb, dsb;
        sw_cubic((st.b - kBswMin) / (kBswMax - kBswMin), sb, dsb);
        dsb /= (kBswMax - kBswMin);
        acc[0] += -v * sr * (1.0 - sb);
        V3 gd = (-(dv * sr + v * dsr) * (1.0 - sb) / r) * d;
        const double beta = v * sr * dsb;
        if (beta != 0.0) gd += bo_grad(g, F, w, i, j, d, r, st, beta);
        scatter(F, w, i, j, d, gd);
    }
#pragma unroll
    for (int q = 0; q < 9; q++) acc[1 + q] = w[q];
    block_sum_store<kNV>(acc, sm, part + (size_t)blockIdx.x * kNV);
}

// Cubic Hermite basis on [0,1] as polynomial coefficients of u^0..u^3:
// h00, h10 (slope at 0), h01, h11 (slope at 1).
constexpr double kHerm[4][4] = {{1, 0, -3, 2}, {0, 1, -2, 1}, {0, 0, 3, -2}, {0, 0, -1, 1}};

}  // namespace

cudaError_t rebo2_coord_launch(const Rebo2Dev& t, const double* pos, const double* hh, const int* cnt,
                               const int* list, int cap, int na, cudaStream_t st) {
    const int nb = std::max(1, std::min((na + 255) / 256, kForceBlocks));
    return launch_pdl(k_rebo2_coord, dim3(nb), dim3(256), 0, st, pos, hh, cnt, list, cap, na, t.ncoord);
}

cudaError_t rebo2_launch(const Rebo2Dev& t, const double* pos, const double* hh, const int* cnt, const int* list,
                         int cap, int na, double* F, double* part, int nblk, cudaStream_t st) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(t.counts, 0, 2 * sizeof(int), st)) != cudaSuccess) return e;
    if ((e = rebo2_coord_launch(t, pos, hh, cnt, list, cap, na, st)) != cudaSuccess) return e;
    const int ns = std::max(1, std::min((int)(((long long)na * cap + 255) / 256), kForceBlocks));
    if ((e = launch_pdl(k_rebo2_scan, dim3(ns), dim3(256), 0, st, pos, hh, cnt, list, cap, na, t)) != cudaSuccess)
        return e;
    return launch_pdl(k_rebo2_bonds, dim3(nblk), dim3(128), 0, st, pos, hh, cnt, list, cap, t, F, part);
}

cudaError_t lj_switch_launch(const Rebo2Dev& t, const double* pos, const double* hh, const int* cnt_b,
                             const int* list_b, int cap_b, const int* cnt_a, const int* list_a, int cap_a, int na,
                             double* F, double* part, int nblk, bool coord_ready, cudaStream_t st) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(t.counts + 1, 0, sizeof(int), st)) != cudaSuccess) return e;
    if (!coord_ready && (e = rebo2_coord_launch(t, pos, hh, cnt_b, list_b, cap_b, na, st)) != cudaSuccess) return e;
    const int ns = std::max(1, std::min((int)(((long long)na * cap_a + 255) / 256), 4 * kForceBlocks));
    if ((e = launch_pdl(k_lj_switch_scan, dim3(ns), dim3(256), 0, st, pos, hh, cnt_a, list_a, cap_a, na, t)) !=
        cudaSuccess)
        return e;
    return launch_pdl(k_lj_switch, dim3(nblk), dim3(128), 0, st, pos, hh, cnt_b, list_b, cap_b, t, F, part);
}

void rebo2_coeffs(const double* knots, double* pcc, double* pirc, double* tcc) {
    // P_CC: knots[n][2] = {P, dP/dN} at N = n
    for (int n = 0; n < kRebo2Nx; n++)
        for (int a = 0; a < 4; a++)
            pcc[4 * n + a] = knots[2 * n] * kHerm[0][a] + knots[2 * n + 1] * kHerm[1][a] +
                             knots[2 * (n + 1)] * kHerm[2][a] + knots[2 * (n + 1) + 1] * kHerm[3][a];
    // tricubic: knots[x][y][z][8], derivative slot of (ax, ay, az)
    static const int didx[2][2][2] = {{{0, 3}, {2, 6}}, {{1, 5}, {4, 7}}};
    const int NY = kRebo2Ny + 1, NZ = kRebo2Nz + 1;
    for (int tab = 0; tab < 2; tab++) {
        const double* kn = knots + 2 * (kRebo2Nx + 1) + (size_t)tab * (kRebo2Nx + 1) * NY * NZ * 8;
        double* out = tab ? tcc : pirc;
        for (int ix = 0; ix < kRebo2Nx; ix++)
            for (int iy = 0; iy < kRebo2Ny; iy++)
                for (int iz = 0; iz < kRebo2Nz; iz++) {
                    double* c = out + (size_t)((ix * kRebo2Ny + iy) * kRebo2Nz + iz) * 64;
                    std::memset(c, 0, sizeof(double) * 64);
                    for (int cx = 0; cx < 2; cx++)
                        for (int cy = 0; cy < 2; cy++)
                            for (int cz = 0; cz < 2; cz++) {
                                const double* kv = kn + (size_t)(((ix + cx) * NY + iy + cy) * NZ + iz + cz) * 8;
                                for (int ax = 0; ax < 2; ax++)
                                    for (int ay = 0; ay < 2; ay++)
                                        for (int az = 0; az < 2; az++) {
                                            const double D = kv[didx[ax][ay][az]];
                                            if (D == 0.0) continue;
                                            const double* hx = kHerm[2 * cx + ax];
                                            const double* hy = kHerm[2 * cy + ay];
                                            const double* hz = kHerm[2 * cz + az];
                                            for (int a = 0; a < 4; a++)
                                                for (int b = 0; b < 4; b++)
                                                    for (int q = 0; q < 4; q++)
                                                        c[a + 4 * b + 16 * q] += D * hx[a] * hy[b] * hz[q];
                                        }
                            }
                }
    }
}

}  // namespace fmd
