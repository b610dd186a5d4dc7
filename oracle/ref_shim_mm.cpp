// ref_shim_mm.cpp -- extern "C" access to the unmodified reference
// molecular-mechanics program.  REF_SRC is set by oracle/Makefile; main() is
// renamed to ref_main.  TEST INFRASTRUCTURE ONLY.
#include REF_SRC

namespace {
void npt_in(const double* a, NPTState& s) {
    s.xi = a[0]; s.Q = a[1];
    for (int k = 0; k < 9; k++) s.Vg[k] = a[2 + k];
    s.W_ = a[11]; s.Pe = a[12]; s.Tt = a[13]; s.Nf = (int)a[14];
}
void npt_out(const NPTState& s, double* a) {
    a[0] = s.xi; a[1] = s.Q;
    for (int k = 0; k < 9; k++) a[2 + k] = s.Vg[k];
    a[11] = s.W_; a[12] = s.Pe; a[13] = s.Tt; a[14] = s.Nf;
}
// Flat topology view over caller arrays (no ownership).
FlatTopology topo_view(int nb, int* bi, double* bk, double* br, int na_, int* ai, double* ak,
                       double* at, int nd, int* di, double* dv, int* dm, double* dg, int ni,
                       int* ii, double* ik, double* ig, int* mol_id) {
    FlatTopology t;
    t.Nb = nb; t.b_i0 = bi; t.b_i1 = bi + nb; t.b_kb = bk; t.b_r0 = br;
    t.Nang = na_; t.ang_i0 = ai; t.ang_i1 = ai + na_; t.ang_i2 = ai + 2 * na_; t.ang_kth = ak; t.ang_th0 = at;
    t.Ndih = nd; t.dih_i0 = di; t.dih_i1 = di + nd; t.dih_i2 = di + 2 * nd; t.dih_i3 = di + 3 * nd;
    t.dih_Vn = dv; t.dih_mult = dm; t.dih_gamma = dg;
    t.Nimp = ni; t.imp_i0 = ii; t.imp_i1 = ii + ni; t.imp_i2 = ii + 2 * ni; t.imp_i3 = ii + 3 * ni;
    t.imp_ki = ik; t.imp_gamma = ig; t.mol_id = mol_id;
    return t;
}
}  // namespace

extern "C" {
void ref_mm_build_nlist_lj(const double* pos, const double* h, const double* hi, int na,
                           const int* mol_id, int* nlc, int* nll) {
    build_nlist_lj(pos, h, hi, na, mol_id, nlc, nll);
}
void ref_mm_make_npt(double T, double Pe, int na, double* npt) { npt_out(make_npt(T, Pe, na), npt); }

// build_flat_topology (MM:254) for a molecule given as coordinates + bond pairs.
// counts[4] = per-molecule {nb, nang, ndih, nimp}; when out arrays are
// non-null they receive the replicated topology (index arrays are
// column-blocked: all i0 then all i1 ...).
void ref_mm_build_topology(const double* coords, int natom, const int* bonds, int nbond, int nmol,
                           double kb, double kth, double v2, double kimp, int* counts,
                           int* bi, double* bk, double* br, int* ai, double* ak, double* at,
                           int* di, double* dv, int* dm, double* dg, int* ii, double* ik, double* ig,
                           int* mol_id) {
    MolData md;
    md.natom = natom;
    md.coords.resize(natom);
    for (int i = 0; i < natom; i++) md.coords[i] = {coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]};
    for (int b = 0; b < nbond; b++) md.bonds.push_back({bonds[2 * b], bonds[2 * b + 1]});
    md.Rmol = md.Dmol = 0;
    FlatTopology ft = build_flat_topology(md, nmol, kb, kth, v2, kimp);
    counts[0] = ft.Nb / nmol; counts[1] = ft.Nang / nmol; counts[2] = ft.Ndih / nmol; counts[3] = ft.Nimp / nmol;
    if (bi) {
        for (int k = 0; k < ft.Nb; k++) { bi[k] = ft.b_i0[k]; bi[ft.Nb + k] = ft.b_i1[k]; bk[k] = ft.b_kb[k]; br[k] = ft.b_r0[k]; }
        for (int k = 0; k < ft.Nang; k++) {
            ai[k] = ft.ang_i0[k]; ai[ft.Nang + k] = ft.ang_i1[k]; ai[2 * ft.Nang + k] = ft.ang_i2[k];
            ak[k] = ft.ang_kth[k]; at[k] = ft.ang_th0[k];
        }
        for (int k = 0; k < ft.Ndih; k++) {
            di[k] = ft.dih_i0[k]; di[ft.Ndih + k] = ft.dih_i1[k]; di[2 * ft.Ndih + k] = ft.dih_i2[k];
            di[3 * ft.Ndih + k] = ft.dih_i3[k]; dv[k] = ft.dih_Vn[k]; dm[k] = ft.dih_mult[k]; dg[k] = ft.dih_gamma[k];
        }
        for (int k = 0; k < ft.Nimp; k++) {
            ii[k] = ft.imp_i0[k]; ii[ft.Nimp + k] = ft.imp_i1[k]; ii[2 * ft.Nimp + k] = ft.imp_i2[k];
            ii[3 * ft.Nimp + k] = ft.imp_i3[k]; ik[k] = ft.imp_ki[k]; ig[k] = ft.imp_gamma[k];
        }
        for (int k = 0; k < nmol * natom; k++) mol_id[k] = ft.mol_id[k];
    }
    delete[] ft.b_i0; delete[] ft.b_i1; delete[] ft.b_kb; delete[] ft.b_r0;
    delete[] ft.ang_i0; delete[] ft.ang_i1; delete[] ft.ang_i2; delete[] ft.ang_kth; delete[] ft.ang_th0;
    delete[] ft.dih_i0; delete[] ft.dih_i1; delete[] ft.dih_i2; delete[] ft.dih_i3;
    delete[] ft.dih_Vn; delete[] ft.dih_mult; delete[] ft.dih_gamma;
    delete[] ft.imp_i0; delete[] ft.imp_i1; delete[] ft.imp_i2; delete[] ft.imp_i3;
    delete[] ft.imp_ki; delete[] ft.imp_gamma; delete[] ft.mol_id;
}

// compute_forces (MM:351) over a caller-held topology; E7 = ForceResult fields.
void ref_mm_compute_forces(double* F, double* vir9, const double* pos, const double* h,
                           const double* hi, int nb, int* bi, double* bk, double* br, int nang,
                           int* ai, double* ak, double* at, int nd, int* di, double* dv, int* dm,
                           double* dg, int ni, int* ii, double* ik, double* ig, const int* nlc,
                           const int* nll, const double* charge, int* mol_id, int has_charge,
                           int na, double* E7) {
    FlatTopology t = topo_view(nb, bi, bk, br, nang, ai, ak, at, nd, di, dv, dm, dg, ni, ii, ik, ig, mol_id);
    ForceResult r = compute_forces(F, vir9, pos, h, hi, t.Nb, t.b_i0, t.b_i1, t.b_kb, t.b_r0,
        t.Nang, t.ang_i0, t.ang_i1, t.ang_i2, t.ang_kth, t.ang_th0,
        t.Ndih, t.dih_i0, t.dih_i1, t.dih_i2, t.dih_i3, t.dih_Vn, t.dih_mult, t.dih_gamma,
        t.Nimp, t.imp_i0, t.imp_i1, t.imp_i2, t.imp_i3, t.imp_ki, t.imp_gamma,
        nlc, nll, charge, mol_id, has_charge != 0, na);
    E7[0] = r.Eb; E7[1] = r.Ea; E7[2] = r.Ed; E7[3] = r.Ei; E7[4] = r.Elj; E7[5] = r.Ecoul; E7[6] = r.Etot;
}

void ref_mm_step_npt(double* pos, double* vel, double* F, double* vir9, double* h, double* hi,
                     int na, double dt, double* npt, int nb, int* bi, double* bk, double* br,
                     int nang, int* ai, double* ak, double* at, int nd, int* di, double* dv,
                     int* dm, double* dg, int ni, int* ii, double* ik, double* ig, const int* nlc,
                     const int* nll, const double* charge, int* mol_id, int has_charge, double* out8) {
    FlatTopology t = topo_view(nb, bi, bk, br, nang, ai, ak, at, nd, di, dv, dm, dg, ni, ii, ik, ig, mol_id);
    NPTState s; npt_in(npt, s);
    auto r = step_npt(pos, vel, F, vir9, h, hi, na, dt, s, t, nlc, nll, charge, mol_id, has_charge != 0);
    npt_out(s, npt);
    out8[0] = r.first.Eb; out8[1] = r.first.Ea; out8[2] = r.first.Ed; out8[3] = r.first.Ei;
    out8[4] = r.first.Elj; out8[5] = r.first.Ecoul; out8[6] = r.first.Etot; out8[7] = r.second;
}

// load_cc1 with bonds (MM:160): returns natom, fills coords and sorted bond pairs.
int ref_mm_load_cc1(const char* path, double* coords, int* bonds, int* nbond) {
    MolData md = load_cc1(path);
    for (int i = 0; i < md.natom; i++)
        for (int a = 0; a < 3; a++) coords[3 * i + a] = md.coords[i][a];
    *nbond = (int)md.bonds.size();
    for (size_t b = 0; b < md.bonds.size(); b++) { bonds[2 * b] = md.bonds[b].first; bonds[2 * b + 1] = md.bonds[b].second; }
    return md.natom;
}
}
