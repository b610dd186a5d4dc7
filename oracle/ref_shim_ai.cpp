// ref_shim_ai.cpp -- exposes the unmodified reference AIREBO program's
// static kernels through extern "C" entry points so tests can call them as
// the parity oracle.  The reference translation unit is included verbatim
// from the path given by the REF_SRC macro (set by oracle/Makefile); its
// main() is renamed to ref_main.  TEST INFRASTRUCTURE ONLY.
#include REF_SRC

namespace {
// NPT state <-> flat array {xi, Q, Vg[9], W, Pe, Tt, Nf}
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
}  // namespace

extern "C" {
void ref_ai_mat_inv9(const double* h, double* hi) { mat_inv9(h, hi); }
void ref_ai_apply_pbc(double* pos, const double* h, const double* hi, int n) { apply_pbc(pos, h, hi, n); }
void ref_ai_build_nlist_rebo(const double* pos, const double* h, const double* hi, int na,
                             const int* mol_id, int* nlc, int* nll) {
    build_nlist_rebo(pos, h, hi, na, mol_id, nlc, nll);
}
void ref_ai_build_nlist_lj(const double* pos, const double* h, const double* hi, int na,
                           const int* mol_id, int* nlc, int* nll) {
    build_nlist_lj(pos, h, hi, na, mol_id, nlc, nll);
}
double ref_ai_compute_rebo(double* F, double* vir9, const double* pos, const double* h,
                           const double* hi, const int* nlc, const int* nll, int na) {
    return compute_rebo(F, vir9, pos, h, hi, nlc, nll, na);
}
double ref_ai_compute_lj(double* F, double* vir9, const double* pos, const double* h,
                         const double* hi, const int* nlc, const int* nll, int na) {
    return compute_lj(F, vir9, pos, h, hi, nlc, nll, na);
}
void ref_ai_compute_forces(double* F, double* vir9, const double* pos, const double* h,
                           const double* hi, const int* nlc_r, const int* nll_r,
                           const int* nlc_l, const int* nll_l, int na, double* E3) {
    ForceResult r = compute_forces(F, vir9, pos, h, hi, nlc_r, nll_r, nlc_l, nll_l, na);
    E3[0] = r.Ep; E3[1] = r.Ep_rebo; E3[2] = r.Ep_lj;
}
void ref_ai_make_npt(double T, double Pe, int na, double* npt) { npt_out(make_npt(T, Pe, na), npt); }
double ref_ai_ke_total(const double* vel, const double* mass, int na) { return ke_total(vel, mass, na); }
void ref_ai_step_npt(double* pos, double* vel, double* F, double* vir9, double* h, double* hi,
                     const double* mass, int na, double dt, double* npt,
                     const int* nlc_r, const int* nll_r, const int* nlc_l, const int* nll_l,
                     double* out4) {
    NPTState s; npt_in(npt, s);
    StepResult r = step_npt(pos, vel, F, vir9, h, hi, mass, na, dt, s, nlc_r, nll_r, nlc_l, nll_l);
    npt_out(s, npt);
    out4[0] = r.Ep; out4[1] = r.Ep_rebo; out4[2] = r.Ep_lj; out4[3] = r.KE;
}
int ref_ai_load_cc1(const char* path, double* coords, int max_atoms, double* rd) {
    MolData md = load_cc1(path);
    for (int i = 0; i < md.natom && i < max_atoms; i++)
        for (int a = 0; a < 3; a++) coords[3 * i + a] = md.coords[i][a];
    rd[0] = md.Rmol; rd[1] = md.Dmol;
    return md.natom;
}
}
