// ref_shim_lj.cpp -- extern "C" access to the unmodified reference rigid-body
// LJ program (full version).  REF_SRC is set by oracle/Makefile; main() is
// renamed to ref_main.  TEST INFRASTRUCTURE ONLY.
#include REF_SRC

namespace {
void npt_in(const double* a, NPTState& s) {
    s.xi = a[0]; s.Q = a[1];
    for (int k = 0; k < 9; k++) s.Vg[k] = a[2 + k];
    s.W = a[11]; s.Pe = a[12]; s.Tt = a[13]; s.Nf = (int)a[14];
}
void npt_out(const NPTState& s, double* a) {
    a[0] = s.xi; a[1] = s.Q;
    for (int k = 0; k < 9; k++) a[2 + k] = s.Vg[k];
    a[11] = s.W; a[12] = s.Pe; a[13] = s.Tt; a[14] = s.Nf;
}
}  // namespace

extern "C" {
int ref_lj_max_neigh() { return MAX_NEIGH; }
void ref_lj_mat_inv9(const double* h, double* hi) { mat_inv9(h, hi); }
void ref_lj_apply_pbc(double* pos, const double* h, const double* hi, int n) { apply_pbc(pos, h, hi, n); }
void ref_lj_nlist_build_sym(const double* pos, const double* h, const double* hi, int n,
                            double rmcut, int* cnt, int* list) {
    nlist_build_sym(pos, h, hi, n, rmcut, cnt, list);
}
double ref_lj_forces(double* F, double* T, double* W9, const double* pos, const double* qv,
                     const double* body, const double* h, const double* hi, const int* cnt,
                     const int* list, int n, int natom, double rmcut2, double* lab) {
    return forces(F, T, W9, pos, qv, body, h, hi, cnt, list, n, natom, rmcut2, lab);
}
void ref_lj_make_npt(double T, double Pe, int n, double* npt) { npt_out(make_npt(T, Pe, n), npt); }
double ref_lj_ke_trans(const double* vel, int n, double m) { return ke_trans(vel, n, m); }
double ref_lj_ke_rot(const double* omg, int n, double i0) { return ke_rot(omg, n, i0); }
void ref_lj_step_npt(double* pos, double* vel, double* qv, double* omg, double* F, double* T,
                     double* W9, double* h, double* hi, const double* body, double i0, double mmol,
                     int n, int natom, double rmcut2, double dt, double* npt, const int* cnt,
                     const int* list, double* lab, double* out2) {
    NPTState s; npt_in(npt, s);
    auto r = step_npt(pos, vel, qv, omg, F, T, W9, h, hi, body, i0, mmol, n, natom, rmcut2, dt, s,
                      cnt, list, lab);
    npt_out(s, npt);
    out2[0] = r.first; out2[1] = r.second;
}
// load_cc1 (LJ:178): returns natom; rd = {Rmol, Dmol, I0, Mmol}
int ref_lj_load_cc1(const char* path, double* coords, double* rd) {
    MolData md = load_cc1(path);
    for (int i = 0; i < md.natom * 3; i++) coords[i] = md.coords[i];
    rd[0] = md.Rmol; rd[1] = md.Dmol; rd[2] = md.I0; rd[3] = md.Mmol;
    return md.natom;
}
double ref_lj_default_a0(double dmax, const char* st, double s) { return default_a0(dmax, st, s); }
int ref_lj_make_crystal(const char* st, double a, int nc, double* pos, double* h) {
    std::string s(st);
    if (s == "FCC") return make_fcc(a, nc, pos, h);
    if (s == "HCP") return make_hcp(a, nc, pos, h);
    return make_bcc(a, nc, pos, h);
}
// Writes the OVITO frame and restart file exactly as the reference does.
void ref_lj_write_ovito(const char* path, int istep, double dt, const double* pos, const double* vel,
                        const double* qv, const double* body, const double* h, int n, int natom) {
    FILE* fp = fopen(path, "w");
    if (!fp) return;
    write_ovito(fp, istep, dt, pos, vel, qv, body, h, n, natom);
    fclose(fp);
}
void ref_lj_write_restart(const char* path, int istep, int nkv, const char** keys, const char** vals,
                          const char* st, int nc, double T, double Pe, int nsteps, double dt, int seed,
                          const char* fspec, double init_scale, const double* h, const double* npt,
                          const double* pos, const double* qv, const double* vel, const double* omg,
                          int n, int natom) {
    std::map<std::string, std::string> opts;
    for (int k = 0; k < nkv; k++) opts[keys[k]] = vals[k];
    NPTState s; npt_in(npt, s);
    write_restart_lj(path, istep, opts, st, nc, T, Pe, nsteps, dt, seed, fspec, init_scale, h, s,
                     pos, qv, vel, omg, n, natom);
}
// restart_filename / build_suffix / unique_file (LJ:571-588) into a caller buffer.
void ref_lj_restart_filename(const char* oname, int istep, int nsteps, char* out, int cap) {
    std::string r = restart_filename(oname, istep, nsteps);
    snprintf(out, cap, "%s", r.c_str());
}
void ref_lj_build_suffix(int nkv, const char** keys, const char** vals, char* out, int cap) {
    std::map<std::string, std::string> opts;
    for (int k = 0; k < nkv; k++) opts[keys[k]] = vals[k];
    snprintf(out, cap, "%s", build_suffix(opts).c_str());
}
}
