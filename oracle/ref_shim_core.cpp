// ref_shim_core.cpp -- extern "C" access to the unmodified reference core
// (serial-only) rigid-body LJ program.  REF_SRC is set by oracle/Makefile;
// main() is renamed to ref_main.  TEST INFRASTRUCTURE ONLY.
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
double ref_core_rmcut() { return RMCUT; }
// generate_c60 (CORE:228): coords[180]; rd = {I0, Mmol, Rmol}
void ref_core_generate_c60(double* coords, double* rd) {
    C60Data d = generate_c60();
    for (int i = 0; i < 180; i++) coords[i] = d.coords[i];
    rd[0] = d.I0; rd[1] = d.Mmol; rd[2] = d.Rmol;
}
int ref_core_make_fcc(double a, int nc, double* pos, double* h) { return make_fcc(a, nc, pos, h); }
void ref_core_nlist_build_sym(const double* pos, const double* h, const double* hi, int n,
                              int* cnt, int* list) {
    nlist_build_sym(pos, h, hi, n, RMCUT, cnt, list);
}
double ref_core_forces(double* F, double* T, double* W9, const double* pos, const double* qv,
                       const double* body, const double* h, const double* hi, const int* cnt,
                       const int* list, int n, double* lab) {
    return forces(F, T, W9, pos, qv, body, h, hi, cnt, list, n, C60_NATOM, RMCUT2, lab);
}
void ref_core_make_npt(double T, double Pe, int n, double* npt) { npt_out(make_npt(T, Pe, n), npt); }
void ref_core_step_npt(double* pos, double* vel, double* qv, double* omg, double* F, double* T,
                       double* W9, double* h, double* hi, const double* body, double i0, double mmol,
                       int n, double dt, double* npt, const int* cnt, const int* list, double* lab,
                       double* out2) {
    NPTState s; npt_in(npt, s);
    auto r = step_npt(pos, vel, qv, omg, F, T, W9, h, hi, body, i0, mmol, n, C60_NATOM, RMCUT2, dt,
                      s, cnt, list, lab);
    npt_out(s, npt);
    out2[0] = r.first; out2[1] = r.second;
}
}
