// Writes the same checkpoints of the three programs with write_restart_* on
// the caller's thread into directory argv[1] and through RestartWriter jobs
// (which own copies of the state, while the caller's arrays keep changing)
// into directory argv[2]; the test compares the files byte for byte.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "fmd_host.hpp"

using namespace fmdh;

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const std::string da = argv[1], db = argv[2];
    const int n = 500, natom = 60, na = n * natom;
    std::vector<double> pos(3 * na), vel(3 * na), qv(4 * n), omg(3 * n), mass(na, 12.011);
    std::vector<int> mol(na);
    double h[9] = {70.1, 0.0, 0.0, 0.0, 70.2, 0.0, 0.0, 0.0, 70.3};
    fmd_npt npt{};
    npt.xi = 1e-3; npt.Q = 2.5; npt.W = 7.5; npt.Pe = 0.1; npt.Tt = 300.0; npt.Nf = 3 * na - 3;
    for (int k = 0; k < 9; k++) npt.Vg[k] = 1e-5 * k;
    for (int i = 0; i < 3 * na; i++) {
        pos[i] = 50.0 * std::sin(0.37 * i) + 1e-3 * i;
        vel[i] = 1e-3 * std::cos(1.3 * i);
    }
    for (int i = 0; i < 4 * n; i++) qv[i] = std::cos(0.01 * i);
    for (int i = 0; i < 3 * n; i++) omg[i] = 1e-4 * std::sin(0.2 * i);
    for (int i = 0; i < na; i++) mol[i] = i / natom + 1;
    Opts o;
    o["cell"] = "5";
    o["restart"] = "10";
    RunInfo ri;
    ri.st = "FCC"; ri.fspec = "C60"; ri.nc = 5; ri.nsteps = 40; ri.seed = 42; ri.T = 300; ri.Pe = 0.1; ri.dt = 0.5;
    ri.init_scale = 1.0;
    {
        RestartWriter w;
        for (int s = 10; s <= 40; s += 10) {
            for (int i = 0; i < 3 * na; i++) pos[i] += 0.01;        // the state moves between checkpoints
            npt.xi += 1e-4;
            h[0] += 0.001;
            const std::string fa = da + "/c" + std::to_string(s), fb = db + "/c" + std::to_string(s);
            write_restart_lj(fa + "_lj.rst", s, o, ri, h, npt, pos.data(), qv.data(), vel.data(), omg.data(), n, natom);
            write_restart_airebo(fa + "_ai.rst", s, o, ri, h, npt, pos.data(), vel.data(), mol.data(), mass.data(), na,
                                 n, natom);
            write_restart_mmmd(fa + "_mm.rst", s, o, ri, h, npt, pos.data(), vel.data(), na, n, natom);
            w.submit([fb, s, o, ri, h, npt, p = pos, q = qv, v = vel, m = omg, n, natom]() {
                write_restart_lj(fb + "_lj.rst", s, o, ri, h, npt, p.data(), q.data(), v.data(), m.data(), n, natom);
            });
            w.submit([fb, s, o, ri, h, npt, p = pos, v = vel, mid = mol, ms = mass, na, n, natom]() {
                write_restart_airebo(fb + "_ai.rst", s, o, ri, h, npt, p.data(), v.data(), mid.data(), ms.data(), na,
                                     n, natom);
            });
            w.submit([fb, s, o, ri, h, npt, p = pos, v = vel, na, n, natom]() {
                write_restart_mmmd(fb + "_mm.rst", s, o, ri, h, npt, p.data(), v.data(), na, n, natom);
            });
        }
        w.finish();
    }
    return 0;
}
