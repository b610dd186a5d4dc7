// Writes the same frames with write_ovito_* and with OvitoWriter (several
// formatting threads, more frames than slots) into two files given on the
// command line; the test compares them byte for byte.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fmd_host.hpp"

using namespace fmdh;

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    const int threads = std::atoi(argv[3]);
    FILE* a = std::fopen(argv[1], "w");
    FILE* b = std::fopen(argv[2], "w");
    if (!a || !b) return 3;
    const int n = 3000, natom = 60, na = 20000;
    std::vector<double> pos(3 * na), vel(3 * na), qv(4 * n), body(3 * natom), h(9, 0.0);
    std::vector<int> mol(na);
    for (int i = 0; i < 3 * na; i++) {
        pos[i] = 50.0 * std::sin(0.37 * i) + 1e-3 * i;
        vel[i] = 1e-3 * std::cos(1.3 * i);
    }
    for (int i = 0; i < n; i++) {
        const double w = std::cos(0.1 * i), x = std::sin(0.1 * i) * 0.6, y = std::sin(0.1 * i) * 0.48,
                     z = std::sin(0.1 * i) * 0.64;
        qv[4 * i] = w; qv[4 * i + 1] = x; qv[4 * i + 2] = y; qv[4 * i + 3] = z;
    }
    for (int k = 0; k < 3 * natom; k++) body[k] = 3.5 * std::sin(0.71 * k + 0.2);
    for (int i = 0; i < na; i++) mol[i] = i / 60;
    h[0] = 70.1; h[4] = 70.2; h[8] = 70.3; h[1] = 0.01;
    {
        OvitoWriter w(b, threads);
        for (int f = 0; f < 5; f++) {
            for (int i = 0; i < 3 * na; i++) pos[i] += 0.01;         // the caller's arrays change after each call
            write_ovito_atoms(a, 100 * f, 0.5, pos.data(), vel.data(), mol.data(), f % 2, h.data(), na);
            w.atoms(100 * f, 0.5, pos.data(), vel.data(), mol.data(), f % 2, h.data(), na);
            write_ovito_rigid(a, 100 * f + 1, 1.0, pos.data(), vel.data(), qv.data(), body.data(), h.data(), n, natom);
            w.rigid(100 * f + 1, 1.0, pos.data(), vel.data(), qv.data(), body.data(), h.data(), n, natom);
        }
        w.rigid(7, 1.0, pos.data(), vel.data(), qv.data(), body.data(), h.data(), 1, natom);   // one molecule
        write_ovito_rigid(a, 7, 1.0, pos.data(), vel.data(), qv.data(), body.data(), h.data(), 1, natom);
        w.finish();
    }
    std::fclose(a);
    std::fclose(b);
    return 0;
}
