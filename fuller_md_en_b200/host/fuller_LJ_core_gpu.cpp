// fuller_LJ_core_gpu -- drop-in for the reference's benchmark core program
// (fuller_LJ_npt_md_core_serial_omp_acc.cpp, main at CORE:651-823): rigid C60
// FCC crystal, nc from `--cell=` or the first positional argument (1-8),
// 1000 NPT steps at 300 K / 0 GPa / dt 1 fs, monitor every 100 steps,
// averages over steps 750-1000, same banner/monitor/"Avg(...)"/"Done" lines.
// All steps run on the B200 as device-resident graphs of the rigid system.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "drv.hpp"

using namespace fmdh;

int main(int argc, char** argv) {
    int nc = 3;
    std::string prec = "fp64";
    for (int i = 1; i < argc; i++) {                       // CORE:653-658
        const std::string a = argv[i];
        if (a.substr(0, 7) == "--cell=") nc = std::atoi(a.substr(7).c_str());
        else if (a.substr(0, 16) == "--gpu_precision=") prec = a.substr(16);
        else if (a[0] != '-') nc = std::atoi(argv[i]);
    }
    if (nc < 1 || nc > 8) {
        printf("Error: nc must be 1-8 (got %d)\n", nc);
        return 1;
    }
    constexpr int nsteps = 1000, mon = 100, nlup = 25, max_neigh = 80, natom = 60;
    constexpr double T = 300.0, Pe = 0.0, dt = 1.0, a0 = 14.17;
    constexpr double sigma = 3.431, RCUT = 3.0 * sigma, RC60 = 3.55, RMCUT = RCUT + 2 * RC60 + 1.0;
    const int avg_from = nsteps - nsteps / 4;

    std::vector<double> body(3 * natom);
    double I0 = 0, Mmol = 0, Rmol = 0;
    generate_c60(body.data(), &I0, &Mmol, &Rmol);
    const int Nmax = 4 * nc * nc * nc;
    std::vector<double> pos(3 * (size_t)Nmax), vel(3 * (size_t)Nmax, 0.0), omg(3 * (size_t)Nmax, 0.0),
        qv(4 * (size_t)Nmax, 0.0);
    double h[9] = {0};
    const int N = make_crystal("FCC", a0, nc, pos.data(), h);

    printf("================================================================\n");
    printf("  C60 LJ NPT-MD Core (CUDA B200)\n");
    printf("================================================================\n");
    printf("  GPU devices     : %d\n", 1);
    printf("  Active device   : %d (NVIDIA)\n", 0);
    printf("  FCC cell        : %dx%dx%d  N=%d molecules\n", nc, nc, nc, N);
    printf("  Atoms/molecule  : %d\n", natom);
    printf("  a0=%.2f A  T=%.0f K  P=%.1f GPa  dt=%.1f fs  steps=%d\n", a0, T, Pe, dt, nsteps);
    printf("  MAX_NEIGH=%d  VECTOR_LENGTH=%d\n", max_neigh, 128);
    const double mem_lab = (double)N * natom * 3 * 8 / 1024 / 1024;
    const double mem_nl = (double)N * max_neigh * 4 / 1024 / 1024;
    const double mem_total = (double)(N * 3 * 8 * 5 + N * 4 * 8 + N * natom * 3 * 8 + natom * 3 * 8 + N * 4 +
                                      N * max_neigh * 4 + 9 * 8 * 3) / 1024 / 1024;
    printf("  Memory          : lab=%.2f MB  nl=%.2f MB  total=%.2f MB\n", mem_lab, mem_nl, mem_total);
    printf("================================================================\n\n");

    std::mt19937 rng(42);                                  // CORE:725-739
    std::normal_distribution<double> gauss(0, 1);
    const double sv = std::sqrt(KB * T * CONV / Mmol), sw = std::sqrt(KB * T * CONV / I0);
    for (int i = 0; i < N; i++) {
        for (int a = 0; a < 3; a++) {
            vel[3 * i + a] = sv * gauss(rng);
            omg[3 * i + a] = sw * gauss(rng);
        }
        for (int a = 0; a < 4; a++) qv[4 * i + a] = gauss(rng);
        const double n = std::sqrt(qv[4 * i] * qv[4 * i] + qv[4 * i + 1] * qv[4 * i + 1] +
                                   qv[4 * i + 2] * qv[4 * i + 2] + qv[4 * i + 3] * qv[4 * i + 3]);
        for (int a = 0; a < 4; a++) qv[4 * i + a] /= n;
    }
    double vcm[3] = {0, 0, 0};
    for (int i = 0; i < N; i++)
        for (int a = 0; a < 3; a++) vcm[a] += vel[3 * i + a];
    for (int a = 0; a < 3; a++) vcm[a] /= N;
    for (int i = 0; i < N; i++)
        for (int a = 0; a < 3; a++) vel[3 * i + a] -= vcm[a];
    const fmd_npt npt = make_npt(T, Pe, 6 * N - 3);

    fmd_ctx* ctx = nullptr;
    const int rc = fmd_ctx_create(&ctx, 0);
    if (rc != FMD_OK) {
        fprintf(stderr, "Error: no usable CUDA device (%s)\n", fmd_status_string(rc));
        return 1;
    }
    fmd_run_params p{};
    p.dt = dt; p.T = T; p.Pe = Pe; p.T_cold = 4.0;
    p.coldstart = 0; p.warmup = 0; p.nsteps = nsteps; p.nlup = nlup;
    p.gavg_from = avg_from; p.gavg_to = nsteps; p.nc = nc; p.nmol = N;
    p.precision = prec == "fp32" ? FMD_PREC_FP32_PAIR : FMD_PREC_FP64;
    p.use_graphs = 1;
    fmd_system* sys = nullptr;
    check(ctx, fmd_system_create_rigid(ctx, &p, N, natom, body.data(), I0, Mmol, RMCUT, max_neigh, pos.data(),
                                       vel.data(), qv.data(), omg.data(), h, &npt, &sys),
          "system set-up");
    check(ctx, fmd_system_init(sys), "initial lists and forces");   // CORE:758-770

    const double t0 = now_s();
    printf("%8s %7s %9s %8s %10s %7s\n", "step", "T[K]", "P[GPa]", "a[A]", "Ecoh[eV]", "t[s]");
    for (int g = 1; g <= nsteps;) {
        const int e = std::min(nsteps, ((g + mon - 1) / mon) * mon);
        fmd_obs o;
        check(ctx, fmd_system_run(sys, g, e, &o), "MD steps");
        printf("%8d %7.1f %9.3f %8.3f %10.5f %7.0f\n", e, o.T, o.P, o.a, o.E[0] / N, elapsed_since(t0));
        g = e + 1;
    }
    fmd_avg av;
    check(ctx, fmd_system_averages(sys, &av), "averages");
    if (av.n > 0)
        printf("Avg(%d): T=%.2f P=%.4f a=%.4f Ecoh=%.5f\n", av.n, av.sT / av.n, av.sP / av.n, av.sa / av.n,
               av.sE[0] / av.n);
    printf("Done %.1fs\n", elapsed_since(t0));
    fmd_system_destroy(sys);
    fmd_ctx_destroy(ctx);
    return 0;
}
