// fuller_LJ_npt_md_gpu -- drop-in for the reference's rigid-body LJ program
// (fuller_LJ_npt_md_serial_omp_acc.cpp, main at LJ:638-953): same options,
// help text, banner/monitor/averages lines, OVITO XYZ, .rst restart files and
// abort.md/stop.md control.  Every MD step runs on the B200 through the
// device-resident system API (libfullermd_cuda.so); the host wakes only at
// monitor, OVITO and restart steps.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "drv.hpp"

using namespace fmdh;

static void usage() {
    printf(
        "fuller_LJ_npt_md_serial_omp_acc — LJ rigid-body fullerene NPT-MD\n\n"
        "Options:\n"
        "  --help                  Show this help\n"
        "  --fullerene=<name>      Fullerene species (default: C60)\n"
        "  --crystal=<fcc|hcp|bcc> Crystal structure (default: fcc)\n"
        "  --cell=<nc>             Unit cell repeats (default: 3)\n"
        "  --temp=<K>              Target temperature [K] (default: 298.0)\n"
        "  --pres=<GPa>            Target pressure [GPa] (default: 0.0)\n"
        "  --step=<N>              Production steps (default: 10000)\n"
        "  --dt=<fs>               Time step [fs] (default: 1.0)\n"
        "  --init_scale=<s>        Lattice scale factor (default: 1.0)\n"
        "  --seed=<n>              Random seed (default: 42)\n"
        "  --coldstart=<N>         Cold-start steps at 4K (default: 0)\n"
        "  --warmup=<N>            Warm-up ramp steps 4K->T (default: 0)\n"
        "  --from=<step>           Averaging start step (default: auto)\n"
        "  --to=<step>             Averaging end step (default: nsteps)\n"
        "  --mon=<N>               Monitor print interval (default: auto)\n"
        "  --warmup_mon=<mode>     Warmup monitor: norm|freq|some (default: norm)\n"
        "  --ovito=<N>             OVITO XYZ output interval, 0=off (default: 0)\n"
        "  --ofile=<filename>      OVITO output filename (default: auto)\n"
        "  --restart=<N>           Restart save interval, 0=off (default: 0)\n"
        "  --resfile=<path>        Resume from restart file\n"
        "  --libdir=<path>         Fullerene library dir (default: FullereneLib)\n\n"
        "Examples:\n"
        "  ./prog --temp=500 --pres=1.0 --step=50000\n"
        "  ./prog --coldstart=2000 --warmup=3000 --step=20000\n"
        "  ./prog --step=10000 --ovito=100\n"
        "  ./prog --step=50000 --restart=5000\n"
        "  ./prog --resfile=restart_LJ_serial_00010000.rst\n");
}

int main(int argc, char** argv) {
    const Opts opts = parse_args(argc, argv);
    if (opts.count("help")) {
        usage();
        return 0;
    }
    std::string st = gopt(opts, "crystal", "fcc");
    for (char& c : st) c = (char)std::toupper((unsigned char)c);
    const int nc = std::atoi(gopt(opts, "cell", "3").c_str());
    const double T = std::atof(gopt(opts, "temp", "298.0").c_str());
    const double Pe = std::atof(gopt(opts, "pres", "0.0").c_str());
    const int nsteps = std::atoi(gopt(opts, "step", "10000").c_str());
    const double dt = std::atof(gopt(opts, "dt", "1.0").c_str());
    const int seed = std::atoi(gopt(opts, "seed", "42").c_str());
    const double init_scale = std::atof(gopt(opts, "init_scale", "1.0").c_str());
    const std::string fspec = gopt(opts, "fullerene", "C60");
    const std::string libdir = gopt(opts, "libdir", "FullereneLib");
    const int coldstart = std::atoi(gopt(opts, "coldstart", "0").c_str());
    const int warmup = std::atoi(gopt(opts, "warmup", "0").c_str());
    int avg_from = std::atoi(gopt(opts, "from", "0").c_str());
    int avg_to = std::atoi(gopt(opts, "to", "0").c_str());
    const int nrec_o = std::atoi(gopt(opts, "ovito", "0").c_str());
    const int nrec_rst = std::atoi(gopt(opts, "restart", "0").c_str());
    const std::string resfile = gopt(opts, "resfile", "");
    const int mon_interval = std::atoi(gopt(opts, "mon", "0").c_str());
    const std::string warmup_mon_mode = gopt(opts, "warmup_mon", "norm");
    const int prec = gopt(opts, "gpu_precision", "fp64") == "fp32" ? FMD_PREC_FP32_PAIR : FMD_PREC_FP64;
    constexpr double T_cold = 4.0;
    int start_step = 0;

    if (avg_to <= 0) avg_to = nsteps;
    if (avg_from <= 0) avg_from = std::max(1, nsteps - nsteps / 4);
    const int total_steps = coldstart + warmup + nsteps;
    const int gavg_from = coldstart + warmup + avg_from, gavg_to = coldstart + warmup + avg_to;
    if (avg_from < 1 || avg_from >= avg_to || avg_to > nsteps) {
        fprintf(stderr, "Error: invalid --from/--to range\n");
        return 1;
    }
    const std::string sfx = build_suffix(opts);
    const std::string ovito_file =
        opts.count("ofile") ? gopt(opts, "ofile", "") : unique_file("ovito_traj_LJ_gpu" + sfx, ".xyz");

    const auto fl = resolve_fullerene(fspec, libdir, Dialect::LJ);
    const Molecule mol = load_cc1(fl.first, Dialect::LJ);
    const int natom = mol.natom;
    const double RCUT = 3.0 * 3.431;
    const double RMCUT = RCUT + 2 * mol.Rmol + 1.0;       // LJ:716
    const double a0 = default_a0(mol.Dmol, st, init_scale);
    const int Nmax = st == "FCC" ? 4 * nc * nc * nc : 2 * nc * nc * nc;

    // Device memory check (LJ:726-738), with this implementation's per-molecule footprint.
    char devname[128] = {0};
    double gpu_gb = 0;
    int nc_max_gpu = 9999;
    if (fmd_device_info(0, devname, sizeof(devname), &gpu_gb) == FMD_OK) {
        const double bpm = 8.0 * (3 * 7 + 4) + 4.0 * (1 + 80) + 8.0 * 10 + 64;   // state, lists, partials, cells
        const double usable = gpu_gb * 1024.0 * 1024.0 * 1024.0 * 0.80;
        nc_max_gpu = (int)std::cbrt(usable / bpm / (st == "FCC" ? 4.0 : 2.0));
    }
    if (nc > nc_max_gpu) {
        printf("Error: nc=%d exceeds GPU memory (max nc=%d for %.1f GB)\n", nc, nc_max_gpu, gpu_gb);
        return 1;
    }

    std::vector<double> pos(3 * (size_t)Nmax, 0.0), vel(3 * (size_t)Nmax, 0.0), omg(3 * (size_t)Nmax, 0.0),
        qv(4 * (size_t)Nmax, 0.0);
    double h[9] = {0}, hi[9] = {0};
    const int N = make_crystal(st, a0, nc, pos.data(), h);
    mat_inv9(h, hi);

    printf("========================================================================\n");
    printf("  Fullerene Crystal NPT-MD — LJ rigid-body (CUDA B200)\n");
    printf("========================================================================\n");
    device_banner(0);
    printf("  Fullerene       : %s (%d atoms/mol)\n", fl.second.c_str(), natom);
    printf("  Crystal         : %s %dx%dx%d  Nmol=%d\n", st.c_str(), nc, nc, nc, N);
    printf("  a0=%.3f A  T=%.1f K  P=%.4f GPa  dt=%.2f fs\n", a0, T, Pe, dt);
    if (coldstart > 0) printf("  Coldstart       : %d steps at %.1f K\n", coldstart, T_cold);
    if (warmup > 0) printf("  Warmup          : %d steps (%.1fK->%.1fK)\n", warmup, T_cold, T);
    printf("  Production      : %d steps  avg=%d-%d\n", nsteps, avg_from, avg_to);
    printf("  Total           : %d steps\n", total_steps);
    printf("========================================================================\n\n");

    // Initial velocities, angular velocities and orientations (LJ:790-801).
    const double T_init = (coldstart > 0 || warmup > 0) ? T_cold : T;
    std::mt19937 rng(seed);
    std::normal_distribution<double> gauss(0, 1);
    const double sv = std::sqrt(KB * T_init * CONV / mol.Mmol), sw = std::sqrt(KB * T_init * CONV / mol.I0);
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

    fmd_npt npt = make_npt(T, Pe, 6 * N - 3);
    npt.Tt = T_init;

    if (!resfile.empty()) {                                 // LJ:805-811
        Restart rd = read_restart_lj(resfile);
        if (rd.ok) {
            start_step = rd.istep;
            for (int k = 0; k < 9; k++) h[k] = rd.h[k];
            npt = rd.npt;
            const int nn = std::min(N, rd.n);
            for (int i = 0; i < nn * 3; i++) { pos[i] = rd.pos[i]; vel[i] = rd.vel[i]; omg[i] = rd.omg[i]; }
            for (int i = 0; i < nn * 4; i++) qv[i] = rd.qv[i];
            printf("  Restarting from global step %d\n", start_step);
        }
    }

    fmd_ctx* ctx = nullptr;
    int rc = fmd_ctx_create(&ctx, 0);
    if (rc != FMD_OK) {
        fprintf(stderr, "Error: no usable CUDA device (%s)\n", fmd_status_string(rc));
        return 1;
    }
    fmd_run_params p{};
    p.dt = dt; p.T = T; p.Pe = Pe; p.T_cold = T_cold;
    p.coldstart = coldstart; p.warmup = warmup; p.nsteps = nsteps; p.nlup = 25;   // LJ:835
    p.gavg_from = gavg_from; p.gavg_to = gavg_to; p.nc = nc; p.nmol = N;
    p.precision = prec; p.use_graphs = 1;
    fmd_system* sys = nullptr;
    check(ctx, fmd_system_create_rigid(ctx, &p, N, natom, mol.coords.data(), mol.I0, mol.Mmol, RMCUT, 80, pos.data(),
                                       vel.data(), qv.data(), omg.data(), h, &npt, &sys),
          "system set-up");
    // --physics=<fmd_physics bits>: opt-in force-field corrections, no
    // reference counterpart (not in the help text, which is the reference's)
    const int physics = std::atoi(gopt(opts, "physics", "0").c_str());
    if (physics) check(ctx, fmd_system_set_physics(sys, physics), "physics corrections");
    check(ctx, fmd_system_init(sys), "initial lists and forces");   // LJ:813-828

    Schedule sc;
    sc.coldstart = coldstart; sc.warmup = warmup; sc.total = total_steps;
    sc.set_monitor(mon_interval, warmup_mon_mode);
    sc.nrec_o = nrec_o; sc.nrec_rst = nrec_rst;
    const double t0 = now_s();
    FILE* io_o = nrec_o > 0 ? fopen(ovito_file.c_str(), "w") : nullptr;
    sc.ovito = io_o != nullptr;
    // frames are formatted and written on a writer thread while the steps go on
    std::unique_ptr<OvitoWriter> ovito(io_o ? new OvitoWriter(io_o) : nullptr);
    printf("  %8s %5s %7s %9s %8s %10s %13s %7s\n", "step", "phase", "T[K]", "P[GPa]", "a[A]", "Ecoh[eV]",
           "Ecoh[kcal/m]", "t[s]");

    RunInfo ri;
    ri.st = st; ri.fspec = fspec; ri.nc = nc; ri.nsteps = nsteps; ri.seed = seed;
    ri.T = T; ri.Pe = Pe; ri.dt = dt; ri.init_scale = init_scale;
    // checkpoints are formatted and written on a writer thread from copies
    std::unique_ptr<RestartWriter> rstw(nrec_rst > 0 ? new RestartWriter() : nullptr);
    auto save = [&](int g) {
        check(ctx, fmd_system_download(sys, pos.data(), vel.data(), qv.data(), omg.data(), h, &npt), "download");
        // h (a C array) and the vectors are captured by copy
        rstw->submit([fn = restart_filename(ovito_file, g, total_steps), g, opts, ri, h, npt, p = pos, q = qv, v = vel,
                      w = omg, N, natom]() {
            write_restart_lj(fn, g, opts, ri, h, npt, p.data(), q.data(), v.data(), w.data(), N, natom);
        });
    };
    bool stop_requested = false;
    for (int g = start_step + 1; g <= total_steps;) {
        const int e = sc.next_event(g);
        fmd_obs o;
        check(ctx, fmd_system_run(sys, g, e, &o), "MD steps");
        const double Ec = o.E[0] / N, an = o.a;
        if (sc.ovito_at(e)) {
            check(ctx, fmd_system_download(sys, pos.data(), vel.data(), qv.data(), nullptr, h, nullptr), "download");
            ovito->rigid(e, dt, pos.data(), vel.data(), qv.data(), mol.coords.data(), h, N, natom);
        }
        if (sc.restart_at(e)) {
            save(e);
            if (stop_requested) {
                printf("\n  *** Stopped at restart checkpoint (step %d) ***\n", e);
                break;
            }
        }
        if (sc.monitor(e)) {
            if (dir_exists("abort.md")) {
                printf("\n  *** abort.md detected at step %d ***\n", e);
                if (nrec_rst > 0) save(e);
                break;
            }
            if (!stop_requested && dir_exists("stop.md")) {
                stop_requested = true;
                printf("\n  *** stop.md detected at step %d — will stop at next checkpoint ***\n", e);
            }
            printf("  %8d %5s %7.1f %9.3f %8.3f %10.5f %13.4f %7.0f\n", e, sc.phase(e), o.T, o.P, an, Ec,
                   Ec * EV2KCAL, elapsed_since(t0));
        }
        g = e + 1;
    }
    ovito.reset();                          // every frame written
    rstw.reset();                           // every checkpoint written
    if (io_o) fclose(io_o);
    fmd_avg av;
    check(ctx, fmd_system_averages(sys, &av), "averages");
    if (av.n > 0) {
        printf("\n========================================================================\n");
        printf("  Averages (%d samples): T=%.2f K  P=%.4f GPa  a=%.4f A  Ecoh=%.5f eV\n", av.n, av.sT / av.n,
               av.sP / av.n, av.sa / av.n, av.sE[0] / av.n);
        printf("========================================================================\n");
    }
    printf("  Done (%.1f sec)\n", elapsed_since(t0));
    fmd_system_destroy(sys);
    fmd_ctx_destroy(ctx);
    return 0;
}
