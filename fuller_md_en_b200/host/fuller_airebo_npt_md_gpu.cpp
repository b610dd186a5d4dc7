// fuller_airebo_npt_md_gpu -- drop-in for the reference's AIREBO program
// (fuller_airebo_npt_md_serial_omp_acc.cpp, main at AI:681-963): same options,
// help text, banner/monitor/averages lines, OVITO XYZ, .rst restart files and
// abort.md/stop.md control.  Every MD step (REBO + LJ forces, NPT integrator,
// list rebuilds every 20 steps) runs on the B200 through the device-resident
// system API.
#include <algorithm>
#include <cctype>
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
        "fuller_airebo_npt_md_serial_omp_acc — AIREBO fullerene NPT-MD\n\n"
        "Options:\n"
        "  --help                  Show this help\n"
        "  --fullerene=<name>      Fullerene species (default: C60)\n"
        "  --crystal=<fcc|hcp|bcc> Crystal structure (default: fcc)\n"
        "  --cell=<nc>             Unit cell repeats (default: 3)\n"
        "  --temp=<K>              Target temperature [K] (default: 298.0)\n"
        "  --pres=<GPa>            Target pressure [GPa] (default: 0.0)\n"
        "  --step=<N>              Production steps (default: 10000)\n"
        "  --dt=<fs>               Time step [fs] (default: 0.5)\n"
        "  --init_scale=<s>        Lattice scale factor (default: 1.0)\n"
        "  --seed=<n>              Random seed (default: 42)\n"
        "  --coldstart=<N>         Cold-start steps at 4K (default: 0)\n"
        "  --warmup=<N>            Warm-up ramp steps 4K->T (default: 0)\n"
        "  --from=<step>           Averaging start step (default: auto)\n"
        "  --to=<step>             Averaging end step (default: nsteps)\n"
        "  --mon=<N>               Monitor print interval (default: auto)\n"
        "  --warmup_mon=<mode>     Warmup monitor: norm|freq|some (default: norm)\n"
        "  --ovito=<N>             OVITO XYZ output interval, 0=off (default: 0)\n"
        "  --restart=<N>           Restart save interval, 0=off (default: 0)\n"
        "  --resfile=<path>        Resume from restart file\n"
        "  --libdir=<path>         Fullerene library dir (default: FullereneLib)\n\n"
        "Examples:\n"
        "  ./prog --temp=500 --pres=1.0 --step=50000\n"
        "  ./prog --coldstart=5000 --warmup=5000 --step=20000\n"
        "  ./prog --step=10000 --ovito=100\n"
        "  ./prog --step=50000 --restart=5000\n"
        "  ./prog --resfile=restart_airebo_serial_00025000.rst\n");
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
    const double dt = std::atof(gopt(opts, "dt", "0.5").c_str());
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
    constexpr double T_cold = 4.0;
    int start_step = 0;

    if (avg_to <= 0) avg_to = nsteps;
    if (avg_from <= 0) avg_from = std::max(1, nsteps - nsteps / 4);
    const int total_steps = coldstart + warmup + nsteps;
    const int gavg_from = coldstart + warmup + avg_from, gavg_to = coldstart + warmup + avg_to;

    const auto fl = resolve_fullerene(fspec, libdir, Dialect::AI);
    const Molecule mol = load_cc1(fl.first, Dialect::AI);
    const double a0 = default_a0(mol.Dmol, st, init_scale);
    const int Nmol_max = st == "FCC" ? 4 * nc * nc * nc : 2 * nc * nc * nc;
    const long Na_max = (long)Nmol_max * mol.natom;

    // Device memory check (AI:749-760) with this implementation's footprint per atom.
    char devname[128] = {0};
    double gpu_gb = 0;
    const double bpa = 8.0 * 3 * 5 + 8 + 4 + 4.0 * (1 + 12) + 4.0 * (1 + 400) + 4.0 * (1 + 1024) + 48;
    const double need = Na_max * bpa;
    if (fmd_device_info(0, devname, sizeof(devname), &gpu_gb) == FMD_OK &&
        need > gpu_gb * 1024.0 * 1024.0 * 1024.0 * 0.80) {
        printf("Error: GPU memory insufficient (need %.1f GB, have %.1f GB)\n", need / 1024.0 / 1024.0 / 1024.0,
               gpu_gb);
        return 1;
    }

    std::vector<double> centres(3 * (size_t)Nmol_max);
    double h[9] = {0}, hi[9] = {0};
    const int Nmol = make_crystal(st, a0, nc, centres.data(), h);
    const int Na = Nmol * mol.natom;
    std::vector<double> pos(3 * (size_t)Na), vel(3 * (size_t)Na, 0.0), mass(Na);
    std::vector<int> mol_id(Na);
    for (int m = 0; m < Nmol; m++)                          // AI:781-786
        for (int a = 0; a < mol.natom; a++) {
            const int idx = m * mol.natom + a;
            for (int c = 0; c < 3; c++) pos[3 * idx + c] = centres[3 * m + c] + mol.coords[3 * a + c];
            mass[idx] = MC;
            mol_id[idx] = m + 1;
        }

    printf("========================================================================\n");
    printf("  Fullerene Crystal NPT-MD — AIREBO (CUDA B200)\n");
    printf("========================================================================\n");
    printf("  GPU VRAM        : %.2f GB (need %.2f MB)\n", gpu_gb, need / 1024.0 / 1024.0);
    printf("  Fullerene       : %s (%d atoms/mol)\n", fl.second.c_str(), mol.natom);
    printf("  Crystal         : %s %dx%dx%d  Nmol=%d  Natom=%d\n", st.c_str(), nc, nc, nc, Nmol, Na);
    printf("  a0=%.3f A  T=%.1f K  P=%.4f GPa  dt=%.3f fs\n", a0, T, Pe, dt);
    printf("  Production      : %d steps  avg=%d-%d  Total=%d\n", nsteps, avg_from, avg_to, total_steps);
    printf("========================================================================\n\n");

    mat_inv9(h, hi);
    const double T_init = (coldstart > 0 || warmup > 0) ? T_cold : T;   // AI:808-815
    std::mt19937 rng(seed);
    std::normal_distribution<double> g(0, 1);
    for (int i = 0; i < Na; i++) {
        const double sv = std::sqrt(KB * T_init * CONV / mass[i]);
        for (int a = 0; a < 3; a++) vel[3 * i + a] = sv * g(rng);
    }
    double vcm[3] = {0, 0, 0};
    for (int i = 0; i < Na; i++)
        for (int a = 0; a < 3; a++) vcm[a] += vel[3 * i + a];
    for (int a = 0; a < 3; a++) vcm[a] /= Na;
    for (int i = 0; i < Na; i++)
        for (int a = 0; a < 3; a++) vel[3 * i + a] -= vcm[a];
    fmd_npt npt = make_npt(T, Pe, 3 * Na - 3);
    npt.Tt = T_init;

    if (!resfile.empty()) {                                 // AI:820-828
        Restart rd = read_restart_airebo(resfile);
        if (rd.ok) {
            start_step = rd.istep;
            for (int k = 0; k < 9; k++) h[k] = rd.h[k];
            mat_inv9(h, hi);
            npt = rd.npt;
            for (int i = 0; i < Na && i < rd.n; i++) {
                for (int c = 0; c < 3; c++) { pos[3 * i + c] = rd.pos[3 * i + c]; vel[3 * i + c] = rd.vel[3 * i + c]; }
                mol_id[i] = rd.mol_id[i];
                mass[i] = rd.mass[i];
            }
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
    p.coldstart = coldstart; p.warmup = warmup; p.nsteps = nsteps; p.nlup = 20;   // AI:860
    p.gavg_from = gavg_from; p.gavg_to = gavg_to; p.nc = nc; p.nmol = Nmol;
    p.precision = FMD_PREC_FP64; p.use_graphs = 1;
    fmd_system* sys = nullptr;
    check(ctx, fmd_system_create_airebo(ctx, &p, Na, pos.data(), vel.data(), mass.data(), mol_id.data(), h, &npt, &sys),
          "system set-up");
    // --physics=<fmd_physics bits>: opt-in force-field corrections, no
    // reference counterpart (not in the help text, which is the reference's)
    const int physics = std::atoi(gopt(opts, "physics", "0").c_str());
    if (physics) check(ctx, fmd_system_set_physics(sys, physics), "physics corrections");
    check(ctx, fmd_system_init(sys), "initial lists and forces");   // AI:830-853

    Schedule sc;
    sc.coldstart = coldstart; sc.warmup = warmup; sc.total = total_steps;
    sc.set_monitor(mon_interval, warmup_mon_mode);
    sc.nrec_o = nrec_o; sc.nrec_rst = nrec_rst;
    const double t0 = now_s();
    const std::string ovito_file = unique_file("ovito_traj_airebo_gpu", ".xyz");
    FILE* io_o = nrec_o > 0 ? fopen(ovito_file.c_str(), "w") : nullptr;
    sc.ovito = io_o != nullptr;
    // frames are formatted and written on a writer thread while the steps go on
    std::unique_ptr<OvitoWriter> ovito(io_o ? new OvitoWriter(io_o) : nullptr);
    printf("  %8s %5s %7s %9s %8s %11s %11s %11s %7s\n", "step", "phase", "T[K]", "P[GPa]", "a[A]", "E_REBO",
           "E_LJ", "E_total", "t[s]");
    const std::string rst_base = nrec_o > 0 ? ovito_file : std::string("restart_airebo_gpu");

    RunInfo ri;
    ri.st = st; ri.fspec = fspec; ri.nc = nc; ri.nsteps = nsteps; ri.seed = seed;
    ri.T = T; ri.Pe = Pe; ri.dt = dt; ri.init_scale = init_scale;
    // checkpoints are formatted and written on a writer thread from copies
    std::unique_ptr<RestartWriter> rstw(nrec_rst > 0 ? new RestartWriter() : nullptr);
    auto save = [&](int s) {
        check(ctx, fmd_system_download(sys, pos.data(), vel.data(), nullptr, nullptr, h, &npt), "download");
        // h (a C array) and the vectors are captured by copy
        rstw->submit([fn = restart_filename(rst_base, s, total_steps), s, opts, ri, h, npt, p = pos, v = vel,
                      mid = mol_id, m = mass, Na, Nmol, natom = mol.natom]() {
            write_restart_airebo(fn, s, opts, ri, h, npt, p.data(), v.data(), mid.data(), m.data(), Na, Nmol, natom);
        });
    };
    bool stop_requested = false;
    for (int gs = start_step + 1; gs <= total_steps;) {
        const int e = sc.next_event(gs);
        fmd_obs o;
        check(ctx, fmd_system_run(sys, gs, e, &o), "MD steps");
        if (sc.ovito_at(e)) {
            check(ctx, fmd_system_download(sys, pos.data(), vel.data(), nullptr, nullptr, h, nullptr), "download");
            ovito->atoms(e, dt, pos.data(), vel.data(), mol_id.data(), 0, h, Na);
        }
        if (sc.restart_at(e)) {
            save(e);
            if (stop_requested) {
                printf("\n  *** Stopped at restart checkpoint (global step %d) ***\n", e);
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
                if (nrec_rst == 0) break;                   // AI:946
            }
            printf("  %8d %5s %7.1f %9.3f %8.3f %11.4f %11.4f %11.4f %7.0f\n", e, sc.phase(e), o.T, o.P, o.a,
                   o.E[1] / Nmol, o.E[2] / Nmol, o.E[0] / Nmol, elapsed_since(t0));
        }
        gs = e + 1;
    }
    ovito.reset();                          // every frame written
    rstw.reset();                           // every checkpoint written
    if (io_o) fclose(io_o);
    fmd_avg av;
    check(ctx, fmd_system_averages(sys, &av), "averages");
    if (av.n > 0)
        printf("\n  Averages (%d): T=%.2f P=%.4f a=%.4f REBO=%.4f LJ=%.4f Total=%.4f\n", av.n, av.sT / av.n,
               av.sP / av.n, av.sa / av.n, av.sE[0] / av.n, av.sE[1] / av.n, av.sE[2] / av.n);
    printf("  Done (%.1f sec)\n", elapsed_since(t0));
    fmd_system_destroy(sys);
    fmd_ctx_destroy(ctx);
    return 0;
}
