// fuller_LJ_npt_mmmd_gpu -- drop-in for the reference's MM force-field program
// (fuller_LJ_npt_mmmd_serial_omp_acc.cpp, main at MM:979-1291): same options,
// help text, topology/banner/monitor/averages lines, OVITO XYZ, .rst restart
// files and abort.md/stop.md control.  Bonded terms, intermolecular LJ, the
// NPT integrator and list rebuilds every 20 steps run on the B200.
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
        "fuller_LJ_npt_mmmd_serial_omp_acc — MM+LJ fullerene NPT-MD\n\n"
        "Options:\n"
        "  --help                  Show this help\n"
        "  --fullerene=<name>      Fullerene species (default: C60)\n"
        "  --crystal=<fcc|hcp|bcc> Crystal structure (default: fcc)\n"
        "  --cell=<nc>             Unit cell repeats (default: 3)\n"
        "  --temp=<K>              Target temperature [K] (default: 298.0)\n"
        "  --pres=<GPa>            Target pressure [GPa] (default: 0.0)\n"
        "  --step=<N>              Production steps (default: 10000)\n"
        "  --dt=<fs>               Time step [fs] (default: 0.1)\n"
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
        "  --libdir=<path>         Fullerene library dir (default: FullereneLib)\n"
        "  --ff_kb=<kcal/mol>      Bond stretch constant (default: 469.0)\n"
        "  --ff_kth=<kcal/mol>     Angle bend constant (default: 63.0)\n"
        "  --ff_v2=<kcal/mol>      Dihedral constant (default: 14.5)\n"
        "  --ff_kimp=<kcal/mol>    Improper constant (default: 15.0)\n\n"
        "Examples:\n"
        "  ./prog --temp=500 --pres=1.0 --step=100000\n"
        "  ./prog --coldstart=5000 --warmup=5000 --step=50000\n"
        "  ./prog --step=20000 --ovito=200\n"
        "  ./prog --step=100000 --restart=10000\n"
        "  ./prog --resfile=restart_mmmd_serial_00050000.rst\n"
        "  ./prog --ff_kb=500 --ff_kth=70 --step=20000\n");
}

int main(int argc, char** argv) {
    const Opts opts = parse_args(argc, argv);
    if (opts.count("help")) {
        usage();
        return 0;
    }
    constexpr double kcal2eV = 1.0 / EV2KCAL;
    std::string st = gopt(opts, "crystal", "fcc");
    for (char& c : st) c = (char)std::toupper((unsigned char)c);
    const int nc = std::atoi(gopt(opts, "cell", "3").c_str());
    const double T = std::atof(gopt(opts, "temp", "298.0").c_str());
    const double Pe = std::atof(gopt(opts, "pres", "0.0").c_str());
    const int nsteps = std::atoi(gopt(opts, "step", "10000").c_str());
    const double dt = std::atof(gopt(opts, "dt", "0.1").c_str());
    const int seed = std::atoi(gopt(opts, "seed", "42").c_str());
    const double init_scale = std::atof(gopt(opts, "init_scale", "1.0").c_str());
    const std::string fspec = gopt(opts, "fullerene", "C60");
    const std::string libdir = gopt(opts, "libdir", "FullereneLib");
    const int coldstart = std::atoi(gopt(opts, "coldstart", "0").c_str());
    const int warmup = std::atoi(gopt(opts, "warmup", "0").c_str());
    int avg_from = std::atoi(gopt(opts, "from", "0").c_str());
    int avg_to = std::atoi(gopt(opts, "to", "0").c_str());
    const int nrec_o = std::atoi(gopt(opts, "ovito", "0").c_str());
    const int mon_interval = std::atoi(gopt(opts, "mon", "0").c_str());
    const int nrec_rst = std::atoi(gopt(opts, "restart", "0").c_str());
    const std::string resfile = gopt(opts, "resfile", "");
    const std::string warmup_mon_mode = gopt(opts, "warmup_mon", "norm");
    constexpr double T_cold = 4.0;
    const double ff_kb = std::atof(gopt(opts, "ff_kb", "469.0").c_str()) * kcal2eV;    // MM:1043-1046
    const double ff_kth = std::atof(gopt(opts, "ff_kth", "63.0").c_str()) * kcal2eV;
    const double ff_v2 = std::atof(gopt(opts, "ff_v2", "14.5").c_str()) * kcal2eV;
    const double ff_kimp = std::atof(gopt(opts, "ff_kimp", "15.0").c_str()) * kcal2eV;
    int start_step = 0;

    if (avg_to <= 0) avg_to = nsteps;
    if (avg_from <= 0) avg_from = std::max(1, nsteps - nsteps / 4);
    const int total_steps = coldstart + warmup + nsteps;
    const int gavg_from = coldstart + warmup + avg_from, gavg_to = coldstart + warmup + avg_to;

    const auto fl = resolve_fullerene(fspec, libdir, Dialect::MM);
    const Molecule mol = load_cc1(fl.first, Dialect::MM);
    const double a0 = default_a0(mol.Dmol, st, init_scale);
    const int Nmol_max = st == "FCC" ? 4 * nc * nc * nc : 2 * nc * nc * nc;
    const long Na_max = (long)Nmol_max * mol.natom;

    char devname[128] = {0};
    double gpu_gb = 0;
    const double need = Na_max * (8.0 * 3 * 5 + 4 + 4.0 * (1 + 400) + 4.0 * (1 + 1024) + 48);
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
    mat_inv9(h, hi);
    std::vector<double> pos(3 * (size_t)Na), vel(3 * (size_t)Na, 0.0), charge(Na, 0.0);   // fullerenes: no charges
    for (int m = 0; m < Nmol; m++)
        for (int a = 0; a < mol.natom; a++)
            for (int c = 0; c < 3; c++)
                pos[3 * ((size_t)m * mol.natom + a) + c] = centres[3 * m + c] + mol.coords[3 * a + c];

    const Topology ft = build_flat_topology(mol, Nmol, ff_kb, ff_kth, ff_v2, ff_kimp);

    printf("========================================================================\n");
    printf("  Fullerene Crystal NPT-MD — MM Force Field (CUDA B200)\n");
    printf("========================================================================\n");
    printf("  GPU device      : 0 (%s)\n", devname[0] ? devname : "NVIDIA");
    printf("  Fullerene       : %s (%d atoms/mol)\n", fl.second.c_str(), mol.natom);
    printf("  Crystal         : %s %dx%dx%d  Nmol=%d  Natom=%d\n", st.c_str(), nc, nc, nc, Nmol, Na);
    printf("  a0=%.3f  T=%.1f K  P=%.4f GPa  dt=%.3f fs\n", a0, T, Pe, dt);
    printf("  Production      : %d steps  Total=%d\n", nsteps, total_steps);
    printf("========================================================================\n\n");

    const double T_init = (coldstart > 0 || warmup > 0) ? T_cold : T;    // MM:1110-1118
    std::mt19937 rng(seed);
    std::normal_distribution<double> gauss(0, 1);
    const double sv = std::sqrt(KB * T_init * CONV / MC);
    for (int i = 0; i < Na; i++)
        for (int a = 0; a < 3; a++) vel[3 * i + a] = sv * gauss(rng);
    double vcm[3] = {0, 0, 0};
    for (int i = 0; i < Na; i++)
        for (int a = 0; a < 3; a++) vcm[a] += vel[3 * i + a];
    for (int a = 0; a < 3; a++) vcm[a] /= Na;
    for (int i = 0; i < Na; i++)
        for (int a = 0; a < 3; a++) vel[3 * i + a] -= vcm[a];
    fmd_npt npt = make_npt_mm(T, Pe, 3 * Na - 3);
    npt.Tt = T_init;

    if (!resfile.empty()) {                                   // MM:1122-1131
        Restart rd = read_restart_mmmd(resfile);
        if (rd.ok) {
            start_step = rd.istep;
            for (int k = 0; k < 9; k++) h[k] = rd.h[k];
            mat_inv9(h, hi);
            npt = rd.npt;
            for (int i = 0; i < Na * 3 && i < rd.n * 3; i++) { pos[i] = rd.pos[i]; vel[i] = rd.vel[i]; }
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
    p.coldstart = coldstart; p.warmup = warmup; p.nsteps = nsteps; p.nlup = 20;   // MM:1180
    p.gavg_from = gavg_from; p.gavg_to = gavg_to; p.nc = nc; p.nmol = Nmol;
    p.precision = FMD_PREC_FP64; p.use_graphs = 1;
    const fmd_mm_topology tv = ft.view();
    fmd_system* sys = nullptr;
    check(ctx, fmd_system_create_mm(ctx, &p, Na, pos.data(), vel.data(), ft.mol_id.data(), &tv, charge.data(), h,
                                    &npt, &sys),
          "system set-up");
    // --physics=<fmd_physics bits>: opt-in force-field corrections, no
    // reference counterpart (not in the help text, which is the reference's)
    const int physics = std::atoi(gopt(opts, "physics", "0").c_str());
    if (physics) check(ctx, fmd_system_set_physics(sys, physics), "physics corrections");
    check(ctx, fmd_system_init(sys), "initial lists and forces");   // MM:1152-1172

    Schedule sc;
    sc.coldstart = coldstart; sc.warmup = warmup; sc.total = total_steps;
    sc.set_monitor(mon_interval, warmup_mon_mode);
    sc.nrec_o = nrec_o; sc.nrec_rst = nrec_rst;
    const double t0 = now_s();
    const std::string ovito_file = unique_file("ovito_traj_mmmd_gpu", ".xyz");
    FILE* io_o = nrec_o > 0 ? fopen(ovito_file.c_str(), "w") : nullptr;
    sc.ovito = io_o != nullptr;
    // frames are formatted and written on a writer thread while the steps go on
    std::unique_ptr<OvitoWriter> ovito(io_o ? new OvitoWriter(io_o) : nullptr);
    printf("  %8s %5s %7s %9s %8s %9s %9s %9s %9s %9s %7s\n", "step", "phase", "T[K]", "P[GPa]", "a[A]", "E_bond",
           "E_angle", "E_dih", "E_LJ", "E_total", "t[s]");
    const std::string rst_base = nrec_o > 0 ? ovito_file : std::string("restart_mmmd_gpu");

    RunInfo ri;
    ri.st = st; ri.fspec = fspec; ri.nc = nc; ri.nsteps = nsteps; ri.seed = seed;
    ri.T = T; ri.Pe = Pe; ri.dt = dt; ri.init_scale = init_scale;
    // checkpoints are formatted and written on a writer thread from copies
    std::unique_ptr<RestartWriter> rstw(nrec_rst > 0 ? new RestartWriter() : nullptr);
    auto save = [&](int s) {
        check(ctx, fmd_system_download(sys, pos.data(), vel.data(), nullptr, nullptr, h, &npt), "download");
        // h (a C array) and the vectors are captured by copy
        rstw->submit([fn = restart_filename(rst_base, s, total_steps), s, opts, ri, h, npt, p = pos, v = vel, Na, Nmol,
                      natom = mol.natom]() {
            write_restart_mmmd(fn, s, opts, ri, h, npt, p.data(), v.data(), Na, Nmol, natom);
        });
    };
    bool stop_requested = false;
    for (int gs = start_step + 1; gs <= total_steps;) {
        const int e = sc.next_event(gs);
        fmd_obs o;
        check(ctx, fmd_system_run(sys, gs, e, &o), "MD steps");
        if (sc.ovito_at(e)) {
            check(ctx, fmd_system_download(sys, pos.data(), vel.data(), nullptr, nullptr, h, nullptr), "download");
            ovito->atoms(e, dt, pos.data(), vel.data(), ft.mol_id.data(), 1, h, Na);
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
                if (nrec_rst == 0) break;
            }
            // o.E = {Eb, Ea, Ed, Ei, Elj, Ecoul, Etot}
            printf("  %8d %5s %7.1f %9.3f %8.3f %9.4f %9.4f %9.4f %9.4f %9.4f %7.0f\n", e, sc.phase(e), o.T, o.P, o.a,
                   o.E[0] / Nmol, o.E[1] / Nmol, (o.E[2] + o.E[3]) / Nmol, o.E[4] / Nmol, o.E[6] / Nmol,
                   elapsed_since(t0));
        }
        gs = e + 1;
    }
    ovito.reset();                          // every frame written
    rstw.reset();                           // every checkpoint written
    if (io_o) fclose(io_o);
    fmd_avg av;
    check(ctx, fmd_system_averages(sys, &av), "averages");
    if (av.n > 0)
        printf("\n  Averages (%d): T=%.2f P=%.4f a=%.4f  bond=%.4f ang=%.4f dih=%.4f LJ=%.4f tot=%.4f\n", av.n,
               av.sT / av.n, av.sP / av.n, av.sa / av.n, av.sE[0] / av.n, av.sE[1] / av.n, av.sE[2] / av.n,
               av.sE[3] / av.n, av.sE[4] / av.n);
    printf("  Done (%.1f sec)\n", elapsed_since(t0));
    fmd_system_destroy(sys);
    fmd_ctx_destroy(ctx);
    return 0;
}
