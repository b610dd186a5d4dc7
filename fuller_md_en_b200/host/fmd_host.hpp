// fmd_host.hpp -- host-side boundary of the drop-in drivers: command line,
// fullerene library, crystal set-up, MM topology, OVITO XYZ and restart
// files.  Formats and semantics follow the reference programs so the
// fuller_*_gpu drivers are drop-in replacements (file:line citations are to
// the reference's src/ directory: LJ = fuller_LJ_npt_md_serial_omp_acc.cpp,
// AI = fuller_airebo_npt_md_serial_omp_acc.cpp,
// MM = fuller_LJ_npt_mmmd_serial_omp_acc.cpp, CORE = ..._core_serial*.cpp).
// No CUDA here; the drivers call libfullermd_cuda.so for all per-step work.
#pragma once
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "fullermd.h"

namespace fmdh {

constexpr double CONV = 9.64853321e-3, KB = 8.617333262e-5;
constexpr double EV2GPA = 160.21766208, EV2KCAL = 23.06054783;
constexpr double MC = 12.011;
constexpr double PI = 3.14159265358979323846;

using Opts = std::map<std::string, std::string>;

// --key=value options, keys lower-cased, later keys win (LJ:558-566).
Opts parse_args(int argc, char** argv);
std::string gopt(const Opts& o, const std::string& k, const std::string& d);
bool file_exists(const std::string& p);
bool dir_exists(const char* p);
// base+ext, else base_1+ext ... base_9999+ext (LJ:579-582).
std::string unique_file(const std::string& base, const std::string& ext);
// ovito_traj -> restart, zero-padded step unless final (LJ:583-588).
std::string restart_filename(const std::string& oname, int istep, int nsteps);
// _key_value for the non-default core options, ':' -> '_', trailing ".0" dropped (LJ:568-577).
std::string build_suffix(const Opts& o);

enum class Dialect { LJ, AI, MM };   // the three programs' message wording differs

// Species name -> (.cc1 path, label) (LJ:210-226); exits with the
// program's message on an unknown species.
std::pair<std::string, std::string> resolve_fullerene(const std::string& spec, const std::string& lib, Dialect d);

struct Molecule {
    int natom = 0;
    std::vector<double> coords;             // centred, natom x 3
    std::vector<std::pair<int, int>> bonds; // sorted unique (lo, hi) from the adjacency columns (MM:169-182)
    double Rmol = 0, Dmol = 0, I0 = 0, Mmol = 0;
};
// .cc1 reader (LJ:178-207, AI:195-210, MM:160-183); exits on a missing file.
Molecule load_cc1(const std::string& path, Dialect d);

// Lattice centres and cell matrix (LJ:229-254).
int make_crystal(const std::string& st, double a, int nc, double* pos, double* h);
double default_a0(double dmax, const std::string& st, double s);
// Golden-ratio truncated icosahedron x 0.72 of the core program (CORE:228-252).
void generate_c60(double* coords, double* I0, double* Mmol, double* Rmol);
void mat_inv9(const double* h, double* hi);
double mat_det9(const double* h);

// Flat MM topology (MM:226-334), owning its arrays.
struct Topology {
    int nb_mol = 0, nang_mol = 0, ndih_mol = 0, nimp_mol = 0;
    std::vector<int> b_i0, b_i1, a_i0, a_i1, a_i2, d_i0, d_i1, d_i2, d_i3, d_mult, m_i0, m_i1, m_i2, m_i3, mol_id;
    std::vector<double> b_kb, b_r0, a_kth, a_th0, d_vn, d_gamma, m_ki, m_gamma;
    fmd_mm_topology view() const;
};
Topology build_flat_topology(const Molecule& mol, int nmol, double kb, double kth, double v2, double kimp);

// OVITO extended XYZ (LJ:541-555: rigid sites; AI:593-601 / MM:893-901: atoms).
void write_ovito_rigid(FILE* fp, int istep, double dt, const double* pos, const double* vel, const double* qv,
                       const double* body, const double* h, int n, int natom);
void write_ovito_atoms(FILE* fp, int istep, double dt, const double* pos, const double* vel, const int* mol_id,
                       int mol_offset, const double* h, int na);

// Asynchronous OVITO output: rigid()/atoms() copy the frame's state and
// return; a writer thread formats it (the lines split over up to `threads`
// worker threads, the same text as write_ovito_*) and appends it to fp,
// flushed frame by frame.  At most two frames are in flight: a third call
// waits for the oldest to be written.  finish() (and the destructor) wait
// for every frame; fp stays open (the caller closes it).
class OvitoWriter {
public:
    explicit OvitoWriter(FILE* fp, int threads = 0);
    ~OvitoWriter();
    OvitoWriter(const OvitoWriter&) = delete;
    OvitoWriter& operator=(const OvitoWriter&) = delete;
    void rigid(int istep, double dt, const double* pos, const double* vel, const double* qv, const double* body,
               const double* h, int n, int natom);
    void atoms(int istep, double dt, const double* pos, const double* vel, const int* mol_id, int mol_offset,
               const double* h, int na);
    void finish();

private:
    struct Frame;
    static constexpr int kSlots = 2;
    void submit(std::unique_ptr<Frame> f);
    void loop();
    void write(const Frame& f);
    FILE* fp_;
    int threads_ = 1;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::unique_ptr<Frame>> queue_;
    int inflight_ = 0;
    bool stop_ = false;
    std::thread th_;
};

// Background restart saves: submit() hands a write job (a callable that owns
// copies of the checkpoint's state and calls write_restart_*) to a writer
// thread and returns, so the step loop goes on while the file is formatted.
// Jobs run one at a time in submission order; at most two are pending, a
// third submit() waits for the oldest.  finish() (and the destructor) wait
// for every job.  The bytes are those of the synchronous call the job makes.
class RestartWriter {
public:
    RestartWriter();
    ~RestartWriter();
    RestartWriter(const RestartWriter&) = delete;
    RestartWriter& operator=(const RestartWriter&) = delete;
    void submit(std::function<void()> job);
    void finish();

private:
    static constexpr int kSlots = 2;
    void loop();
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> queue_;
    int inflight_ = 0;
    bool stop_ = false;
    std::thread th_;
};

// Restart files (LJ:590-635, AI:629-677, MM:930-976).
struct RunInfo {
    std::string st, fspec;
    int nc = 0, nsteps = 0, seed = 0;
    double T = 0, Pe = 0, dt = 0, init_scale = 0;
};
void write_restart_lj(const std::string& f, int istep, const Opts& o, const RunInfo& r, const double* h,
                      const fmd_npt& npt, const double* pos, const double* qv, const double* vel, const double* omg,
                      int n, int natom);
void write_restart_airebo(const std::string& f, int istep, const Opts& o, const RunInfo& r, const double* h,
                          const fmd_npt& npt, const double* pos, const double* vel, const int* mol_id,
                          const double* mass, int na, int nmol, int natom_mol);
void write_restart_mmmd(const std::string& f, int istep, const Opts& o, const RunInfo& r, const double* h,
                        const fmd_npt& npt, const double* pos, const double* vel, int na, int nmol, int natom);

struct Restart {
    bool ok = false;
    int istep = 0, n = 0;
    double h[9] = {0};
    fmd_npt npt{};
    std::vector<double> pos, vel, qv, omg, mass;
    std::vector<int> mol_id;
};
Restart read_restart_lj(const std::string& f);
Restart read_restart_airebo(const std::string& f);
Restart read_restart_mmmd(const std::string& f);

fmd_npt make_npt(double T, double Pe, int nf);   // Nf given: 6N-3 rigid, 3Na-3 atomistic
// The MM program scales Q and W by 1e4 and 1e6 in one multiply (MM:805-808),
// which can round differently from the two-step x100 x100 of LJ:426-430.
fmd_npt make_npt_mm(double T, double Pe, int nf);

double elapsed_since(double t0);
double now_s();

}  // namespace fmdh
