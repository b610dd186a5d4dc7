// kernels.h -- host-side launch interface of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include "fmd_internal.h"

namespace fmd {

// ---------------------------------------------------------------- cells ----
// Cell grid in fractional space, computed on the device from the current
// cell matrix so a list rebuild needs no host round trip.
struct GridDev {
    int n[3];        // cells per axis
    int ncell;
    int lo[3];       // first stencil offset per axis
    int span[3];     // stencil width per axis (1..3, never repeats a cell)
    int prefilter;   // 1 if the FP32 pre-filter is exact-safe for this box
    float hf[9];     // cell matrix in FP32 for the pre-filter
    float rc2_hi;    // conservative FP32 rejection threshold
};

// Device allocation hook: a system passes its own allocator (blocks it owns
// and releases to the context's cache); the *_free calls then leave such
// memory to its owner.  Without a hook, cudaMalloc / cudaFree.
struct DevAlloc {
    void* user = nullptr;
    cudaError_t (*fn)(void* user, void** p, size_t bytes) = nullptr;
    cudaError_t operator()(void** p, size_t bytes) const { return fn ? fn(user, p, bytes) : cudaMalloc(p, bytes); }
};

struct CellList {
    GridDev* grid = nullptr;    // device
    int* cell_count = nullptr;  // [cap_cells]
    int* cell_start = nullptr;  // [cap_cells + 1]
    int* cell_atoms = nullptr;  // [n]
    int* slot_of = nullptr;     // [n]
    int* cell_of = nullptr;     // [n]
    float4* s4 = nullptr;       // [n] fractional coordinates (FP32)
    float4* s4s = nullptr;      // [n] the same in cell order (cell_atoms order)
    int* mols = nullptr;        // [n] molecule ids in cell order
    int cap_n[3] = {1, 1, 1};
    int cap_cells = 1;
    int n = 0;
    int K = 1;                  // cells per cutoff length (cell width >= rc / K)
    bool ext = false;           // arrays from a DevAlloc hook (owned elsewhere)
};

// Host helper: cells per axis for a cell matrix and list radius.
void grid_dims_host(const double* h, double rc, int K, int* n);
// K = 2 halves the candidate volume for large cutoffs; K = 1 suits small ones.
cudaError_t cells_alloc(CellList& cl, int n, const double* h_host, double rc, int K = 1,
                        const DevAlloc& da = DevAlloc{});
void cells_free(CellList& cl);
// hh = device pointer to {h[9], hi[9]}.  Bins pos[3*n] into cells; mol_id
// (may be null) is copied into cell order beside the fractional coordinates.
// gate (device int, may be null): the cell-grid kernels do nothing while it is set.
cudaError_t cells_build(CellList& cl, const double* pos, int n, const double* hh, double rc,
                        DevErr* err, cudaStream_t st, const int* mol_id = nullptr, const int* gate = nullptr);

// -------------------------------------------------------- neighbour lists ----
enum ListMode { LIST_SYM = 0, LIST_INTRA = 1, LIST_HALF = 2 };
// Reference-exact list into cnt[n], list[n*cap]; *dropped (device int) += overflow.
cudaError_t nlist_build(const CellList& cl, int mode, const double* pos, const int* mol_id, int n,
                        const double* hh, double rc2, int cap, int* cnt, int* list, int* dropped,
                        DevErr* err, cudaStream_t st, const int* gate = nullptr);
// Full rows of a half list for the LJ gather: row j (stride in_cap) is the
// incoming entries i < j (ascending, at most in_cap - cap) then row j itself;
// in_cnt[j] = their total.
cudaError_t nlist_transpose(const int* cnt, const int* list, int cap, int n, int* in_cnt,
                            int* in_list, int in_cap, DevErr* err, cudaStream_t st, const int* gate = nullptr);
size_t nlist_bitmap_smem(int n, int* warps_per_block);

// ---------------------------------------------------------------- forces ----
constexpr int kForceBlocks = kSMs * 4;     // grid of the reduction-producing kernels
constexpr int kLJMaxBlocks = kSMs * 8;     // LJ gather grid cap (partial records of part_f2)
constexpr int kNV = 10;                    // {E, W[9]} per block partial

// REBO (a7): atomics into F, per-block {E, W9} partials in part[grid*kNV].
cudaError_t rebo_launch(const double* pos, const double* hh, const int* cnt, const int* list,
                        int cap, int na, double* F, double* part, cudaStream_t st);
// Same kernel on an explicit grid of `nblocks` blocks of 128 threads
// (nblocks partial records).
cudaError_t rebo_launch_grid(const double* pos, const double* hh, const int* cnt, const int* list,
                             int cap, int na, double* F, double* part, int nblocks, cudaStream_t st);
// Same, but the whole grid returns at once unless *gate == want (device int).
cudaError_t rebo_launch_gated(const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                              int na, double* F, double* part, int nblocks, const int* gate, int want,
                              cudaStream_t st);
// REBO through per-slot records (the fast path): `slots` holds
// kReboSlotDoubles doubles per list slot (na * cap geometry records, then
// na * cap bond-order records; device scratch owned by the caller); otherwise
// as rebo_launch_gated (gate may be null).
constexpr int kReboSlotDoubles = 16;
// ids (may be null): the occupied slots in atom-major order packed into
// 32-lane bins (no atom's slots cross a bin; unused lanes -1), ids[0] the
// padded length and ids[1 + k] the slot i * cap + jn, then at
// ids[1 + kIdsLanes * na + t] the partner slot of slot t (i's position in j's
// row, -1 if absent) (rebo_ids_build); lanes then walk only occupied slots,
// and the slots of one atom share a warp.
// phys: the gradient of the bond-order term in place of the reference's
// three-body forces (FMD_PHYS_REBO).
cudaError_t rebo_slots_launch(const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                              int na, double* slots, double* F, double* part, int nblocks, const int* gate,
                              int want, cudaStream_t st, const int* ids = nullptr, bool phys = false);
// REBO-II extension (rebo2.cu; no reference counterpart): bond order with
// P_CC(N, 0), pi^rc_CC(N_ij, N_ji, N_conj) and the dihedral term
// T_CC(...) sum (1 - cos^2 w) f_c f_c, and AIREBO's switched LJ.  Splines on
// integer knots N in [0, kRebo2Nx] x [0, kRebo2Ny] x [0, kRebo2Nz] (P_CC on
// [0, kRebo2Nx]); tables are per-cell polynomial coefficients: pcc[4 * cell
// + a] of u^a, pirc/tcc[cell * 64 + a + 4 b + 16 c] of u^a v^b w^c.
constexpr int kRebo2Nx = 4, kRebo2Ny = 4, kRebo2Nz = 9;
constexpr int kRebo2PccCoef = 4 * kRebo2Nx;
constexpr int kRebo2TriCoef = kRebo2Nx * kRebo2Ny * kRebo2Nz * 64;
// knots as fmd_rebo2_knots: P_CC {P, dP/dN} x (Nx+1), then pi^rc and T_CC,
// each (Nx+1)(Ny+1)(Nz+1) x {f, fx, fy, fz, fxy, fxz, fyz, fxyz}
constexpr int kRebo2Knots = 2 * (kRebo2Nx + 1) + 2 * (kRebo2Nx + 1) * (kRebo2Ny + 1) * (kRebo2Nz + 1) * 8;
// Close LJ pairs per atom the switched-LJ work list holds (more is an
// FMD_ERR_CAPACITY): far above the ~40 atoms dense carbon places within
// 2^(1/6) sigma of an atom.
constexpr int kRebo2SwitchPerAtom = 64;
struct Rebo2Dev {
    const double* pcc = nullptr;
    const double* pirc = nullptr;
    const double* tcc = nullptr;
    double* ncoord = nullptr;      // [n] scratch: sum of f_c over each atom's REBO row
    int2* bonds = nullptr;         // [n * cap_b] scratch: compacted bonds (i, j)
    int2* sw_pairs = nullptr;      // [sw_cap] scratch: compacted close LJ pairs
    int* counts = nullptr;         // [2] lengths of the two lists
    int sw_cap = 0;                // n * kRebo2SwitchPerAtom
    DevErr* err = nullptr;
};
// Host: the per-cell coefficients of the cubic Hermite splines through the
// knots (kRebo2Knots doubles) into pcc, pirc, tcc.
void rebo2_coeffs(const double* knots, double* pcc, double* pirc, double* tcc);
// N_k into t.ncoord.
cudaError_t rebo2_coord_launch(const Rebo2Dev& t, const double* pos, const double* hh, const int* cnt,
                               const int* list, int cap, int na, cudaStream_t st);
// REBO-II energy over the bonds i < j of the REBO rows: forces -grad E ADDED
// into F, {E, W9} partials in part[nblk * kNV] (full virial).  Computes
// t.ncoord first.
cudaError_t rebo2_launch(const Rebo2Dev& t, const double* pos, const double* hh, const int* cnt, const int* list,
                         int cap, int na, double* F, double* part, int nblk, cudaStream_t st);
// Switched-LJ correction over the LJ half rows (cnt_a, list_a): energy
// -V S(t_r) (1 - S(t_b(b*))) per pair, forces ADDED into F, {E, W9} partials.
// coord_ready: t.ncoord already holds this configuration's N_k.
cudaError_t lj_switch_launch(const Rebo2Dev& t, const double* pos, const double* hh, const int* cnt_b,
                             const int* list_b, int cap_b, const int* cnt_a, const int* list_a, int cap_a, int na,
                             double* F, double* part, int nblk, bool coord_ready, cudaStream_t st);

// Builds ids (1 + kIdsLanes n + n cap ints) from the list (cap <= 32);
// scratch: rebo_ids_scratch(n) ints.
constexpr int kIdsLanes = 32;
cudaError_t rebo_ids_build(const int* cnt, const int* list, int cap, int n, int* ids, int* scratch,
                           cudaStream_t st);
int rebo_ids_scratch(int n);
// Half-list LJ gather (a8, a14): F[i] = Facc[i] + LJ(i); Facc[i] zeroed
// (unless Facc == F).  ff: FMD_FF_AIREBO / FMD_FF_MM.  precision:
// FMD_PREC_FP64 (the reference's arithmetic) or FMD_PREC_FP32_PAIR (pair
// algebra in FP32, FP64 minimum image, cutoff test and accumulation).
// shape: threads per block (128/256), list entries in flight per lane (2/4)
// and the row feed (pipe 0: loads as used, 1: software-pipelined loads,
// 2: rows staged in shared memory by bulk asynchronous copies, needs
// in_cap % 4 == 0 and an error word); the grid is one full wave of the
// instantiation (resident blocks per SM x SMs, at most kLJMaxBlocks) and
// writes that many partial records -- lj_gather_blocks returns it (0: the
// shape cannot run with this row stride).  po.cnt non-null: a pruning
// gather, which also writes per atom i the entries of its row with
// r^2 <= po.r2 now, in row order, to po.list + i * in_cap (po.cnt[i] of them)
// and its fractional position to po.sb (ljprune.cu); with po.words also set
// the gather first decides (lj_prune_needed) and walks the pruned rows
// instead when no prune is due.  nrec > grid: the records grid .. nrec-1 are
// written as zeros.
struct LJShape {
    int threads = 256, unroll = 4, pipe = 0;
    // contig = 1: block b walks the atoms [b na / nblk, (b+1) na / nblk) in
    // order (the warps of a block share partner molecules, so their partner
    // positions stay in L1); 0: atoms strided over the whole grid.
    int contig = 0;
};
// The feed value of the shape entry points: bits 0-1 the row feed (0..2),
// bit 2 contig.
inline bool lj_feed_valid(int feed) { return feed >= 0 && feed <= 6 && (feed & 3) <= 2; }
struct LJPruneOut {
    int* cnt = nullptr;
    int* list = nullptr;
    double* sb = nullptr;
    double r2 = 0.0;
    // with words set, the gather decides per evaluation (lj_prune_needed):
    // full rows plus pruned-row output, or the pruned rows (cnt, list) as input
    const unsigned long long* words = nullptr;
    const double* hb = nullptr;
    double delta = 0.0, rc = 0.0;
};
int lj_gather_blocks(int ff, int precision, const LJShape& shape, int in_cap);
cudaError_t lj_gather_launch(int ff, const double* pos, const double* hh, const int* cnt,
                             const int* list, int cap, const int* in_cnt, const int* in_list,
                             int in_cap, int na, double* F, double* Facc, double* part,
                             cudaStream_t st, int precision = FMD_PREC_FP64, const LJShape& shape = LJShape{},
                             DevErr* err = nullptr, const LJPruneOut& po = LJPruneOut{}, int nrec = 0);
// Rigid site-site LJ (a5-a6): writes F, T; per-block {E, W9} partials (grid n).
// lab (may be null): scratch of n * natom * 4 doubles for the lab-frame sites;
// with it (and natom <= 64) the warp-per-neighbour kernel runs, in launch
// shape 0 (4 warps per molecule), 1 (4 warps, registers capped for 4 blocks
// per SM) or 2 (8 warps, capped for 2 blocks per SM).
constexpr int kRigidLabDoubles = 4;   // per site
// Site pairs within the cutoff (each molecule pair once) into *total
// (device), by the FP64 test; rebuilds the lab-frame sites in FP64 into lab.
cudaError_t rigid_count_pairs(const double* pos, const double* qv, const double* body, const double* hh,
                              const int* cnt, const int* list, int cap, int n, int natom, double rmcut2, double* lab,
                              unsigned long long* total, cudaStream_t st);
cudaError_t rigid_launch(int precision, const double* pos, const double* qv, const double* body,
                         const double* hh, const int* cnt, const int* list, int cap, int n,
                         int natom, double rmcut2, double* F, double* T, double* part,
                         cudaStream_t st, double* lab = nullptr, int shape = 0);
int rigid_grid(int n);

// MM bonded terms (a10-a13): atomics into Facc; partials {E_b,E_a,E_d,E_i, W00,W11,W22}
struct MMTopoDev {
    int nb, nang, ndih, nimp;
    const int *b_i0, *b_i1; const double *b_kb, *b_r0;
    const int *a_i0, *a_i1, *a_i2; const double *a_kth, *a_th0;
    const int *d_i0, *d_i1, *d_i2, *d_i3; const double *d_vn; const int *d_mult; const double *d_gamma;
    const int *m_i0, *m_i1, *m_i2, *m_i3; const double *m_ki, *m_gamma;
    int physical;                 // 1: bond and angle forces as -grad E (FMD_PHYS_MM_BONDED)
};
constexpr int kMMNV = 7;
// Writable view of a system's topology arrays (the replication's output).
struct MMTopoOut {
    int *b_i0, *b_i1; double *b_kb, *b_r0;
    int *a_i0, *a_i1, *a_i2; double *a_kth, *a_th0;
    int *d_i0, *d_i1, *d_i2, *d_i3; double* d_vn; int* d_mult; double* d_gamma;
    int *m_i0, *m_i1, *m_i2, *m_i3; double *m_ki, *m_gamma;
};
// The flat topology of nmol copies of one molecule of `natom` atoms (the
// replication of build_flat_topology, MM:254-334): term k of copy m is the
// molecule's term k with every index offset by m natom, copies in order,
// each term kind molecule-major.  `mol` holds one molecule's terms.
cudaError_t mm_replicate_launch(const MMTopoDev& mol, int nmol, int natom, const MMTopoOut& out, cudaStream_t st);
cudaError_t mm_bonded_launch(const MMTopoDev& t, const double* pos, const double* hh, double* Facc,
                             double* part, cudaStream_t st);
// Cut Coulomb (a15), all pairs of different molecules: adds into Facc; {Ecoul} partials.
cudaError_t mm_coulomb_launch(const double* pos, const double* hh, const double* charge,
                              const int* mol_id, int na, double* Facc, double* part, cudaStream_t st);

// Sums `nblk` partial records of width nv into out[nv] (deterministic).
cudaError_t reduce_partials(const double* part, int nblk, int nv, double* out, cudaStream_t st);

// Geometry helpers on device data.
cudaError_t apply_pbc_launch(double* pos, int n, const double* hh, cudaStream_t st);
cudaError_t inv9_launch(double* hh, cudaStream_t st);   // hh[9..17] = inv(hh[0..8])

}  // namespace fmd
