// nlist.cu -- neighbour lists on the device, bit-exact with the reference's
// O(N^2) host builders (LJ:257-268, AI:251-272, MM:337-346).
//
// Design.  The reference keeps, per row, the FIRST `cap` accepted partners in
// ascending index order, where a pair is accepted by one FP64 test on one
// periodic image.  Membership of a row therefore depends only on the row's
// own accepted set, so rows are independent and map to one warp each:
//   1. particles are binned into a fractional-space cell grid whose cells are
//      at least rc wide (computed on the device from the current cell matrix;
//      a list rebuild never needs the host);
//   2. the warp walks the <=27 neighbouring cells; a cheap FP32 pre-filter
//      rejects far candidates (only when the box is wider than 2 rc, where
//      FP32 and FP64 cannot pick different images of an accepted pair), and the
//      survivors get the reference's FP64 test with the reference's operation
//      order (geom.cuh);
//   3. accepted partners set bits in a per-warp shared-memory bitmap indexed by
//      partner id; scanning the bitmap yields them in ascending order, and the
//      first `cap` are written -- the reference's truncation, exactly.
#include <climits>
#include <cmath>
#include "kernels.h"
#include "geom.cuh"

namespace fmd {

namespace {

// Cells per axis with cell width >= rc / K (K cells span the cutoff).
__host__ __device__ inline void grid_dims(const double* h, double rc, int K, int* n, double* wmin) {
    // Columns of h are the lattice vectors; the perpendicular width along
    // vector a is V / |b x c|.
    const double c[3][3] = {{h[0], h[3], h[6]}, {h[1], h[4], h[7]}, {h[2], h[5], h[8]}};
    double V = fabs(c[0][0] * (c[1][1] * c[2][2] - c[1][2] * c[2][1]) -
                    c[0][1] * (c[1][0] * c[2][2] - c[1][2] * c[2][0]) +
                    c[0][2] * (c[1][0] * c[2][1] - c[1][1] * c[2][0]));
    double rcb = rc * (1.0 + 1e-9) + 1e-9;
    double wm = 1e300;
    for (int a = 0; a < 3; a++) {
        const double* u = c[(a + 1) % 3];
        const double* v = c[(a + 2) % 3];
        double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
        double w = V / sqrt(x * x + y * y + z * z);
        wm = w < wm ? w : wm;
        int k = (int)floor(K * w / rcb);
        n[a] = k < 1 ? 1 : k;
    }
    *wmin = wm;
}

__global__ void k_grid(const double* __restrict__ hh, double rc, int K, int c0, int c1, int c2, GridDev* g) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int n[3];
    double wmin;
    grid_dims(hh, rc, K, n, &wmin);
    const int cap[3] = {c0, c1, c2};
    GridDev G;
    for (int a = 0; a < 3; a++) {
        // Fewer, wider cells are always correct, so clamp to the allocation.
        G.n[a] = n[a] < cap[a] ? n[a] : cap[a];
        // A pair within rc differs by at most K cells per axis; with fewer
        // than 2K+1 cells the stencil is every cell of that axis, once.
        if (G.n[a] >= 2 * K + 1) { G.lo[a] = -K; G.span[a] = 2 * K + 1; }
        else { G.lo[a] = 0; G.span[a] = G.n[a]; }
    }
    G.ncell = G.n[0] * G.n[1] * G.n[2];
    G.prefilter = (wmin >= 2.0 * rc * (1.0 + 1e-5)) ? 1 : 0;
    for (int k = 0; k < 9; k++) G.hf[k] = (float)hh[k];
    G.rc2_hi = (float)(rc * rc * (1.0 + 2e-4) + 0.01);
    *g = G;
}

// gate (may be null): a set value means the molecule path builds this list.
__global__ void k_bin(const double* __restrict__ pos, int n, const double* __restrict__ hh,
                      const GridDev* __restrict__ g, int* __restrict__ cell_count,
                      int* __restrict__ cell_of, int* __restrict__ slot_of, float4* __restrict__ s4,
                      const int* __restrict__ gate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate)) return;
    const double* hi = hh + 9;
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    double s[3] = {hi[0] * x + hi[1] * y + hi[2] * z, hi[3] * x + hi[4] * y + hi[5] * z,
                   hi[6] * x + hi[7] * y + hi[8] * z};
    int c[3];
    for (int a = 0; a < 3; a++) {
        s[a] -= floor(s[a]);
        int k = (int)(s[a] * g->n[a]);
        c[a] = k < 0 ? 0 : (k >= g->n[a] ? g->n[a] - 1 : k);
    }
    int cid = (c[0] * g->n[1] + c[1]) * g->n[2] + c[2];
    cell_of[i] = cid;
    slot_of[i] = atomicAdd(&cell_count[cid], 1);
    s4[i] = make_float4((float)s[0], (float)s[1], (float)s[2], 0.f);
}

// Exclusive scan of cell counts (one block of 1024 threads; ncell is read on
// the device).  Each thread owns a contiguous run of cells, so there is a
// single block-wide scan whatever ncell is.
__global__ void __launch_bounds__(1024)
k_scan(const int* __restrict__ cell_count, const GridDev* __restrict__ g, int* __restrict__ cell_start,
       const int* __restrict__ gate) {
    if (gate && *gate) return;
    __shared__ int sm[1024];
    const int ncell = g->ncell;
    const int per = (ncell + 1023) / 1024;
    const int b0 = min(threadIdx.x * per, ncell), b1 = min(b0 + per, ncell);
    int s = 0;
    for (int c = b0; c < b1; c++) s += cell_count[c];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int t = threadIdx.x >= o ? sm[threadIdx.x - o] : 0;
        __syncthreads();
        sm[threadIdx.x] += t;
        __syncthreads();
    }
    int run = sm[threadIdx.x] - s;
    for (int c = b0; c < b1; c++) {
        cell_start[c] = run;
        run += cell_count[c];
    }
    if (threadIdx.x == 1023) cell_start[ncell] = sm[1023];
}

// Cell order: the candidate loop of the list kernel then reads ids,
// fractional coordinates and molecule ids contiguously (coalesced) instead
// of gathering them through the ids.
__global__ void k_scatter(int n, const int* __restrict__ cell_of, const int* __restrict__ slot_of,
                          const int* __restrict__ cell_start, int* __restrict__ cell_atoms,
                          const float4* __restrict__ s4, const int* __restrict__ mol_id, float4* __restrict__ s4s,
                          int* __restrict__ mols, const int* __restrict__ gate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate)) return;
    const int k = cell_start[cell_of[i]] + slot_of[i];
    cell_atoms[k] = i;
    s4s[k] = s4[i];
    mols[k] = mol_id ? mol_id[i] : 0;
}

__device__ __forceinline__ int wrapc(int x, int n) {
    x += (x < 0) ? n : 0;
    x -= (x >= n) ? n : 0;
    return x;
}

// Emits the set bits of bm[wlo..whi] in ascending order into row[0..cap),
// clearing the words.  Returns the number of set bits.
__device__ __forceinline__ int bitmap_emit(unsigned* bm, int wlo, int whi, int* row, int cap, int lane) {
    int emitted = 0;
    for (int w0 = wlo; w0 <= whi; w0 += 32) {
        int w = w0 + lane;
        unsigned bits = 0u;
        if (w <= whi) { bits = bm[w]; bm[w] = 0u; }
        int c = __popc(bits), incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        int base = emitted + incl - c;
        while (bits) {
            int b = __ffs(bits) - 1;
            bits &= bits - 1u;
            if (base < cap) row[base] = (w << 5) + b;
            base++;
        }
        emitted += __shfl_sync(kFull, incl, 31);
    }
    return emitted;
}

template <int MODE>
__global__ void __launch_bounds__(256)
k_nlist(const GridDev* __restrict__ g, const int* __restrict__ cell_start,
        const int* __restrict__ cell_atoms, const int* __restrict__ cell_of,
        const float4* __restrict__ s4, const float4* __restrict__ s4s, const int* __restrict__ mols,
        const double* __restrict__ pos, const int* __restrict__ mol_id, int n, const double* __restrict__ hh,
        double rc2, int cap, int words, int* __restrict__ cnt, int* __restrict__ list, int* __restrict__ dropped,
        const int* __restrict__ gate) {
    if (gate && *gate) return;
    extern __shared__ unsigned bm_all[];
    __shared__ double s_hh[18];
    __shared__ GridDev G;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    unsigned* bm = bm_all + (size_t)wib * words;
    for (int w = lane; w < words; w += 32) bm[w] = 0u;
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    if (threadIdx.x == 0) G = *g;
    __syncthreads();
    const double* h = s_hh;
    const double* hi = s_hh + 9;
    // Diagonal cell: the reference's mimg reduces exactly to per-axis products.
    const bool diag = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0 &&
                      hi[1] == 0.0 && hi[2] == 0.0 && hi[3] == 0.0 && hi[5] == 0.0 && hi[6] == 0.0 && hi[7] == 0.0;
    for (int i = blockIdx.x * wpb + wib; i < n; i += gridDim.x * wpb) {
        const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        const float4 si = s4[i];
        const int mi = (MODE != LIST_SYM) ? mol_id[i] : 0;
        const int ci = cell_of[i];
        const int n1 = G.n[1], n2 = G.n[2];
        const int cz = ci % n2, cy = (ci / n2) % n1, cx = ci / (n1 * n2);
        int jmin = INT_MAX, jmax = -1, tot = 0;
        for (int a = 0; a < G.span[0]; a++) {
            const int x = wrapc(cx + G.lo[0] + a, G.n[0]);
            for (int b = 0; b < G.span[1]; b++) {
                const int y = wrapc(cy + G.lo[1] + b, n1);
                // The z-run of stencil cells is contiguous in cell order: one
                // candidate range, or two when it wraps around the box.
                const int base = (x * n1 + y) * n2;
                int z0 = cz + G.lo[2];
                z0 += (z0 < 0) ? n2 : 0;
                const int zlen = G.span[2];
                const int first_len = (z0 + zlen <= n2) ? zlen : n2 - z0;
                for (int part = 0; part < 2; part++) {
                    const int zs = part == 0 ? z0 : 0;
                    const int zl = part == 0 ? first_len : zlen - first_len;
                    if (zl <= 0) continue;
                    const int beg = cell_start[base + zs], end = cell_start[base + zs + zl];
                    for (int k = beg + lane; k < end; k += 32) {
                        const int j = cell_atoms[k];
                        bool ok = (MODE == LIST_HALF) ? (j > i) : (j != i);
                        if (ok && MODE != LIST_SYM) {
                            const int mj = mols[k];
                            ok = (MODE == LIST_INTRA) ? (mj == mi) : (mj != mi);
                        }
                        if (ok && G.prefilter) {
                            const float4 sj = s4s[k];
                            float dx = sj.x - si.x, dy = sj.y - si.y, dz = sj.z - si.z;
                            dx -= rintf(dx); dy -= rintf(dy); dz -= rintf(dz);
                            float ex = G.hf[0] * dx + G.hf[1] * dy + G.hf[2] * dz;
                            float ey = G.hf[3] * dx + G.hf[4] * dy + G.hf[5] * dz;
                            float ez = G.hf[6] * dx + G.hf[7] * dy + G.hf[8] * dz;
                            ok = (ex * ex + ey * ey + ez * ez) <= G.rc2_hi;
                        }
                        if (ok) {
                            double dx = __dsub_rn(pos[3 * j], px), dy = __dsub_rn(pos[3 * j + 1], py),
                                   dz = __dsub_rn(pos[3 * j + 2], pz);
                            if (diag) {
                                double s0 = __dmul_rn(hi[0], dx), s1 = __dmul_rn(hi[4], dy), s2 = __dmul_rn(hi[8], dz);
                                s0 = __dsub_rn(s0, round(s0));
                                s1 = __dsub_rn(s1, round(s1));
                                s2 = __dsub_rn(s2, round(s2));
                                dx = __dmul_rn(h[0], s0); dy = __dmul_rn(h[4], s1); dz = __dmul_rn(h[8], s2);
                            } else {
                                mimg(dx, dy, dz, hi, h);
                            }
                            ok = norm2_rn(dx, dy, dz) < rc2;
                        }
                        if (ok) {
                            atomicOr(&bm[j >> 5], 1u << (j & 31));
                            jmin = j < jmin ? j : jmin;
                            jmax = j > jmax ? j : jmax;
                            tot++;
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            jmin = min(jmin, __shfl_xor_sync(kFull, jmin, o));
            jmax = max(jmax, __shfl_xor_sync(kFull, jmax, o));
            tot += __shfl_xor_sync(kFull, tot, o);
        }
        __syncwarp();
        if (tot > 0) bitmap_emit(bm, jmin >> 5, jmax >> 5, list + (size_t)i * cap, cap, lane);
        if (lane == 0) {
            cnt[i] = tot < cap ? tot : cap;
            if (tot > cap && dropped) atomicAdd(dropped, tot - cap);
        }
        __syncwarp();
    }
}

// Full rows for the LJ gather: row j (stride in_cap) holds the incoming
// entries i < j of the half list (at most in_cap - cap, ascending) followed
// by j's own half-list row.
// Scatter half-list entries (i -> j) into row j.
__global__ void k_transpose_scatter(const int* __restrict__ cnt, const int* __restrict__ list, int cap,
                                    int n, int* __restrict__ in_cnt, int* __restrict__ in_list,
                                    int in_cap, DevErr* err, const int* __restrict__ gate) {
    if (gate && *gate) return;
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    const int m = cnt[i];
    for (int k = lane; k < m; k += 32) {
        const int j = list[(size_t)i * cap + k];
        const int slot = atomicAdd(&in_cnt[j], 1);
        if (slot < in_cap - cap) in_list[(size_t)j * in_cap + slot] = i;
        else if (atomicCAS(&err->code, FMD_OK, FMD_ERR_CAPACITY) == FMD_OK) {
            err->where = K_TRANSPOSE; err->index = j; err->value = slot + 1;
        }
    }
}

// Sorts each incoming row ascending through the bitmap, then appends the
// atom's own half-list row.
__global__ void __launch_bounds__(256)
k_transpose_sort(int n, int* __restrict__ in_cnt, int* __restrict__ in_list, int in_cap, int words,
                 const int* __restrict__ cnt, const int* __restrict__ list, int cap, const int* __restrict__ gate) {
    if (gate && *gate) return;
    extern __shared__ unsigned bm_all[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    unsigned* bm = bm_all + (size_t)wib * words;
    for (int w = lane; w < words; w += 32) bm[w] = 0u;
    __syncwarp();
    for (int j = blockIdx.x * wpb + wib; j < n; j += gridDim.x * wpb) {
        int m = in_cnt[j];
        m = m < in_cap - cap ? m : in_cap - cap;
        int* row = in_list + (size_t)j * in_cap;
        int lo = INT_MAX, hi = -1;
        for (int k = lane; k < m; k += 32) {
            const int i = row[k];
            atomicOr(&bm[i >> 5], 1u << (i & 31));
            lo = i < lo ? i : lo;
            hi = i > hi ? i : hi;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(kFull, lo, o));
            hi = max(hi, __shfl_xor_sync(kFull, hi, o));
        }
        __syncwarp();
        if (m > 0) bitmap_emit(bm, lo >> 5, hi >> 5, row, in_cap - cap, lane);
        const int mo = cnt[j];
        for (int k = lane; k < mo; k += 32) row[m + k] = list[(size_t)j * cap + k];
        if (lane == 0) in_cnt[j] = m + mo;
        __syncwarp();
    }
}

__global__ void k_apply_pbc(double* __restrict__ pos, int n, const double* __restrict__ hh) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    wrap_point(x, y, z, hh, hh + 9);
    pos[3 * i] = x; pos[3 * i + 1] = y; pos[3 * i + 2] = z;
}

__global__ void k_inv9(double* hh) {
    if (threadIdx.x == 0 && blockIdx.x == 0) inv9(hh, hh + 9);
}

}  // namespace

void grid_dims_host(const double* h, double rc, int K, int* n) {
    double wmin;
    grid_dims(h, rc, K, n, &wmin);
}

cudaError_t cells_alloc(CellList& cl, int n, const double* h_host, double rc, int K, const DevAlloc& da) {
    int nd[3];
    cl.K = K;
    grid_dims_host(h_host, rc, K, nd);
    cl.cap_cells = 1;
    for (int a = 0; a < 3; a++) {
        // Room for the box to grow to twice its width before cells get wider.
        cl.cap_n[a] = 2 * nd[a] + 2;
        cl.cap_cells *= cl.cap_n[a];
    }
    cl.n = n;
    cl.ext = da.fn != nullptr;
    cudaError_t e;
    if ((e = da((void**)&cl.grid, sizeof(GridDev))) != cudaSuccess) return e;
    if ((e = da((void**)&cl.cell_count, sizeof(int) * cl.cap_cells)) != cudaSuccess) return e;
    if ((e = da((void**)&cl.cell_start, sizeof(int) * (cl.cap_cells + 1))) != cudaSuccess) return e;
    size_t nn = n > 0 ? n : 1;
    if ((e = da((void**)&cl.cell_atoms, sizeof(int) * nn)) != cudaSuccess) return e;
    if ((e = da((void**)&cl.slot_of, sizeof(int) * nn)) != cudaSuccess) return e;
    if ((e = da((void**)&cl.cell_of, sizeof(int) * nn)) != cudaSuccess) return e;
    if ((e = da((void**)&cl.s4, sizeof(float4) * nn)) != cudaSuccess) return e;
    if ((e = da((void**)&cl.s4s, sizeof(float4) * nn)) != cudaSuccess) return e;
    if ((e = da((void**)&cl.mols, sizeof(int) * nn)) != cudaSuccess) return e;
    return cudaSuccess;
}

void cells_free(CellList& cl) {
    if (cl.ext) {
        cl = CellList();
        return;
    }
    cudaFree(cl.grid); cudaFree(cl.cell_count); cudaFree(cl.cell_start); cudaFree(cl.cell_atoms);
    cudaFree(cl.slot_of); cudaFree(cl.cell_of); cudaFree(cl.s4); cudaFree(cl.s4s); cudaFree(cl.mols);
    cl = CellList();
}

cudaError_t cells_build(CellList& cl, const double* pos, int n, const double* hh, double rc,
                        DevErr* err, cudaStream_t st, const int* mol_id, const int* gate) {
    (void)err;
    k_grid<<<1, 32, 0, st>>>(hh, rc, cl.K, cl.cap_n[0], cl.cap_n[1], cl.cap_n[2], cl.grid);
    cudaMemsetAsync(cl.cell_count, 0, sizeof(int) * cl.cap_cells, st);
    if (n > 0) {
        k_bin<<<(n + 255) / 256, 256, 0, st>>>(pos, n, hh, cl.grid, cl.cell_count, cl.cell_of, cl.slot_of, cl.s4,
                                               gate);
    }
    k_scan<<<1, 1024, 0, st>>>(cl.cell_count, cl.grid, cl.cell_start, gate);
    if (n > 0) {
        k_scatter<<<(n + 255) / 256, 256, 0, st>>>(n, cl.cell_of, cl.slot_of, cl.cell_start, cl.cell_atoms, cl.s4,
                                                   mol_id, cl.s4s, cl.mols, gate);
    }
    return cudaGetLastError();
}

size_t nlist_bitmap_smem(int n, int* warps_per_block) {
    size_t words = ((size_t)(n > 0 ? n : 1) + 31) / 32;
    size_t per_warp = words * 4;
    int wpb = (int)((96 * 1024) / per_warp);
    if (wpb > 8) wpb = 8;
    if (wpb < 1) wpb = 1;
    *warps_per_block = wpb;
    return per_warp * wpb;
}

namespace {
template <int MODE>
cudaError_t launch_nlist(const CellList& cl, const double* pos, const int* mol_id, int n,
                         const double* hh, double rc2, int cap, int* cnt, int* list, int* dropped,
                         cudaStream_t st, const int* gate) {
    int wpb;
    size_t smem = nlist_bitmap_smem(n, &wpb);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_nlist<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set = true;
    }
    int words = (n + 31) / 32;
    int blocks = (n + wpb - 1) / wpb;
    if (blocks > kSMs * 16) blocks = kSMs * 16;
    if (blocks < 1) blocks = 1;
    k_nlist<MODE><<<blocks, 32 * wpb, smem, st>>>(cl.grid, cl.cell_start, cl.cell_atoms, cl.cell_of, cl.s4,
                                                  cl.s4s, cl.mols, pos, mol_id, n, hh, rc2, cap, words, cnt, list,
                                                  dropped, gate);
    return cudaGetLastError();
}
}  // namespace

cudaError_t nlist_build(const CellList& cl, int mode, const double* pos, const int* mol_id, int n,
                        const double* hh, double rc2, int cap, int* cnt, int* list, int* dropped,
                        DevErr* err, cudaStream_t st, const int* gate) {
    (void)err;
    if (n <= 0) return cudaSuccess;
    switch (mode) {
        case LIST_SYM: return launch_nlist<LIST_SYM>(cl, pos, mol_id, n, hh, rc2, cap, cnt, list, dropped, st, gate);
        case LIST_INTRA:
            return launch_nlist<LIST_INTRA>(cl, pos, mol_id, n, hh, rc2, cap, cnt, list, dropped, st, gate);
        default: return launch_nlist<LIST_HALF>(cl, pos, mol_id, n, hh, rc2, cap, cnt, list, dropped, st, gate);
    }
}

cudaError_t nlist_transpose(const int* cnt, const int* list, int cap, int n, int* in_cnt, int* in_list,
                            int in_cap, DevErr* err, cudaStream_t st, const int* gate) {
    if (n <= 0) return cudaSuccess;
    cudaMemsetAsync(in_cnt, 0, sizeof(int) * n, st);
    k_transpose_scatter<<<(n * 32 + 255) / 256, 256, 0, st>>>(cnt, list, cap, n, in_cnt, in_list, in_cap, err, gate);
    int wpb;
    size_t smem = nlist_bitmap_smem(n, &wpb);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_transpose_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set = true;
    }
    int blocks = (n + wpb - 1) / wpb;
    if (blocks > kSMs * 16) blocks = kSMs * 16;
    k_transpose_sort<<<blocks, 32 * wpb, smem, st>>>(n, in_cnt, in_list, in_cap, (n + 31) / 32, cnt, list, cap, gate);
    return cudaGetLastError();
}

cudaError_t apply_pbc_launch(double* pos, int n, const double* hh, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_apply_pbc<<<(n + 255) / 256, 256, 0, st>>>(pos, n, hh);
    return cudaGetLastError();
}

cudaError_t inv9_launch(double* hh, cudaStream_t st) {
    k_inv9<<<1, 32, 0, st>>>(hh);
    return cudaGetLastError();
}

}  // namespace fmd
