// abi.cu -- the extern "C" boundary: context management and the
// host-pointer entry points that each replace one reference routine.
// Host-pointer calls copy their inputs to scratch device memory, run the same
// kernels the device-resident systems use, copy the outputs back and
// synchronise; they are the parity surface the tests check.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "step.h"
#include "system.h"

using namespace fmd;

// ------------------------------------------------------------------ context --
int fmd_ctx::need(int slot, size_t bytes, void** out) {
    if ((int)scratch.size() <= slot) scratch.resize(slot + 1);
    DevBuf& b = scratch[slot];
    if (b.bytes < bytes) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
        cudaError_t e = cudaMalloc(&b.p, bytes);
        if (e != cudaSuccess) return fail(FMD_ERR_CUDA, std::string("scratch allocation: ") + cudaGetErrorString(e));
        b.bytes = bytes;
    }
    *out = b.p;
    return FMD_OK;
}

int fmd_ctx::sync_check(const char* what) {
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(FMD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FMD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    cudaMemcpy(h_err, d_err, sizeof(DevErr), cudaMemcpyDeviceToHost);
    if (h_err->code != FMD_OK) {
        DevErr de = *h_err;
        cudaMemset(d_err, 0, sizeof(DevErr));
        return fail(de.code, std::string(what) + ": device reported status " + std::to_string(de.code) +
                                 " in kernel " + std::to_string(de.where) + " at index " +
                                 std::to_string(de.index) + " (value " + std::to_string(de.value) + ")");
    }
    return FMD_OK;
}

extern "C" int fmd_version(void) { return 100; }

extern "C" const char* fmd_status_string(int code) {
    switch (code) {
        case FMD_OK: return "ok";
        case FMD_ERR_ARG: return "bad argument";
        case FMD_ERR_CUDA: return "CUDA error";
        case FMD_ERR_CAPACITY: return "capacity exceeded";
        case FMD_ERR_NONFINITE: return "non-finite value";
        case FMD_ERR_STATE: return "call out of order";
        default: return "unknown status";
    }
}

extern "C" int fmd_device_info(int device, char* name, int name_cap, double* total_gib) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        cudaGetLastError();
        return FMD_ERR_CUDA;
    }
    if (name && name_cap > 0) snprintf(name, name_cap, "%s", prop.name);
    if (total_gib) *total_gib = prop.totalGlobalMem / 1024.0 / 1024.0 / 1024.0;
    return FMD_OK;
}

extern "C" int fmd_ctx_create(fmd_ctx** out, int device) {
    if (!out) return FMD_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return FMD_ERR_CUDA;
    if (device < 0 || device >= ndev) return FMD_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return FMD_ERR_CUDA;
    fmd_ctx* c = new fmd_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_err, sizeof(DevErr)) != cudaSuccess ||
        cudaMallocHost(&c->h_err, sizeof(DevErr)) != cudaSuccess ||
        cudaMemset(c->d_err, 0, sizeof(DevErr)) != cudaSuccess) {
        delete c;
        return FMD_ERR_CUDA;
    }
    c->own_stream = true;
    *out = c;
    return FMD_OK;
}

extern "C" int fmd_ctx_destroy(fmd_ctx* ctx) {
    if (!ctx) return FMD_OK;
    cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->scratch) if (b.p) cudaFree(b.p);
    for (auto& b : ctx->mem_cache) cudaFree(b.second);
    ctx->mem_cache.clear();
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->h_err) cudaFreeHost(ctx->h_err);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return FMD_OK;
}

extern "C" int fmd_ctx_set_stream(fmd_ctx* ctx, void* s) {
    if (!ctx) return FMD_ERR_ARG;
    cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = (cudaStream_t)s;
    ctx->own_stream = false;
    return FMD_OK;
}

extern "C" void* fmd_ctx_get_stream(fmd_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" int fmd_ctx_synchronize(fmd_ctx* ctx) {
    if (!ctx) return FMD_ERR_ARG;
    return ctx->sync_check("synchronize");
}

extern "C" const char* fmd_ctx_last_error(const fmd_ctx* ctx) {
    return ctx ? ctx->last_msg.c_str() : "no context";
}

// ------------------------------------------------------------- host calls --
namespace {

// Scratch slots used by the host-pointer entry points.
enum Slot {
    S_POS = 0, S_HH, S_MOL, S_CNT, S_LIST, S_CNT2, S_LIST2, S_INCNT, S_INLIST, S_DROP,
    S_F, S_FACC, S_T, S_QV, S_BODY, S_VEL, S_OMG, S_MASS, S_PART1, S_PART2, S_PART3, S_PARTKE,
    S_SCAL, S_CHARGE, S_RSLOT, S_RLAB, S_R2TAB, S_R2NC, S_R2BOND, S_R2PAIR, S_R2CNT, S_TOPO0
};

template <class T>
int up(fmd_ctx* ctx, int slot, const T* src, size_t count, T** dst) {
    void* p;
    int rc = ctx->need(slot, sizeof(T) * (count > 0 ? count : 1), &p);
    if (rc != FMD_OK) return rc;
    *dst = (T*)p;
    if (src && count)
        if (cudaMemcpyAsync(p, src, sizeof(T) * count, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "host to device copy failed");
    return FMD_OK;
}

template <class T>
int down(fmd_ctx* ctx, T* dst, const T* src, size_t count) {
    if (!dst || !count) return FMD_OK;
    if (cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "device to host copy failed");
    return FMD_OK;
}

// Temporary cell list for one host call (freed at scope exit).
struct TmpCells {
    CellList cl;
    ~TmpCells() { cells_free(cl); }
};

int upload_cell(fmd_ctx* ctx, const double* h, const double* hi, double** hh) {
    int rc = up<double>(ctx, S_HH, nullptr, 18, hh);
    if (rc) return rc;
    double buf[18];
    std::memcpy(buf, h, sizeof(double) * 9);
    std::memcpy(buf + 9, hi, sizeof(double) * 9);
    if (cudaMemcpy(*hh, buf, sizeof(buf), cudaMemcpyHostToDevice) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "cell upload failed");
    return FMD_OK;
}

int list_call(fmd_ctx* ctx, int mode, const double* pos, const double* h, const double* hi, int n,
              const int* mol_id, double rc, int cap, int* cnt, int* list, int* dropped) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !h || !hi || !cnt || !list || n < 0 || cap < 1 || (mode != LIST_SYM && !mol_id))
        return ctx->fail(FMD_ERR_ARG, "neighbour list: bad argument");
    if (n == 0) { if (dropped) *dropped = 0; return FMD_OK; }
    int wpb;
    if (nlist_bitmap_smem(n, &wpb) > 200 * 1024) return ctx->fail(FMD_ERR_CAPACITY, "too many particles for the list builder");
    double *dpos, *hh; int *dmol = nullptr, *dcnt, *dlist, *ddrop;
    int rc_ = up(ctx, S_POS, pos, 3 * (size_t)n, &dpos);
    if (!rc_) rc_ = upload_cell(ctx, h, hi, &hh);
    if (!rc_ && mol_id) rc_ = up(ctx, S_MOL, mol_id, n, &dmol);
    if (!rc_) rc_ = up<int>(ctx, S_CNT, nullptr, n, &dcnt);
    if (!rc_) rc_ = up<int>(ctx, S_LIST, nullptr, (size_t)n * cap, &dlist);
    if (!rc_) rc_ = up<int>(ctx, S_DROP, nullptr, 1, &ddrop);
    if (rc_) return rc_;
    cudaMemsetAsync(dlist, 0, sizeof(int) * (size_t)n * cap, ctx->stream);
    cudaMemsetAsync(ddrop, 0, sizeof(int), ctx->stream);
    TmpCells tc;
    if (cells_alloc(tc.cl, n, h, rc, mode == LIST_INTRA ? 1 : 2) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "cell allocation failed");
    if (cells_build(tc.cl, dpos, n, hh, rc, ctx->d_err, ctx->stream, dmol) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "cell build launch failed");
    const double rc2 = rc * rc;
    if (nlist_build(tc.cl, mode, dpos, dmol, n, hh, rc2, cap, dcnt, dlist, ddrop, ctx->d_err, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "list launch failed");
    down(ctx, cnt, dcnt, n);
    down(ctx, list, dlist, (size_t)n * cap);
    int drop = 0;
    down(ctx, &drop, ddrop, 1);
    int r = ctx->sync_check("neighbour list");
    if (dropped) *dropped = drop;
    return r;
}

}  // namespace

extern "C" int fmd_ctx_set_precision(fmd_ctx* ctx, int precision) {
    if (!ctx) return FMD_ERR_ARG;
    if (precision != FMD_PREC_FP64 && precision != FMD_PREC_FP32_PAIR)
        return ctx->fail(FMD_ERR_ARG, "fmd_ctx_set_precision: unknown precision");
    ctx->precision = precision;
    return FMD_OK;
}

extern "C" int fmd_mat_inv9(fmd_ctx* ctx, const double* h, double* hi) {
    if (!ctx || !h || !hi) return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_mat_inv9: null") : FMD_ERR_ARG;
    // {h, hi}: the slot holds 18 doubles, the kernel writes hi into [9, 18)
    double* hh;
    int rc = up<double>(ctx, S_HH, nullptr, 18, &hh);
    if (rc) return rc;
    if (cudaMemcpyAsync(hh, h, sizeof(double) * 9, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "host to device copy failed");
    if (inv9_launch(hh, ctx->stream) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "launch failed");
    down(ctx, hi, hh + 9, 9);
    return ctx->sync_check("mat_inv9");
}

extern "C" int fmd_apply_pbc(fmd_ctx* ctx, double* pos, const double* h, const double* hi, int n) {
    if (!ctx || !pos || !h || !hi || n < 0) return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_apply_pbc: bad argument") : FMD_ERR_ARG;
    if (n == 0) return FMD_OK;
    double *dpos, *hh;
    int rc = up(ctx, S_POS, pos, 3 * (size_t)n, &dpos);
    if (!rc) rc = upload_cell(ctx, h, hi, &hh);
    if (rc) return rc;
    if (apply_pbc_launch(dpos, n, hh, ctx->stream) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "launch failed");
    down(ctx, pos, dpos, 3 * (size_t)n);
    return ctx->sync_check("apply_pbc");
}

extern "C" int fmd_nlist_rigid(fmd_ctx* ctx, const double* pos, const double* h, const double* hi, int n,
                               double rmcut, int max_neigh, int* nl_count, int* nl_list, int* dropped) {
    return list_call(ctx, LIST_SYM, pos, h, hi, n, nullptr, rmcut + 3.0, max_neigh, nl_count, nl_list, dropped);
}

extern "C" int fmd_nlist_lj_half(fmd_ctx* ctx, const double* pos, const double* h, const double* hi, int na,
                                 const int* mol_id, double rc_list, int max_neigh, int* nlc, int* nll,
                                 int* dropped) {
    return list_call(ctx, LIST_HALF, pos, h, hi, na, mol_id, rc_list, max_neigh, nlc, nll, dropped);
}

extern "C" int fmd_nlist_rebo(fmd_ctx* ctx, const double* pos, const double* h, const double* hi, int na,
                              const int* mol_id, double rc, int max_neigh, int* nlc, int* nll, int* dropped) {
    return list_call(ctx, LIST_INTRA, pos, h, hi, na, mol_id, rc, max_neigh, nlc, nll, dropped);
}

namespace {

// Every count in [0, cap] and every listed index in [0, n): caller-supplied
// lists index device arrays, so they are checked before any launch.
bool list_ok(fmd_ctx* ctx, const int* cnt, const int* list, int cap, int n, const char* what) {
    for (int i = 0; i < n; i++) {
        const int c = cnt[i];
        if (c < 0 || c > cap) {
            ctx->fail(FMD_ERR_ARG, std::string(what) + ": count out of range at row " + std::to_string(i));
            return false;
        }
        const int* row = list + (size_t)i * cap;
        for (int k = 0; k < c; k++)
            if (row[k] < 0 || row[k] >= n) {
                ctx->fail(FMD_ERR_ARG, std::string(what) + ": index out of range at row " + std::to_string(i));
                return false;
            }
    }
    return true;
}

bool index_ok(const int* a, int m, int n) {
    for (int k = 0; k < m; k++)
        if (a[k] < 0 || a[k] >= n) return false;
    return true;
}

bool topo_index_ok(const fmd_mm_topology* t, int na) {
    return index_ok(t->b_i0, t->nb, na) && index_ok(t->b_i1, t->nb, na) && index_ok(t->ang_i0, t->nang, na) &&
           index_ok(t->ang_i1, t->nang, na) && index_ok(t->ang_i2, t->nang, na) &&
           index_ok(t->dih_i0, t->ndih, na) && index_ok(t->dih_i1, t->ndih, na) &&
           index_ok(t->dih_i2, t->ndih, na) && index_ok(t->dih_i3, t->ndih, na) &&
           index_ok(t->imp_i0, t->nimp, na) && index_ok(t->imp_i1, t->nimp, na) &&
           index_ok(t->imp_i2, t->nimp, na) && index_ok(t->imp_i3, t->nimp, na);
}

// Uploads a reference-layout list and its transpose for the LJ gather.
int upload_half_list(fmd_ctx* ctx, const int* nlc, const int* nll, int cap, int na, StepArrays& a) {
    if (!list_ok(ctx, nlc, nll, cap, na, "LJ list")) return FMD_ERR_ARG;
    int *dc, *dl, *ic, *il;
    int rc = up(ctx, S_CNT, nlc, na, &dc);
    if (!rc) rc = up(ctx, S_LIST, nll, (size_t)na * cap, &dl);
    if (!rc) rc = up<int>(ctx, S_INCNT, nullptr, na, &ic);
    if (!rc) rc = up<int>(ctx, S_INLIST, nullptr, (size_t)na * (kInCap + cap), &il);
    if (rc) return rc;
    if (nlist_transpose(dc, dl, cap, na, ic, il, kInCap + cap, ctx->d_err, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "transpose launch failed");
    a.cnt_a = dc; a.list_a = dl; a.cap_a = cap; a.in_cnt = ic; a.in_list = il; a.in_cap = kInCap + cap;
    return FMD_OK;
}

// Scalars block with h, hi, W9 (and optionally npt) preloaded.
int upload_scal(fmd_ctx* ctx, const double* h, const double* hi, const double* W9, const fmd_npt* npt,
                SysScal** S) {
    void* p;
    int rc = ctx->need(S_SCAL, sizeof(SysScal), &p);
    if (rc) return rc;
    SysScal s;
    std::memset(&s, 0, sizeof(s));
    if (h) std::memcpy(s.h, h, sizeof(double) * 9);
    if (hi) std::memcpy(s.hi, hi, sizeof(double) * 9);
    if (W9) std::memcpy(s.W9, W9, sizeof(double) * 9);
    if (npt) s.npt = *npt;
    if (cudaMemcpy(p, &s, sizeof(s), cudaMemcpyHostToDevice) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "scalar upload failed");
    *S = (SysScal*)p;
    return FMD_OK;
}

int alloc_partials(fmd_ctx* ctx, StepArrays& a) {
    int rc = up<double>(ctx, S_PART1, nullptr, (size_t)std::max(kForceBlocks, a.n) * kNV, &a.part_f1);
    if (!rc) rc = up<double>(ctx, S_PART2, nullptr, (size_t)kLJMaxBlocks * kNV, &a.part_f2);
    a.lj_blocks = lj_gather_blocks(a.kind == FMD_SYS_MM ? FMD_FF_MM : FMD_FF_AIREBO, a.precision, a.lj_shape, 0);
    if (!rc) rc = up<double>(ctx, S_PART3, nullptr, (size_t)kForceBlocks, &a.part_f3);
    if (!rc) rc = up<double>(ctx, S_PARTKE, nullptr, (size_t)kForceBlocks * 2, &a.part_ke);
    return rc;
}

int zeros(fmd_ctx* ctx, int slot, size_t count, double** p) {
    int rc = up<double>(ctx, slot, nullptr, count, p);
    if (rc) return rc;
    cudaMemsetAsync(*p, 0, sizeof(double) * count, ctx->stream);
    return FMD_OK;
}

int fetch_scal(fmd_ctx* ctx, const SysScal* S, SysScal* out) {
    if (cudaMemcpyAsync(out, S, sizeof(SysScal), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "scalar copy failed");
    return FMD_OK;
}

int upload_topo(fmd_ctx* ctx, const fmd_mm_topology* t, MMTopoDev& d) {
    int s = S_TOPO0, rc = 0;
    int *i0, *i1, *i2, *i3, *mu;
    double *x0, *x1, *x2;
    d.nb = t->nb; d.nang = t->nang; d.ndih = t->ndih; d.nimp = t->nimp;
    d.physical = 0;                                  // the reference's forces
    rc |= up(ctx, s++, t->b_i0, t->nb, &i0); rc |= up(ctx, s++, t->b_i1, t->nb, &i1);
    rc |= up(ctx, s++, t->b_kb, t->nb, &x0); rc |= up(ctx, s++, t->b_r0, t->nb, &x1);
    if (rc) return FMD_ERR_CUDA;
    d.b_i0 = i0; d.b_i1 = i1; d.b_kb = x0; d.b_r0 = x1;
    rc |= up(ctx, s++, t->ang_i0, t->nang, &i0); rc |= up(ctx, s++, t->ang_i1, t->nang, &i1);
    rc |= up(ctx, s++, t->ang_i2, t->nang, &i2); rc |= up(ctx, s++, t->ang_kth, t->nang, &x0);
    rc |= up(ctx, s++, t->ang_th0, t->nang, &x1);
    if (rc) return FMD_ERR_CUDA;
    d.a_i0 = i0; d.a_i1 = i1; d.a_i2 = i2; d.a_kth = x0; d.a_th0 = x1;
    rc |= up(ctx, s++, t->dih_i0, t->ndih, &i0); rc |= up(ctx, s++, t->dih_i1, t->ndih, &i1);
    rc |= up(ctx, s++, t->dih_i2, t->ndih, &i2); rc |= up(ctx, s++, t->dih_i3, t->ndih, &i3);
    rc |= up(ctx, s++, t->dih_vn, t->ndih, &x0); rc |= up(ctx, s++, t->dih_mult, t->ndih, &mu);
    rc |= up(ctx, s++, t->dih_gamma, t->ndih, &x2);
    if (rc) return FMD_ERR_CUDA;
    d.d_i0 = i0; d.d_i1 = i1; d.d_i2 = i2; d.d_i3 = i3; d.d_vn = x0; d.d_mult = mu; d.d_gamma = x2;
    rc |= up(ctx, s++, t->imp_i0, t->nimp, &i0); rc |= up(ctx, s++, t->imp_i1, t->nimp, &i1);
    rc |= up(ctx, s++, t->imp_i2, t->nimp, &i2); rc |= up(ctx, s++, t->imp_i3, t->nimp, &i3);
    rc |= up(ctx, s++, t->imp_ki, t->nimp, &x0); rc |= up(ctx, s++, t->imp_gamma, t->nimp, &x1);
    if (rc) return FMD_ERR_CUDA;
    d.m_i0 = i0; d.m_i1 = i1; d.m_i2 = i2; d.m_i3 = i3; d.m_ki = x0; d.m_gamma = x1;
    return FMD_OK;
}

bool topo_ok(const fmd_mm_topology* t) {
    if (!t || t->nb < 0 || t->nang < 0 || t->ndih < 0 || t->nimp < 0) return false;
    if (t->nb && (!t->b_i0 || !t->b_i1 || !t->b_kb || !t->b_r0)) return false;
    if (t->nang && (!t->ang_i0 || !t->ang_i1 || !t->ang_i2 || !t->ang_kth || !t->ang_th0)) return false;
    if (t->ndih && (!t->dih_i0 || !t->dih_i1 || !t->dih_i2 || !t->dih_i3 || !t->dih_vn || !t->dih_mult ||
                    !t->dih_gamma))
        return false;
    if (t->nimp && (!t->imp_i0 || !t->imp_i1 || !t->imp_i2 || !t->imp_i3 || !t->imp_ki || !t->imp_gamma))
        return false;
    return true;
}

}  // namespace

extern "C" int fmd_lj_rigid_forces(fmd_ctx* ctx, const double* pos, const double* qv, const double* body,
                                   const double* h, const double* hi, const int* nl_count, const int* nl_list,
                                   int max_neigh, int n, int natom, double rmcut2, int precision, double* Fv,
                                   double* Tv, double* Wm9, double* Ep) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !qv || !body || !h || !hi || !nl_count || !nl_list || !Fv || !Tv || !Wm9 || !Ep || n < 1 ||
        natom < 1 || natom > 96 || max_neigh < 1)
        return ctx->fail(FMD_ERR_ARG, "fmd_lj_rigid_forces: bad argument");
    if (!list_ok(ctx, nl_count, nl_list, max_neigh, n, "molecule list")) return FMD_ERR_ARG;
    StepArrays a;
    a.precision = ctx->precision;
    a.kind = FMD_SYS_RIGID; a.n = n; a.natom = natom; a.rmcut2 = rmcut2; a.precision = precision;
    if (up<double>(ctx, S_RLAB, nullptr, (size_t)n * natom * kRigidLabDoubles, &a.rigid_lab)) return FMD_ERR_CUDA;
    double *dpos, *dq, *db, *dF, *dT;
    int *dc, *dl;
    int rc = up(ctx, S_POS, pos, 3 * (size_t)n, &dpos);
    if (!rc) rc = up(ctx, S_QV, qv, 4 * (size_t)n, &dq);
    if (!rc) rc = up(ctx, S_BODY, body, 3 * (size_t)natom, &db);
    if (!rc) rc = up(ctx, S_CNT, nl_count, n, &dc);
    if (!rc) rc = up(ctx, S_LIST, nl_list, (size_t)n * max_neigh, &dl);
    if (!rc) rc = up<double>(ctx, S_F, nullptr, 3 * (size_t)n, &dF);
    if (!rc) rc = up<double>(ctx, S_T, nullptr, 3 * (size_t)n, &dT);
    if (!rc) rc = alloc_partials(ctx, a);
    SysScal* S;
    if (!rc) rc = upload_scal(ctx, h, hi, nullptr, nullptr, &S);
    if (rc) return rc;
    a.pos = dpos; a.qv = dq; a.body = db; a.cnt_a = dc; a.list_a = dl; a.cap_a = max_neigh; a.F = dF; a.T = dT; a.S = S;
    if (enqueue_forces(a, ctx->stream) != cudaSuccess || enqueue_force_reduce(a, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "rigid force launch failed");
    SysScal out;
    down(ctx, Fv, dF, 3 * (size_t)n);
    down(ctx, Tv, dT, 3 * (size_t)n);
    fetch_scal(ctx, S, &out);
    rc = ctx->sync_check("rigid forces");
    if (rc) return rc;
    std::memcpy(Wm9, out.W9, sizeof(double) * 9);
    *Ep = out.E[0];
    return FMD_OK;
}

// REBO or LJ alone, adding into F/vir9 like the reference routines.
static int atom_term(fmd_ctx* ctx, int term, int ff, const double* pos, const double* h, const double* hi,
                     const int* nlc, const int* nll, int max_neigh, int na, double* F, double* vir9, double* E) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !h || !hi || !nlc || !nll || !F || !vir9 || !E || na < 1 || max_neigh < 1)
        return ctx->fail(FMD_ERR_ARG, "force term: bad argument");
    StepArrays a;
    a.precision = ctx->precision;
    a.n = na;
    double *dpos, *dF, *dFacc, *hh;
    int rc = up(ctx, S_POS, pos, 3 * (size_t)na, &dpos);
    if (!rc) rc = upload_cell(ctx, h, hi, &hh);
    if (!rc) rc = up(ctx, S_F, F, 3 * (size_t)na, &dF);
    if (!rc) rc = zeros(ctx, S_FACC, 3 * (size_t)na, &dFacc);
    if (!rc) rc = alloc_partials(ctx, a);
    if (rc) return rc;
    double* part = a.part_f1;
    if (term == 0) {
        int *dc, *dl;
        if (!list_ok(ctx, nlc, nll, max_neigh, na, "REBO list")) return FMD_ERR_ARG;
        rc = up(ctx, S_CNT2, nlc, na, &dc);
        if (!rc) rc = up(ctx, S_LIST2, nll, (size_t)na * max_neigh, &dl);
        if (rc) return rc;
        double* slots;
        if ((rc = up<double>(ctx, S_RSLOT, nullptr, (size_t)na * max_neigh * kReboSlotDoubles, &slots))) return rc;
        if (rebo_slots_launch(dpos, hh, dc, dl, max_neigh, na, slots, dF, part, kForceBlocks, nullptr, 0,
                              ctx->stream) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "rebo launch failed");
    } else {
        if ((rc = upload_half_list(ctx, nlc, nll, max_neigh, na, a))) return rc;
        // F += LJ: fold the caller's F through the accumulator.
        if (cudaMemcpyAsync(dFacc, dF, sizeof(double) * 3 * na, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "copy failed");
        if (lj_gather_launch(ff, dpos, hh, a.cnt_a, a.list_a, a.cap_a, a.in_cnt, a.in_list, a.in_cap, na, dF, dFacc,
                             part, ctx->stream, ctx->precision) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "lj launch failed");
    }
    double* red;
    if ((rc = up<double>(ctx, S_PART3, nullptr, 16, &red))) return rc;
    if (reduce_partials(part, term == 0 ? kForceBlocks : lj_gather_blocks(ff, ctx->precision, LJShape{}, 0), kNV, red,
                        ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "reduce launch failed");
    double r[kNV];
    down(ctx, F, dF, 3 * (size_t)na);
    down(ctx, r, red, kNV);
    rc = ctx->sync_check(term == 0 ? "rebo forces" : "lj forces");
    if (rc) return rc;
    *E = r[0];
    for (int q = 0; q < 9; q++) vir9[q] += r[1 + q];
    return FMD_OK;
}

extern "C" int fmd_rebo_forces(fmd_ctx* ctx, const double* pos, const double* h, const double* hi, const int* nlc,
                               const int* nll, int max_neigh, int na, double* F, double* vir9, double* E) {
    return atom_term(ctx, 0, FMD_FF_AIREBO, pos, h, hi, nlc, nll, max_neigh, na, F, vir9, E);
}

extern "C" int fmd_lj_half_forces(fmd_ctx* ctx, int ff, const double* pos, const double* h, const double* hi,
                                  const int* nlc, const int* nll, int max_neigh, int na, double* F, double* vir9,
                                  double* E) {
    if (ff != FMD_FF_AIREBO && ff != FMD_FF_MM)
        return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_lj_half_forces: unknown force field") : FMD_ERR_ARG;
    return atom_term(ctx, 1, ff, pos, h, hi, nlc, nll, max_neigh, na, F, vir9, E);
}

namespace {

// REBO-II tables of one host call: the knots expanded into per-cell
// coefficients and uploaded, and the coordination scratch.
int rebo2_tables(fmd_ctx* ctx, const fmd_rebo2_knots* kn, int na, int cap_b, Rebo2Dev& t) {
    static_assert(sizeof(fmd_rebo2_knots) == sizeof(double) * kRebo2Knots, "knot layout");
    std::vector<double> c(kRebo2PccCoef + 2 * (size_t)kRebo2TriCoef);
    rebo2_coeffs(&kn->pcc[0][0], c.data(), c.data() + kRebo2PccCoef, c.data() + kRebo2PccCoef + kRebo2TriCoef);
    double *tab, *nc;
    int2 *bonds, *pairs;
    int* counts;
    int rc = up(ctx, S_R2TAB, c.data(), c.size(), &tab);
    if (!rc) rc = up<double>(ctx, S_R2NC, nullptr, (size_t)na, &nc);
    if (!rc) rc = up<int2>(ctx, S_R2BOND, nullptr, (size_t)na * cap_b, &bonds);
    if (!rc) rc = up<int2>(ctx, S_R2PAIR, nullptr, (size_t)na * kRebo2SwitchPerAtom, &pairs);
    if (!rc) rc = up<int>(ctx, S_R2CNT, nullptr, 2, &counts);
    if (rc) return rc;
    t.pcc = tab;
    t.pirc = tab + kRebo2PccCoef;
    t.tcc = tab + kRebo2PccCoef + kRebo2TriCoef;
    t.ncoord = nc;
    t.bonds = bonds;
    t.sw_pairs = pairs;
    t.counts = counts;
    t.sw_cap = na * kRebo2SwitchPerAtom;
    t.err = ctx->d_err;
    // the staging vector dies at return: finish the copy first
    return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? FMD_OK
                                                             : ctx->fail(FMD_ERR_CUDA, "table upload failed");
}

// Reduces nblk {E, W9} partial records, adds the virial into vir9 and copies
// the forces back.
int finish_term(fmd_ctx* ctx, const double* part, int nblk, const double* dF, double* F, int na, double* vir9,
                double* E, const char* what) {
    double* red;
    int rc = up<double>(ctx, S_PART3, nullptr, 16, &red);
    if (rc) return rc;
    if (reduce_partials(part, nblk, kNV, red, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "reduce launch failed");
    double r[kNV];
    down(ctx, F, dF, 3 * (size_t)na);
    down(ctx, r, red, kNV);
    if ((rc = ctx->sync_check(what))) return rc;
    *E = r[0];
    for (int q = 0; q < 9; q++) vir9[q] += r[1 + q];
    return FMD_OK;
}

}  // namespace

extern "C" int fmd_rebo2_coeffs(const fmd_rebo2_knots* kn, double* out) {
    if (!kn || !out) return FMD_ERR_ARG;
    rebo2_coeffs(&kn->pcc[0][0], out, out + kRebo2PccCoef, out + kRebo2PccCoef + kRebo2TriCoef);
    return FMD_OK;
}

extern "C" int fmd_rebo2_forces(fmd_ctx* ctx, const double* pos, const double* h, const double* hi, const int* nlc,
                                const int* nll, int max_neigh, int na, const fmd_rebo2_knots* kn, double* F,
                                double* vir9, double* E) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !h || !hi || !nlc || !nll || !kn || !F || !vir9 || !E || na < 1 || max_neigh < 1)
        return ctx->fail(FMD_ERR_ARG, "fmd_rebo2_forces: bad argument");
    if (!list_ok(ctx, nlc, nll, max_neigh, na, "REBO list")) return FMD_ERR_ARG;
    double *dpos, *hh, *dF, *part;
    int *dc, *dl;
    Rebo2Dev t;
    int rc = up(ctx, S_POS, pos, 3 * (size_t)na, &dpos);
    if (!rc) rc = upload_cell(ctx, h, hi, &hh);
    if (!rc) rc = up(ctx, S_F, F, 3 * (size_t)na, &dF);
    if (!rc) rc = up(ctx, S_CNT2, nlc, na, &dc);
    if (!rc) rc = up(ctx, S_LIST2, nll, (size_t)na * max_neigh, &dl);
    if (!rc) rc = up<double>(ctx, S_PART1, nullptr, (size_t)kForceBlocks * kNV, &part);
    if (!rc) rc = rebo2_tables(ctx, kn, na, max_neigh, t);
    if (rc) return rc;
    if (rebo2_launch(t, dpos, hh, dc, dl, max_neigh, na, dF, part, kForceBlocks, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "rebo2 launch failed");
    return finish_term(ctx, part, kForceBlocks, dF, F, na, vir9, E, "rebo2 forces");
}

extern "C" int fmd_lj_switch_forces(fmd_ctx* ctx, const double* pos, const double* h, const double* hi,
                                    const int* nlc_r, const int* nll_r, int max_neigh_r, const int* nlc_l,
                                    const int* nll_l, int max_neigh_l, int na, const fmd_rebo2_knots* kn, double* F,
                                    double* vir9, double* E) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !h || !hi || !nlc_r || !nll_r || !nlc_l || !nll_l || !kn || !F || !vir9 || !E || na < 1 ||
        max_neigh_r < 1 || max_neigh_l < 1)
        return ctx->fail(FMD_ERR_ARG, "fmd_lj_switch_forces: bad argument");
    if (!list_ok(ctx, nlc_r, nll_r, max_neigh_r, na, "REBO list") ||
        !list_ok(ctx, nlc_l, nll_l, max_neigh_l, na, "LJ list"))
        return FMD_ERR_ARG;
    double *dpos, *hh, *dF, *part;
    int *dcr, *dlr, *dcl, *dll;
    Rebo2Dev t;
    int rc = up(ctx, S_POS, pos, 3 * (size_t)na, &dpos);
    if (!rc) rc = upload_cell(ctx, h, hi, &hh);
    if (!rc) rc = up(ctx, S_F, F, 3 * (size_t)na, &dF);
    if (!rc) rc = up(ctx, S_CNT2, nlc_r, na, &dcr);
    if (!rc) rc = up(ctx, S_LIST2, nll_r, (size_t)na * max_neigh_r, &dlr);
    if (!rc) rc = up(ctx, S_CNT, nlc_l, na, &dcl);
    if (!rc) rc = up(ctx, S_LIST, nll_l, (size_t)na * max_neigh_l, &dll);
    if (!rc) rc = up<double>(ctx, S_PART1, nullptr, (size_t)kForceBlocks * kNV, &part);
    if (!rc) rc = rebo2_tables(ctx, kn, na, max_neigh_r, t);
    if (rc) return rc;
    if (lj_switch_launch(t, dpos, hh, dcr, dlr, max_neigh_r, dcl, dll, max_neigh_l, na, dF, part, kForceBlocks,
                         false, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "lj switch launch failed");
    return finish_term(ctx, part, kForceBlocks, dF, F, na, vir9, E, "lj switch forces");
}

namespace {

// Shared set-up of the atomistic force/step entry points.
int atom_setup(fmd_ctx* ctx, int kind, const double* pos, const double* h, const double* hi, const double* W9,
               const fmd_npt* npt, int na, StepArrays& a) {
    a.kind = kind;
    a.n = na;
    double *dpos, *dF, *dFacc;
    int rc = up(ctx, S_POS, pos, 3 * (size_t)na, &dpos);
    if (!rc) rc = zeros(ctx, S_F, 3 * (size_t)na, &dF);
    if (!rc) rc = zeros(ctx, S_FACC, 3 * (size_t)na, &dFacc);
    if (!rc) rc = alloc_partials(ctx, a);
    SysScal* S;
    if (!rc) rc = upload_scal(ctx, h, hi, W9, npt, &S);
    if (rc) return rc;
    a.pos = dpos; a.F = dF; a.Facc = dFacc; a.S = S;
    return FMD_OK;
}

int airebo_lists(fmd_ctx* ctx, const int* nlc_r, const int* nll_r, const int* nlc_l, const int* nll_l, int na,
                 StepArrays& a) {
    int *dc, *dl;
    if (!list_ok(ctx, nlc_r, nll_r, 12, na, "REBO list")) return FMD_ERR_ARG;
    int rc = up(ctx, S_CNT2, nlc_r, na, &dc);
    if (!rc) rc = up(ctx, S_LIST2, nll_r, (size_t)na * 12, &dl);
    if (rc) return rc;
    a.cnt_b = dc; a.list_b = dl; a.cap_b = 12;
    if ((rc = up<double>(ctx, S_RSLOT, nullptr, (size_t)na * 12 * kReboSlotDoubles, &a.rebo_slots))) return rc;
    return upload_half_list(ctx, nlc_l, nll_l, 400, na, a);
}

}  // namespace

extern "C" int fmd_airebo_forces(fmd_ctx* ctx, const double* pos, const double* h, const double* hi,
                                 const int* nlc_r, const int* nll_r, const int* nlc_l, const int* nll_l, int na,
                                 double* F, double* vir9, double* E3) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !h || !hi || !nlc_r || !nll_r || !nlc_l || !nll_l || !F || !vir9 || !E3 || na < 1)
        return ctx->fail(FMD_ERR_ARG, "fmd_airebo_forces: bad argument");
    StepArrays a;
    a.precision = ctx->precision;
    int rc = atom_setup(ctx, FMD_SYS_AIREBO, pos, h, hi, nullptr, nullptr, na, a);
    if (!rc) rc = airebo_lists(ctx, nlc_r, nll_r, nlc_l, nll_l, na, a);
    if (rc) return rc;
    if (enqueue_forces(a, ctx->stream) != cudaSuccess || enqueue_force_reduce(a, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "airebo force launch failed");
    SysScal out;
    down(ctx, F, a.F, 3 * (size_t)na);
    fetch_scal(ctx, a.S, &out);
    if ((rc = ctx->sync_check("airebo forces"))) return rc;
    std::memcpy(vir9, out.W9, sizeof(double) * 9);
    E3[0] = out.E[0]; E3[1] = out.E[1]; E3[2] = out.E[2];
    return FMD_OK;
}

extern "C" int fmd_mm_forces(fmd_ctx* ctx, const fmd_mm_topology* t, const double* pos, const double* h,
                             const double* hi, const int* nlc, const int* nll, const double* charge,
                             const int* mol_id, int has_charge, int na, double* F, double* vir9, double* E7) {
    if (!ctx) return FMD_ERR_ARG;
    if (!topo_ok(t) || !pos || !h || !hi || !nlc || !nll || !F || !vir9 || !E7 || na < 1 ||
        (has_charge && (!charge || !mol_id)) || !topo_index_ok(t, na))
        return ctx->fail(FMD_ERR_ARG, "fmd_mm_forces: bad argument");
    StepArrays a;
    a.precision = ctx->precision;
    int rc = atom_setup(ctx, FMD_SYS_MM, pos, h, hi, nullptr, nullptr, na, a);
    if (!rc) rc = upload_half_list(ctx, nlc, nll, 400, na, a);
    if (!rc) rc = upload_topo(ctx, t, a.topo);
    if (!rc && has_charge) {
        double* q; int* m;
        rc = up(ctx, S_CHARGE, charge, na, &q);
        if (!rc) rc = up(ctx, S_MOL, mol_id, na, &m);
        a.charge = q; a.mol_id = m; a.has_charge = 1;
    }
    if (rc) return rc;
    if (enqueue_forces(a, ctx->stream) != cudaSuccess || enqueue_force_reduce(a, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "mm force launch failed");
    SysScal out;
    down(ctx, F, a.F, 3 * (size_t)na);
    fetch_scal(ctx, a.S, &out);
    if ((rc = ctx->sync_check("mm forces"))) return rc;
    std::memcpy(vir9, out.W9, sizeof(double) * 9);
    for (int q = 0; q < 7; q++) E7[q] = out.E[q];
    return FMD_OK;
}

// ------------------------------------------------------------ host steps --
namespace {
StepParams plain_params(double dt) {
    StepParams p;
    p.dt = dt;
    p.schedule = 0;
    return p;
}
}  // namespace

extern "C" int fmd_rigid_step(fmd_ctx* ctx, double* pos, double* vel, double* qv, double* omg, double* Fv,
                              double* Tv, double* Wm9, double* h, double* hi, const double* body, double I0,
                              double Mmol, int n, int natom, double rmcut2, double dt, fmd_npt* npt,
                              const int* nl_count, const int* nl_list, int max_neigh, int precision, double* out2) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !vel || !qv || !omg || !Fv || !Tv || !Wm9 || !h || !hi || !body || !npt || !nl_count ||
        !nl_list || !out2 || n < 1 || natom < 1 || natom > 96 || max_neigh < 1)
        return ctx->fail(FMD_ERR_ARG, "fmd_rigid_step: bad argument");
    if (!list_ok(ctx, nl_count, nl_list, max_neigh, n, "molecule list")) return FMD_ERR_ARG;
    StepArrays a;
    a.precision = ctx->precision;
    a.kind = FMD_SYS_RIGID; a.n = n; a.natom = natom; a.rmcut2 = rmcut2; a.Mmol = Mmol; a.I0 = I0;
    if (up<double>(ctx, S_RLAB, nullptr, (size_t)n * natom * kRigidLabDoubles, &a.rigid_lab)) return FMD_ERR_CUDA;
    a.precision = precision;
    double *dpos, *dvel, *dq, *dw, *dF, *dT, *db;
    int *dc, *dl;
    int rc = up(ctx, S_POS, pos, 3 * (size_t)n, &dpos);
    if (!rc) rc = up(ctx, S_VEL, vel, 3 * (size_t)n, &dvel);
    if (!rc) rc = up(ctx, S_QV, qv, 4 * (size_t)n, &dq);
    if (!rc) rc = up(ctx, S_OMG, omg, 3 * (size_t)n, &dw);
    if (!rc) rc = up(ctx, S_F, Fv, 3 * (size_t)n, &dF);
    if (!rc) rc = up(ctx, S_T, Tv, 3 * (size_t)n, &dT);
    if (!rc) rc = up(ctx, S_BODY, body, 3 * (size_t)natom, &db);
    if (!rc) rc = up(ctx, S_CNT, nl_count, n, &dc);
    if (!rc) rc = up(ctx, S_LIST, nl_list, (size_t)n * max_neigh, &dl);
    if (!rc) rc = alloc_partials(ctx, a);
    SysScal* S;
    if (!rc) rc = upload_scal(ctx, h, hi, Wm9, npt, &S);
    if (rc) return rc;
    a.pos = dpos; a.vel = dvel; a.qv = dq; a.omg = dw; a.F = dF; a.T = dT; a.body = db;
    a.cnt_a = dc; a.list_a = dl; a.cap_a = max_neigh; a.S = S;
    if (enqueue_ke(a, ctx->stream) != cudaSuccess || enqueue_step(a, plain_params(dt), false, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "rigid step launch failed");
    SysScal out;
    down(ctx, pos, dpos, 3 * (size_t)n); down(ctx, vel, dvel, 3 * (size_t)n);
    down(ctx, qv, dq, 4 * (size_t)n); down(ctx, omg, dw, 3 * (size_t)n);
    down(ctx, Fv, dF, 3 * (size_t)n); down(ctx, Tv, dT, 3 * (size_t)n);
    fetch_scal(ctx, S, &out);
    if ((rc = ctx->sync_check("rigid step"))) return rc;
    std::memcpy(Wm9, out.W9, sizeof(double) * 9);
    std::memcpy(h, out.h, sizeof(double) * 9);
    std::memcpy(hi, out.hi, sizeof(double) * 9);
    *npt = out.npt;
    out2[0] = out.E[0];
    out2[1] = out.KE;
    return FMD_OK;
}

extern "C" int fmd_airebo_step(fmd_ctx* ctx, double* pos, double* vel, double* F, double* vir9, double* h,
                               double* hi, const double* mass, int na, double dt, fmd_npt* npt, const int* nlc_r,
                               const int* nll_r, const int* nlc_l, const int* nll_l, double* out4) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !vel || !F || !vir9 || !h || !hi || !mass || !npt || !nlc_r || !nll_r || !nlc_l || !nll_l ||
        !out4 || na < 1)
        return ctx->fail(FMD_ERR_ARG, "fmd_airebo_step: bad argument");
    StepArrays a;
    a.precision = ctx->precision;
    int rc = atom_setup(ctx, FMD_SYS_AIREBO, pos, h, hi, vir9, npt, na, a);
    double *dvel, *dm;
    if (!rc) rc = up(ctx, S_VEL, vel, 3 * (size_t)na, &dvel);
    if (!rc) rc = up(ctx, S_MASS, mass, na, &dm);
    if (!rc && cudaMemcpyAsync(a.F, F, sizeof(double) * 3 * na, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        rc = ctx->fail(FMD_ERR_CUDA, "copy failed");
    if (!rc) rc = airebo_lists(ctx, nlc_r, nll_r, nlc_l, nll_l, na, a);
    if (rc) return rc;
    a.vel = dvel; a.mass = dm;
    if (enqueue_ke(a, ctx->stream) != cudaSuccess || enqueue_step(a, plain_params(dt), false, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "airebo step launch failed");
    SysScal out;
    down(ctx, pos, a.pos, 3 * (size_t)na); down(ctx, vel, dvel, 3 * (size_t)na); down(ctx, F, a.F, 3 * (size_t)na);
    fetch_scal(ctx, a.S, &out);
    if ((rc = ctx->sync_check("airebo step"))) return rc;
    std::memcpy(vir9, out.W9, sizeof(double) * 9);
    std::memcpy(h, out.h, sizeof(double) * 9);
    std::memcpy(hi, out.hi, sizeof(double) * 9);
    *npt = out.npt;
    out4[0] = out.E[0]; out4[1] = out.E[1]; out4[2] = out.E[2]; out4[3] = out.KE;
    return FMD_OK;
}

extern "C" int fmd_mm_step(fmd_ctx* ctx, double* pos, double* vel, double* F, double* vir9, double* h, double* hi,
                           int na, double dt, fmd_npt* npt, const fmd_mm_topology* t, const int* nlc, const int* nll,
                           const double* charge, const int* mol_id, int has_charge, double* out8) {
    if (!ctx) return FMD_ERR_ARG;
    if (!pos || !vel || !F || !vir9 || !h || !hi || !npt || !topo_ok(t) || !nlc || !nll || !out8 || na < 1 ||
        (has_charge && (!charge || !mol_id)) || !topo_index_ok(t, na))
        return ctx->fail(FMD_ERR_ARG, "fmd_mm_step: bad argument");
    StepArrays a;
    a.precision = ctx->precision;
    int rc = atom_setup(ctx, FMD_SYS_MM, pos, h, hi, vir9, npt, na, a);
    double* dvel;
    if (!rc) rc = up(ctx, S_VEL, vel, 3 * (size_t)na, &dvel);
    if (!rc && cudaMemcpyAsync(a.F, F, sizeof(double) * 3 * na, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        rc = ctx->fail(FMD_ERR_CUDA, "copy failed");
    if (!rc) rc = upload_half_list(ctx, nlc, nll, 400, na, a);
    if (!rc) rc = upload_topo(ctx, t, a.topo);
    if (!rc && has_charge) {
        double* q; int* m;
        rc = up(ctx, S_CHARGE, charge, na, &q);
        if (!rc) rc = up(ctx, S_MOL, mol_id, na, &m);
        a.charge = q; a.mol_id = m; a.has_charge = 1;
    }
    if (rc) return rc;
    a.vel = dvel;
    if (enqueue_ke(a, ctx->stream) != cudaSuccess || enqueue_step(a, plain_params(dt), false, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "mm step launch failed");
    SysScal out;
    down(ctx, pos, a.pos, 3 * (size_t)na); down(ctx, vel, dvel, 3 * (size_t)na); down(ctx, F, a.F, 3 * (size_t)na);
    fetch_scal(ctx, a.S, &out);
    if ((rc = ctx->sync_check("mm step"))) return rc;
    std::memcpy(vir9, out.W9, sizeof(double) * 9);
    std::memcpy(h, out.h, sizeof(double) * 9);
    std::memcpy(hi, out.hi, sizeof(double) * 9);
    *npt = out.npt;
    for (int q = 0; q < 7; q++) out8[q] = out.E[q];
    out8[7] = out.KE;
    return FMD_OK;
}
