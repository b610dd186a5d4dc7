// sg_abi.cu -- C-ABI of the learned bond-order potential (fmd_sg_*).
// The model owns its FP64 master parameters, their BF16/FP32 device images
// and a row workspace; the host-pointer call mirrors fmd_rebo_forces.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "fmd_internal.h"
#include "kernels.h"
#include "sg_host.h"
#include "sg_train.cuh"
#include "surrogate.cuh"
#include "umma.cuh"

namespace {

// Training state of one model (allocated on first use).
struct Trainer {
    fmd::sg::TrainWork tw;
    float* grad = nullptr;       // [GRAD_N]
    double *m = nullptr, *v = nullptr;
    double* F = nullptr;         // [3 * na] scratch
    int F_na = 0;
    double* hist = nullptr;      // [2 * steps]
    int hist_n = 0;
    long long t = 0;             // Adam step count
};

void trainer_free(Trainer& tr) {
    fmd::sg::train_free(tr.tw);
    cudaFree(tr.grad); cudaFree(tr.m); cudaFree(tr.v); cudaFree(tr.F); cudaFree(tr.hist);
    tr = Trainer{};
}

}  // namespace

struct fmd_sg {
    fmd_ctx* ctx = nullptr;
    double* P = nullptr;        // [NPARAM] master parameters (device)
    uint16_t* img = nullptr;    // [IMG_N] BF16 weight images
    float* vec = nullptr;       // [V_N]
    fmd::sg::Work work;
    // host-pointer staging
    double *pos = nullptr, *hh = nullptr, *F = nullptr, *out = nullptr;
    int *cnt = nullptr, *list = nullptr;
    int stage_na = 0, stage_cap = 0;
    int last_na = 0;
    Trainer tr;
};

namespace {

using namespace fmd;

int stage(fmd_sg* s, int na, int cap) {
    if (na <= s->stage_na && cap == s->stage_cap) return FMD_OK;
    cudaFree(s->pos); cudaFree(s->F); cudaFree(s->cnt); cudaFree(s->list);
    s->pos = s->F = nullptr;
    s->cnt = s->list = nullptr;
    if (cudaMalloc(&s->pos, sizeof(double) * 3 * (size_t)na) != cudaSuccess ||
        cudaMalloc(&s->F, sizeof(double) * 3 * (size_t)na) != cudaSuccess ||
        cudaMalloc(&s->cnt, sizeof(int) * (size_t)na) != cudaSuccess ||
        cudaMalloc(&s->list, sizeof(int) * (size_t)na * cap) != cudaSuccess) {
        s->stage_na = 0;
        return s->ctx->fail(FMD_ERR_CUDA, "fmd_sg: staging allocation failed");
    }
    s->stage_na = na;
    s->stage_cap = cap;
    return FMD_OK;
}

bool params_ok(const double* p) {
    for (int k = 0; k < sg::NPARAM; k++)
        if (!(p[k] == p[k]) || p[k] > 1e30 || p[k] < -1e30) return false;
    for (int f = 0; f < sg::D; f++)
        if (!(p[sg::OS + f] > 0.0)) return false;
    return true;
}

}  // namespace

void fmd::sg_model_images(const fmd_sg* m, const uint16_t** img, const float** vec) {
    *img = m->img;
    *vec = m->vec;
}

extern "C" int fmd_sg_nparams(void) { return fmd::sg::NPARAM; }

extern "C" int fmd_sg_set_params(fmd_sg* s, const double* params) {
    if (!s || !params) return FMD_ERR_ARG;
    if (!params_ok(params)) return s->ctx->fail(FMD_ERR_ARG, "fmd_sg_set_params: non-finite value or scale <= 0");
    FMD_CUDA_TRY(s->ctx, cudaMemcpyAsync(s->P, params, sizeof(double) * sg::NPARAM, cudaMemcpyHostToDevice,
                                         s->ctx->stream));
    FMD_CUDA_TRY(s->ctx, sg::pack_params(s->P, s->img, s->vec, s->ctx->stream));
    return s->ctx->sync_check("fmd_sg_set_params");
}

extern "C" int fmd_sg_get_params(fmd_sg* s, double* params) {
    if (!s || !params) return FMD_ERR_ARG;
    FMD_CUDA_TRY(s->ctx, cudaMemcpyAsync(params, s->P, sizeof(double) * sg::NPARAM, cudaMemcpyDeviceToHost,
                                         s->ctx->stream));
    return s->ctx->sync_check("fmd_sg_get_params");
}

extern "C" int fmd_sg_create(fmd_ctx* ctx, const double* params, fmd_sg** out) {
    if (!ctx || !params || !out) return FMD_ERR_ARG;
    *out = nullptr;
    fmd_sg* s = new fmd_sg();
    s->ctx = ctx;
    if (cudaMalloc(&s->P, sizeof(double) * sg::NPARAM) != cudaSuccess ||
        cudaMalloc(&s->img, sizeof(uint16_t) * sg::IMG_N) != cudaSuccess ||
        cudaMalloc(&s->vec, sizeof(float) * sg::V_N) != cudaSuccess ||
        cudaMalloc(&s->hh, sizeof(double) * 18) != cudaSuccess ||
        cudaMalloc(&s->out, sizeof(double) * kNV) != cudaSuccess) {
        cudaFree(s->P); cudaFree(s->img); cudaFree(s->vec); cudaFree(s->hh); cudaFree(s->out);
        delete s;
        return ctx->fail(FMD_ERR_CUDA, "fmd_sg_create: allocation failed");
    }
    const int rc = fmd_sg_set_params(s, params);
    if (rc != FMD_OK) {
        cudaFree(s->P); cudaFree(s->img); cudaFree(s->vec); cudaFree(s->hh); cudaFree(s->out);
        delete s;
        return rc;
    }
    *out = s;
    return FMD_OK;
}

// Does not touch the context (it may already be gone when a garbage
// collector destroys the model last).
extern "C" int fmd_sg_destroy(fmd_sg* s) {
    if (!s) return FMD_ERR_ARG;
    cudaDeviceSynchronize();
    sg::work_free(s->work);
    trainer_free(s->tr);
    cudaFree(s->P); cudaFree(s->img); cudaFree(s->vec); cudaFree(s->hh); cudaFree(s->out);
    cudaFree(s->pos); cudaFree(s->F); cudaFree(s->cnt); cudaFree(s->list);
    delete s;
    return FMD_OK;
}

extern "C" int fmd_sg_rebo_forces(fmd_sg* s, const double* pos, const double* h, const double* hi, const int* nlc,
                                  const int* nll, int max_neigh, int na, double* F, double* vir9, double* E) {
    if (!s || !pos || !h || !hi || !nlc || !nll || !F || !vir9 || !E || na <= 0 || max_neigh <= 0)
        return s ? s->ctx->fail(FMD_ERR_ARG, "fmd_sg_rebo_forces: bad argument") : FMD_ERR_ARG;
    fmd_ctx* ctx = s->ctx;
    for (int i = 0; i < na; i++) {
        if (nlc[i] < 0 || nlc[i] > max_neigh) return ctx->fail(FMD_ERR_ARG, "fmd_sg_rebo_forces: bad list count");
        for (int k = 0; k < nlc[i]; k++) {
            const int j = nll[(size_t)i * max_neigh + k];
            if (j < 0 || j >= na) return ctx->fail(FMD_ERR_ARG, "fmd_sg_rebo_forces: list entry out of range");
        }
    }
    int rc = stage(s, na, max_neigh);
    if (rc) return rc;
    FMD_CUDA_TRY(ctx, sg::work_alloc(s->work, na, max_neigh));
    cudaStream_t st = ctx->stream;
    double hh[18];
    std::memcpy(hh, h, sizeof(double) * 9);
    std::memcpy(hh + 9, hi, sizeof(double) * 9);
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(s->hh, hh, sizeof(hh), cudaMemcpyHostToDevice, st));
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(s->pos, pos, sizeof(double) * 3 * (size_t)na, cudaMemcpyHostToDevice, st));
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(s->cnt, nlc, sizeof(int) * (size_t)na, cudaMemcpyHostToDevice, st));
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(s->list, nll, sizeof(int) * (size_t)na * max_neigh, cudaMemcpyHostToDevice, st));
    FMD_CUDA_TRY(ctx, cudaMemsetAsync(s->F, 0, sizeof(double) * 3 * (size_t)na, st));
    FMD_CUDA_TRY(ctx, cudaMemsetAsync(s->work.err, 0, sizeof(int) * 4, st));
    FMD_CUDA_TRY(ctx, sg::rebo_forces(s->work, s->img, s->vec, s->pos, s->hh, s->cnt, s->list, max_neigh, na, s->F,
                                      s->work.part, st));
    FMD_CUDA_TRY(ctx, reduce_partials(s->work.part, sg::kRowBlocks, kNV, s->out, st));
    std::vector<double> Fh(3 * (size_t)na);
    double o[kNV];
    int err[4];
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(Fh.data(), s->F, sizeof(double) * 3 * (size_t)na, cudaMemcpyDeviceToHost, st));
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(o, s->out, sizeof(o), cudaMemcpyDeviceToHost, st));
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(err, s->work.err, sizeof(err), cudaMemcpyDeviceToHost, st));
    rc = ctx->sync_check("fmd_sg_rebo_forces");
    if (rc) return rc;
    if (err[0]) return ctx->fail(FMD_ERR_ARG, "fmd_sg_rebo_forces: REBO list is not symmetric (row without partner)");
    if (err[1]) return ctx->fail(FMD_ERR_CUDA, "fmd_sg_rebo_forces: tensor-core wait timed out");
    for (size_t k = 0; k < 3 * (size_t)na; k++) F[k] += Fh[k];
    for (int k = 0; k < 9; k++) vir9[k] += o[1 + k];
    *E = o[0];
    s->last_na = na;
    return FMD_OK;
}

// Rows of the last evaluation: count, and (any may be NULL) row_i, row_j,
// the normalised BF16 descriptors xn[rows*32] (as float), b[rows],
// gx[rows*32] = db/dxn.
extern "C" int fmd_sg_last_rows(fmd_sg* s, int cap_rows, int* nrows, int* row_i, int* row_j, float* xn, float* b,
                                float* gx) {
    if (!s || !nrows) return FMD_ERR_ARG;
    fmd_ctx* ctx = s->ctx;
    if (s->last_na == 0) return ctx->fail(FMD_ERR_STATE, "fmd_sg_last_rows: nothing evaluated yet");
    cudaStream_t st = ctx->stream;
    int R = 0;
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(&R, s->work.aoff + s->last_na, sizeof(int), cudaMemcpyDeviceToHost, st));
    int rc = ctx->sync_check("fmd_sg_last_rows");
    if (rc) return rc;
    *nrows = R;
    if (!row_i && !row_j && !xn && !b && !gx) return FMD_OK;
    if (cap_rows < R) return ctx->fail(FMD_ERR_CAPACITY, "fmd_sg_last_rows: arrays smaller than the row count");
    std::vector<int> ri(R), rs(R), cnt(s->last_na), lst((size_t)s->last_na * s->work.cap);
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(ri.data(), s->work.row_i, sizeof(int) * R, cudaMemcpyDeviceToHost, st));
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(rs.data(), s->work.row_s, sizeof(int) * R, cudaMemcpyDeviceToHost, st));
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(lst.data(), s->list, sizeof(int) * lst.size(), cudaMemcpyDeviceToHost, st));
    if (b) FMD_CUDA_TRY(ctx, cudaMemcpyAsync(b, s->work.b, sizeof(float) * R, cudaMemcpyDeviceToHost, st));
    if (gx) FMD_CUDA_TRY(ctx, cudaMemcpyAsync(gx, s->work.gx, sizeof(float) * R * sg::D, cudaMemcpyDeviceToHost, st));
    std::vector<uint16_t> X;
    if (xn) {
        const size_t nt = ((size_t)R + sg::TILE - 1) / sg::TILE;
        X.resize(nt * sg::TILE * sg::D);
        FMD_CUDA_TRY(ctx, cudaMemcpyAsync(X.data(), s->work.X, sizeof(uint16_t) * X.size(), cudaMemcpyDeviceToHost, st));
    }
    rc = ctx->sync_check("fmd_sg_last_rows");
    if (rc) return rc;
    for (int r = 0; r < R; r++) {
        if (row_i) row_i[r] = ri[r];
        if (row_j) row_j[r] = lst[(size_t)ri[r] * s->work.cap + rs[r]];
        if (xn) {
            const unsigned char* tile = reinterpret_cast<const unsigned char*>(X.data()) +
                                        (size_t)(r / sg::TILE) * sg::TILE * sg::D * 2;
            for (int f = 0; f < sg::D; f++) {
                uint16_t bits;
                std::memcpy(&bits, tile + umma::il_off(r % sg::TILE, f, sg::D), 2);
                const uint32_t u = (uint32_t)bits << 16;
                float v;
                std::memcpy(&v, &u, 4);
                xn[(size_t)r * sg::D + f] = v;
            }
        }
    }
    return FMD_OK;
}

// ------------------------------------------------------------------ training

namespace {

struct Snap {
    int na = 0, cap = 0;
    double *pos = nullptr, *hh = nullptr, *Fref = nullptr, *ref10 = nullptr;
    int *cnt = nullptr, *list = nullptr;
};

void snap_free(Snap& s) {
    cudaFree(s.pos); cudaFree(s.hh); cudaFree(s.Fref); cudaFree(s.ref10); cudaFree(s.cnt); cudaFree(s.list);
    s = Snap{};
}

}  // namespace

struct fmd_sg_data {
    fmd_ctx* ctx = nullptr;
    std::vector<Snap> snaps;
    double* part = nullptr;   // plain REBO partials (kForceBlocks records)
};

// Copies a snapshot that is already on the device and computes its reference
// REBO energy, forces and virial with the plain REBO kernel.
int fmd::sg_data_add_device(fmd_sg_data* d, const double* pos, const double* hh, const int* cnt, const int* list,
                            int cap, int na, cudaStream_t st) {
    fmd_ctx* ctx = d->ctx;
    Snap s;
    s.na = na;
    s.cap = cap;
    if (cudaMalloc(&s.pos, sizeof(double) * 3 * (size_t)na) != cudaSuccess ||
        cudaMalloc(&s.hh, sizeof(double) * 18) != cudaSuccess ||
        cudaMalloc(&s.Fref, sizeof(double) * 3 * (size_t)na) != cudaSuccess ||
        cudaMalloc(&s.ref10, sizeof(double) * kNV) != cudaSuccess ||
        cudaMalloc(&s.cnt, sizeof(int) * (size_t)na) != cudaSuccess ||
        cudaMalloc(&s.list, sizeof(int) * (size_t)na * cap) != cudaSuccess) {
        snap_free(s);
        return ctx->fail(FMD_ERR_CUDA, "fmd_sg_data: snapshot allocation failed");
    }
    if (!d->part && cudaMalloc(&d->part, sizeof(double) * kForceBlocks * kNV) != cudaSuccess) {
        snap_free(s);
        return ctx->fail(FMD_ERR_CUDA, "fmd_sg_data: allocation failed");
    }
    cudaMemcpyAsync(s.pos, pos, sizeof(double) * 3 * (size_t)na, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(s.hh, hh, sizeof(double) * 18, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(s.cnt, cnt, sizeof(int) * (size_t)na, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(s.list, list, sizeof(int) * (size_t)na * cap, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(s.Fref, 0, sizeof(double) * 3 * (size_t)na, st);
    rebo_launch(s.pos, s.hh, s.cnt, s.list, cap, na, s.Fref, d->part, st);
    reduce_partials(d->part, kForceBlocks, kNV, s.ref10, st);
    const int rc = ctx->sync_check("fmd_sg_data_add");
    if (rc) {
        snap_free(s);
        return rc;
    }
    d->snaps.push_back(s);
    return FMD_OK;
}

extern "C" int fmd_sg_data_create(fmd_ctx* ctx, fmd_sg_data** out) {
    if (!ctx || !out) return FMD_ERR_ARG;
    *out = new fmd_sg_data();
    (*out)->ctx = ctx;
    return FMD_OK;
}

extern "C" int fmd_sg_data_destroy(fmd_sg_data* d) {
    if (!d) return FMD_ERR_ARG;
    cudaDeviceSynchronize();
    for (auto& s : d->snaps) snap_free(s);
    cudaFree(d->part);
    delete d;
    return FMD_OK;
}

extern "C" int fmd_sg_data_count(const fmd_sg_data* d) { return d ? (int)d->snaps.size() : -1; }

extern "C" int fmd_sg_data_add(fmd_sg_data* d, const double* pos, const double* h, const double* hi, const int* nlc,
                               const int* nll, int max_neigh, int na) {
    if (!d || !pos || !h || !hi || !nlc || !nll || na <= 0 || max_neigh <= 0) return FMD_ERR_ARG;
    fmd_ctx* ctx = d->ctx;
    for (int i = 0; i < na; i++) {
        if (nlc[i] < 0 || nlc[i] > max_neigh) return ctx->fail(FMD_ERR_ARG, "fmd_sg_data_add: bad list count");
        for (int k = 0; k < nlc[i]; k++) {
            const int j = nll[(size_t)i * max_neigh + k];
            if (j < 0 || j >= na) return ctx->fail(FMD_ERR_ARG, "fmd_sg_data_add: list entry out of range");
        }
    }
    double *dp = nullptr, *dh = nullptr;
    int *dc = nullptr, *dl = nullptr;
    if (cudaMalloc(&dp, sizeof(double) * 3 * (size_t)na) != cudaSuccess || cudaMalloc(&dh, sizeof(double) * 18) != cudaSuccess ||
        cudaMalloc(&dc, sizeof(int) * (size_t)na) != cudaSuccess ||
        cudaMalloc(&dl, sizeof(int) * (size_t)na * max_neigh) != cudaSuccess) {
        cudaFree(dp); cudaFree(dh); cudaFree(dc); cudaFree(dl);
        return ctx->fail(FMD_ERR_CUDA, "fmd_sg_data_add: allocation failed");
    }
    double hh[18];
    std::memcpy(hh, h, 72);
    std::memcpy(hh + 9, hi, 72);
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(dp, pos, sizeof(double) * 3 * (size_t)na, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dh, hh, sizeof(hh), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dc, nlc, sizeof(int) * (size_t)na, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dl, nll, sizeof(int) * (size_t)na * max_neigh, cudaMemcpyHostToDevice, st);
    const int rc = fmd::sg_data_add_device(d, dp, dh, dc, dl, max_neigh, na, st);
    cudaFree(dp); cudaFree(dh); cudaFree(dc); cudaFree(dl);
    return rc;
}

// Reference E, W9 and F of snapshot k (host copies), for tests.
extern "C" int fmd_sg_data_get(fmd_sg_data* d, int k, int* na, double* E, double* W9, double* F) {
    if (!d || k < 0 || k >= (int)d->snaps.size() || !na) return FMD_ERR_ARG;
    const Snap& s = d->snaps[k];
    *na = s.na;
    double r[kNV];
    cudaStream_t st = d->ctx->stream;
    cudaMemcpyAsync(r, s.ref10, sizeof(r), cudaMemcpyDeviceToHost, st);
    if (F) cudaMemcpyAsync(F, s.Fref, sizeof(double) * 3 * (size_t)s.na, cudaMemcpyDeviceToHost, st);
    const int rc = d->ctx->sync_check("fmd_sg_data_get");
    if (rc) return rc;
    if (E) *E = r[0];
    if (W9) std::memcpy(W9, r + 1, 72);
    return FMD_OK;
}

namespace {

int prepare(fmd_sg* s, Trainer& tr, int na, int cap) {
    fmd_ctx* ctx = s->ctx;
    FMD_CUDA_TRY(ctx, fmd::sg::work_alloc(s->work, std::max(na, s->work.na_cap), cap));
    FMD_CUDA_TRY(ctx, fmd::sg::train_alloc(tr.tw, s->work));
    if (!tr.grad) {
        FMD_CUDA_TRY(ctx, cudaMalloc(&tr.grad, sizeof(float) * fmd::sg::GRAD_N));
        FMD_CUDA_TRY(ctx, cudaMalloc(&tr.m, sizeof(double) * fmd::sg::NPARAM));
        FMD_CUDA_TRY(ctx, cudaMalloc(&tr.v, sizeof(double) * fmd::sg::NPARAM));
        FMD_CUDA_TRY(ctx, cudaMemset(tr.m, 0, sizeof(double) * fmd::sg::NPARAM));
        FMD_CUDA_TRY(ctx, cudaMemset(tr.v, 0, sizeof(double) * fmd::sg::NPARAM));
    }
    if (na > tr.F_na) {
        cudaFree(tr.F);
        tr.F = nullptr;
        FMD_CUDA_TRY(ctx, cudaMalloc(&tr.F, sizeof(double) * 3 * (size_t)na));
        tr.F_na = na;
    }
    return FMD_OK;
}

int check_errs(fmd_sg* s, const char* what) {
    int err[4];
    fmd_ctx* ctx = s->ctx;
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(err, s->work.err, sizeof(err), cudaMemcpyDeviceToHost, ctx->stream));
    const int rc = ctx->sync_check(what);
    if (rc) return rc;
    if (err[0]) return ctx->fail(FMD_ERR_ARG, std::string(what) + ": REBO list is not symmetric");
    if (err[1] || err[2] || err[3]) return ctx->fail(FMD_ERR_CUDA, std::string(what) + ": tensor-core wait timed out");
    return FMD_OK;
}

}  // namespace

// Loss and its gradient (master-parameter layout, zeros for m, s, b0, bs) on
// one snapshot given by host arrays and reference values.
extern "C" int fmd_sg_loss_grad(fmd_sg* s, const double* pos, const double* h, const double* hi, const int* nlc,
                                const int* nll, int max_neigh, int na, const double* F_ref, double E_ref,
                                const double* W_ref, double wE, double wF, double wW, double* loss, double* grad) {
    if (!s || !pos || !h || !hi || !nlc || !nll || !F_ref || !W_ref || !loss || !grad || na <= 0) return FMD_ERR_ARG;
    fmd_ctx* ctx = s->ctx;
    Trainer& tr = s->tr;
    int rc = stage(s, na, max_neigh);
    if (!rc) rc = prepare(s, tr, na, max_neigh);
    if (rc) return rc;
    for (int i = 0; i < na; i++)
        for (int k = 0; k < nlc[i]; k++) {
            const int j = nll[(size_t)i * max_neigh + k];
            if (nlc[i] > max_neigh || j < 0 || j >= na) return ctx->fail(FMD_ERR_ARG, "fmd_sg_loss_grad: bad list");
        }
    cudaStream_t st = ctx->stream;
    double hh[18], ref10[kNV];
    std::memcpy(hh, h, 72);
    std::memcpy(hh + 9, hi, 72);
    ref10[0] = E_ref;
    std::memcpy(ref10 + 1, W_ref, 72);
    double *dref = nullptr, *dFref = nullptr, *dloss = nullptr, *dgrad = nullptr;
    FMD_CUDA_TRY(ctx, cudaMalloc(&dref, sizeof(ref10)));
    FMD_CUDA_TRY(ctx, cudaMalloc(&dFref, sizeof(double) * 3 * (size_t)na));
    FMD_CUDA_TRY(ctx, cudaMalloc(&dloss, sizeof(double) * 2));
    FMD_CUDA_TRY(ctx, cudaMalloc(&dgrad, sizeof(double) * fmd::sg::NPARAM));
    cudaMemcpyAsync(s->hh, hh, sizeof(hh), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->pos, pos, sizeof(double) * 3 * (size_t)na, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->cnt, nlc, sizeof(int) * (size_t)na, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->list, nll, sizeof(int) * (size_t)na * max_neigh, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dref, ref10, sizeof(ref10), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dFref, F_ref, sizeof(double) * 3 * (size_t)na, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(dloss, 0, sizeof(double) * 2, st);
    cudaMemsetAsync(tr.grad, 0, sizeof(float) * fmd::sg::GRAD_N, st);
    cudaMemsetAsync(s->work.err, 0, sizeof(int) * 4, st);
    cudaError_t e = fmd::sg::accumulate_grad(s->work, tr.tw, s->img, s->vec, s->pos, s->hh, s->cnt, s->list, max_neigh,
                                             na, dFref, dref, wE, wF, wW, tr.F, dloss, tr.grad, st);
    if (e == cudaSuccess) e = fmd::sg::grad_to_params(tr.grad, 1.0, dgrad, st);
    double lh[2];
    if (e == cudaSuccess) e = cudaMemcpyAsync(lh, dloss, sizeof(lh), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad, dgrad, sizeof(double) * fmd::sg::NPARAM, cudaMemcpyDeviceToHost, st);
    rc = e == cudaSuccess ? check_errs(s, "fmd_sg_loss_grad") : ctx->fail(FMD_ERR_CUDA, cudaGetErrorString(e));
    cudaFree(dref); cudaFree(dFref); cudaFree(dloss); cudaFree(dgrad);
    if (rc) return rc;
    *loss = lh[0];
    s->last_na = na;
    return FMD_OK;
}

extern "C" int fmd_sg_train(fmd_sg* s, fmd_sg_data* d, const fmd_sg_train_args* a, double* history) {
    if (!s || !d || !a || a->steps <= 0 || a->batch <= 0 || d->snaps.empty()) return FMD_ERR_ARG;
    fmd_ctx* ctx = s->ctx;
    Trainer& tr = s->tr;
    int namax = 0, cap = d->snaps[0].cap;
    for (auto& sn : d->snaps) {
        namax = std::max(namax, sn.na);
        if (sn.cap != cap) return ctx->fail(FMD_ERR_ARG, "fmd_sg_train: snapshots with different list widths");
    }
    const int n_use = a->n_train > 0 ? std::min(a->n_train, (int)d->snaps.size()) : (int)d->snaps.size();
    int rc = prepare(s, tr, namax, cap);
    if (rc) return rc;
    if (a->steps > tr.hist_n) {
        cudaFree(tr.hist);
        tr.hist = nullptr;
        FMD_CUDA_TRY(ctx, cudaMalloc(&tr.hist, sizeof(double) * 2 * a->steps));
        tr.hist_n = a->steps;
    }
    cudaStream_t st = ctx->stream;
    FMD_CUDA_TRY(ctx, cudaMemsetAsync(tr.hist, 0, sizeof(double) * 2 * a->steps, st));
    FMD_CUDA_TRY(ctx, cudaMemsetAsync(s->work.err, 0, sizeof(int) * 4, st));
    std::mt19937_64 rng((uint64_t)a->seed);
    const double b1 = 0.9, b2 = 0.999;
    for (int step = 0; step < a->steps; step++) {
        FMD_CUDA_TRY(ctx, cudaMemsetAsync(tr.grad, 0, sizeof(float) * fmd::sg::GRAD_N, st));
        for (int b = 0; b < a->batch; b++) {
            const Snap& sn = d->snaps[rng() % (uint64_t)n_use];
            FMD_CUDA_TRY(ctx, fmd::sg::accumulate_grad(s->work, tr.tw, s->img, s->vec, sn.pos, sn.hh, sn.cnt, sn.list,
                                                       sn.cap, sn.na, sn.Fref, sn.ref10, a->wE, a->wF, a->wW, tr.F,
                                                       tr.hist + 2 * step, tr.grad, st));
        }
        tr.t++;
        const double frac = a->steps > 1 ? (double)step / (a->steps - 1) : 1.0;
        fmd::sg::AdamArgs aa;
        aa.lr = a->lr_final + 0.5 * (a->lr - a->lr_final) * (1.0 + std::cos(3.14159265358979323846 * frac));
        aa.b1 = b1; aa.b2 = b2; aa.eps = 1e-12;
        aa.bc1 = 1.0 - std::pow(b1, (double)tr.t);
        aa.bc2 = 1.0 - std::pow(b2, (double)tr.t);
        aa.scale = 1.0 / a->batch;
        aa.clip = a->clip;
        FMD_CUDA_TRY(ctx, fmd::sg::adam_step(s->P, tr.m, tr.v, tr.grad, aa, s->img, s->vec, st));
        if ((step + 1) % 200 == 0 || step + 1 == a->steps) {
            rc = check_errs(s, "fmd_sg_train");
            if (rc) return rc;
        }
    }
    if (history) {
        FMD_CUDA_TRY(ctx, cudaMemcpyAsync(history, tr.hist, sizeof(double) * 2 * a->steps, cudaMemcpyDeviceToHost, st));
    }
    rc = check_errs(s, "fmd_sg_train");
    if (rc) return rc;
    if (history)
        for (int k = 0; k < a->steps; k++) {
            history[2 * k] /= a->batch;
            history[2 * k + 1] = std::sqrt(history[2 * k + 1] / a->batch);
        }
    return FMD_OK;
}

// Force RMSE of the model against the reference REBO forces of snapshots
// [first, first + n): rmse[k] per snapshot (n values).
extern "C" int fmd_sg_eval(fmd_sg* s, fmd_sg_data* d, int first, int n, double* rmse) {
    if (!s || !d || !rmse || first < 0 || n <= 0 || first + n > (int)d->snaps.size()) return FMD_ERR_ARG;
    fmd_ctx* ctx = s->ctx;
    Trainer& tr = s->tr;
    int namax = 0;
    for (int k = first; k < first + n; k++) namax = std::max(namax, d->snaps[k].na);
    int rc = prepare(s, tr, namax, d->snaps[first].cap);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    double* dl = nullptr;
    FMD_CUDA_TRY(ctx, cudaMalloc(&dl, sizeof(double) * 2 * n));
    FMD_CUDA_TRY(ctx, cudaMemsetAsync(dl, 0, sizeof(double) * 2 * n, st));
    FMD_CUDA_TRY(ctx, cudaMemsetAsync(s->work.err, 0, sizeof(int) * 4, st));
    for (int k = 0; k < n; k++) {
        const Snap& sn = d->snaps[first + k];
        if (sn.cap != s->work.cap) {
            cudaFree(dl);
            return ctx->fail(FMD_ERR_ARG, "fmd_sg_eval: snapshots with different list widths");
        }
        FMD_CUDA_TRY(ctx, cudaMemsetAsync(tr.F, 0, sizeof(double) * 3 * (size_t)sn.na, st));
        FMD_CUDA_TRY(ctx, fmd::sg::rebo_forces(s->work, s->img, s->vec, sn.pos, sn.hh, sn.cnt, sn.list, sn.cap, sn.na,
                                               tr.F, s->work.part, st));
        FMD_CUDA_TRY(ctx, fmd::sg::force_mse(tr.F, sn.Fref, sn.na, tr.tw.part, dl + 2 * k, st));
    }
    std::vector<double> h(2 * n);
    FMD_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), dl, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, st));
    rc = check_errs(s, "fmd_sg_eval");
    cudaFree(dl);
    if (rc) return rc;
    for (int k = 0; k < n; k++) rmse[k] = std::sqrt(h[2 * k]);
    return FMD_OK;
}

// Mean and standard deviation of the raw descriptors over the rows of
// snapshots [first, first+n) (for the normalisation m, s of a new model).
extern "C" int fmd_sg_feature_stats(fmd_sg* s, fmd_sg_data* d, int first, int n, double* mean, double* stdev) {
    if (!s || !d || !mean || !stdev || first < 0 || n <= 0 || first + n > (int)d->snaps.size()) return FMD_ERR_ARG;
    fmd_ctx* ctx = s->ctx;
    Trainer& tr = s->tr;
    int namax = 0;
    for (int k = first; k < first + n; k++) namax = std::max(namax, d->snaps[k].na);
    int rc = prepare(s, tr, namax, d->snaps[first].cap);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    float raw[sg::V_N];
    for (int e = 0; e < sg::V_N; e++) raw[e] = 0.f;
    for (int f = 0; f < sg::D; f++) raw[sg::V_SINV + f] = 1.f;
    float* dvec = nullptr;
    double* acc = nullptr;
    int* rows = nullptr;
    FMD_CUDA_TRY(ctx, cudaMalloc(&dvec, sizeof(raw)));
    FMD_CUDA_TRY(ctx, cudaMalloc(&acc, sizeof(double) * 2 * sg::D));
    FMD_CUDA_TRY(ctx, cudaMalloc(&rows, sizeof(int) * n));
    cudaMemcpyAsync(dvec, raw, sizeof(raw), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(acc, 0, sizeof(double) * 2 * sg::D, st);
    for (int k = 0; k < n; k++) {
        const Snap& sn = d->snaps[first + k];
        FMD_CUDA_TRY(ctx, sg::build_rows(s->work, dvec, sn.pos, sn.hh, sn.cnt, sn.list, sn.cap, sn.na, st));
        FMD_CUDA_TRY(ctx, sg::feature_sums(s->work, acc, st));
        cudaMemcpyAsync(rows + k, s->work.aoff + sn.na, sizeof(int), cudaMemcpyDeviceToDevice, st);
    }
    double h[2 * sg::D];
    std::vector<int> hr(n);
    cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hr.data(), rows, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    rc = ctx->sync_check("fmd_sg_feature_stats");
    cudaFree(dvec); cudaFree(acc); cudaFree(rows);
    if (rc) return rc;
    double R = 0;
    for (int k = 0; k < n; k++) R += hr[k];
    if (R <= 0) return ctx->fail(FMD_ERR_ARG, "fmd_sg_feature_stats: no rows");
    for (int f = 0; f < sg::D; f++) {
        mean[f] = h[2 * f] / R;
        stdev[f] = std::sqrt(std::max(h[2 * f + 1] / R - mean[f] * mean[f], 0.0));
    }
    return FMD_OK;
}
