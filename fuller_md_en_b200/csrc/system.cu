// system.cu -- device-resident systems: state in HBM for the whole run, list
// rebuilds on the device every nlup steps, each step replayed as a CUDA graph
// (one graph per {rebuild, cold/warm} variant, captured on first use).
// The host only sees observables at the steps it asks for.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <tuple>
#include "step.h"
#include "system.h"
#include "sg_host.h"

using namespace fmd;

namespace fmd {

namespace {
template <class T>
size_t dbytes(size_t count) {
    return sizeof(T) * (count > 0 ? count : 1);
}

// Runs the rebuild's cell-grid fallback (a conditional graph node) only when
// the molecule path was rejected for this rebuild (flag[0] == 0).
__global__ void k_fallback_cond(const int* __restrict__ flag, cudaGraphConditionalHandle cond) {
    if (threadIdx.x == 0) cudaGraphSetConditional(cond, flag[0] == 0 ? 1u : 0u);
}
}  // namespace

void System::drop_graphs() {
    for (auto& a : graphs)
        for (auto& b : a)
            for (auto& g : b)
                if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

void System::release() {
    drop_graphs();
    for (auto& ev : obs_ev)
        if (ev) { cudaEventDestroy(ev); ev = nullptr; }
    if (side) {
        cudaStreamDestroy(side);
        side = nullptr;
    }
    if (sg) sg::work_free(sg->work);
    sg.reset();
    arr.sg = nullptr;
    if (ctx) {
        // every stream that used these blocks has finished with them
        cudaStreamSynchronize(ctx->stream);
        for (auto& b : owned) ctx->dev_release(b.first, b.second);
    } else {
        for (auto& b : owned) cudaFree(b.first);
    }
    owned.clear();
    cells_free(cells_a);
    cells_free(cells_b);
    prune = LJPrune();                  // its arrays are among the owned blocks
    arr.prune = nullptr; arr.prune_sb = nullptr; arr.prune_umax = nullptr; arr.prune_hb = nullptr;
    arr.prune_stats = nullptr; arr.prune_delta = 0.0;
    mol_lists_free(mol);
}

template <class T>
cudaError_t System::alloc(T** p, size_t count, const T* src) {
    const size_t bytes = dbytes<T>(count);
    cudaError_t e = ctx->dev_alloc((void**)p, bytes);
    if (e != cudaSuccess) return e;
    owned.emplace_back((void*)*p, bytes);
    if (src == nullptr || count == 0) return cudaSuccess;
    return cudaMemcpyAsync(*p, src, sizeof(T) * count, cudaMemcpyHostToDevice, ctx->stream);
}

cudaError_t System::alloc_raw(void* self, void** p, size_t bytes) {
    return static_cast<System*>(self)->alloc(reinterpret_cast<char**>(p), bytes, (const char*)nullptr);
}

int System::alloc_common(const double* pos_h, const double* vel_h, const double* h_h, const fmd_npt* npt_h) {
    cudaStream_t st = ctx->stream;
    const int n = arr.n;
    if (alloc(&arr.pos, 3 * (size_t)n, pos_h) || alloc(&arr.vel, 3 * (size_t)n, vel_h) ||
        alloc(&arr.F, 3 * (size_t)n, (const double*)nullptr) || alloc(&arr.Facc, 3 * (size_t)n, (const double*)nullptr) ||
        alloc(&arr.part_f1, (size_t)std::max(kForceBlocks, n) * kNV, (const double*)nullptr) ||
        alloc(&arr.part_f2, (size_t)kLJMaxBlocks * kNV, (const double*)nullptr) ||
        alloc(&arr.part_f3, (size_t)kForceBlocks, (const double*)nullptr) ||
        alloc(&arr.part_ke, (size_t)kForceBlocks * 2, (const double*)nullptr) ||
        alloc(&dropped, 2, (const int*)nullptr) || alloc(&arr.S, 1, (const SysScal*)nullptr))
        return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
    arr.err = ctx->d_err;
    cudaMemsetAsync(arr.F, 0, sizeof(double) * 3 * n, st);
    cudaMemsetAsync(arr.Facc, 0, sizeof(double) * 3 * n, st);
    cudaMemsetAsync(dropped, 0, sizeof(int) * 2, st);
    SysScal s;
    std::memset(&s, 0, sizeof(s));
    for (int k = 0; k < 9; k++) s.h[k] = h_h[k];
    s.npt = *npt_h;
    s.gstep = 0;
    cudaMemcpyAsync(arr.S, &s, sizeof(s), cudaMemcpyHostToDevice, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, cudaGetErrorString(e));
    std::memcpy(h0, h_h, sizeof(h0));
    return FMD_OK;
}

int System::alloc_lists(double rc_list_a, int cap_a_, double rc_list_b, int cap_b_, bool transpose) {
    const int n = arr.n;
    rc_a = rc_list_a; rc2_a = rc_a * rc_a; arr.cap_a = cap_a_;
    int* cnt; int* lst;
    if (alloc(&cnt, n, (const int*)nullptr) || alloc(&lst, (size_t)n * cap_a_, (const int*)nullptr))
        return ctx->fail(FMD_ERR_CUDA, "list allocation failed");
    cudaMemsetAsync(lst, 0, sizeof(int) * (size_t)n * cap_a_, ctx->stream);
    arr.cnt_a = cnt; arr.list_a = lst;
    if (cells_alloc(cells_a, n, h0, rc_a, 2, owned_alloc()) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "cell allocation failed");
    if (cap_b_ > 0) {
        rc_b = rc_list_b; rc2_b = rc_b * rc_b; arr.cap_b = cap_b_;
        if (alloc(&cnt, n, (const int*)nullptr) || alloc(&lst, (size_t)n * cap_b_, (const int*)nullptr))
            return ctx->fail(FMD_ERR_CUDA, "list allocation failed");
        cudaMemsetAsync(lst, 0, sizeof(int) * (size_t)n * cap_b_, ctx->stream);
        arr.cnt_b = cnt; arr.list_b = lst;
        if (cells_alloc(cells_b, n, h0, rc_b, 1, owned_alloc()) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "cell allocation failed");
        if (alloc(&arr.rebo_slots, (size_t)n * cap_b_ * kReboSlotDoubles, (const double*)nullptr))
            return ctx->fail(FMD_ERR_CUDA, "list allocation failed");
        int* ids;
        if (alloc(&ids, 1 + (size_t)kIdsLanes * n + (size_t)n * cap_b_, (const int*)nullptr) ||
            alloc(&rebo_bsum, (size_t)rebo_ids_scratch(n), (const int*)nullptr))
            return ctx->fail(FMD_ERR_CUDA, "list allocation failed");
        cudaMemsetAsync(ids, 0, sizeof(int), ctx->stream);
        arr.rebo_ids = ids;
    }
    if (transpose) {
        arr.in_cap = kInCap + cap_a_;   // full rows: incoming entries then the row itself
        if (alloc(&cnt, n, (const int*)nullptr) || alloc(&lst, (size_t)n * arr.in_cap, (const int*)nullptr))
            return ctx->fail(FMD_ERR_CUDA, "list allocation failed");
        arr.in_cnt = cnt; arr.in_list = lst;
    }
    return FMD_OK;
}

// Rebuild of every list this kind uses, as the driver does at gstep % nlup == 0.
int System::alloc_prune(double rc_lj) {
    if (!arr.in_list) return FMD_OK;
    const int n = arr.n;
    LJPrune q;
    if (alloc(&q.cnt, n, (const int*)nullptr) || alloc(&q.list, (size_t)n * arr.in_cap, (const int*)nullptr) ||
        alloc(&q.sb, 3 * (size_t)n, (const double*)nullptr) || alloc(&q.hb, 9, (const double*)nullptr) ||
        alloc(&q.words, 1, (const unsigned long long*)nullptr) ||
        alloc(&q.stats, 2, (const unsigned long long*)nullptr))
        return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
    q.n = n;
    q.stride = arr.in_cap;
    q.rc = rc_lj;
    q.delta = kPruneDelta;
    q.ok = true;
    if (lj_prune_clear(q, ctx->stream) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
    prune = q;
    arr.prune = &prune;
    arr.prune_sb = prune.sb;
    arr.prune_umax = prune.words;
    arr.prune_hb = prune.hb;
    arr.prune_stats = prune.stats;
    arr.prune_delta = prune.delta;
    arr.prune_rc = prune.rc;
    return FMD_OK;
}

cudaError_t System::enqueue_rebuild(cudaStream_t st) {
    cudaError_t e;
    double* hh = arr.S->h;
    if ((e = inv9_launch(hh, st)) != cudaSuccess) return e;
    int* cnt_a = const_cast<int*>(arr.cnt_a);
    int* list_a = const_cast<int*>(arr.list_a);
    if (arr.kind == FMD_SYS_RIGID) {
        if ((e = cells_build(cells_a, arr.pos, arr.n, hh, rc_a, ctx->d_err, st)) != cudaSuccess) return e;
        return nlist_build(cells_a, LIST_SYM, arr.pos, nullptr, arr.n, hh, rc2_a, arr.cap_a, cnt_a, list_a,
                           dropped, ctx->d_err, st);
    }
    if (arr.kind == FMD_SYS_AIREBO) {
        if (mol.ok) {
            if ((e = mol_rows_intra(mol, arr.pos, hh, rc2_b, arr.cap_b, const_cast<int*>(arr.cnt_b),
                                    const_cast<int*>(arr.list_b), dropped + 1, st)) != cudaSuccess)
                return e;
        } else {
            if ((e = cells_build(cells_b, arr.pos, arr.n, hh, rc_b, ctx->d_err, st, arr.mol_id)) != cudaSuccess) return e;
            if ((e = nlist_build(cells_b, LIST_INTRA, arr.pos, arr.mol_id, arr.n, hh, rc2_b, arr.cap_b,
                                 const_cast<int*>(arr.cnt_b), const_cast<int*>(arr.list_b), dropped + 1,
                                 ctx->d_err, st)) != cudaSuccess)
                return e;
        }
        if (arr.rebo_ids &&
            (e = rebo_ids_build(arr.cnt_b, arr.list_b, arr.cap_b, arr.n, const_cast<int*>(arr.rebo_ids), rebo_bsum,
                                st)) !=
                cudaSuccess)
            return e;
    }
    // Half list: the molecule path when valid for this rebuild (decided on
    // the device), else the cell-grid path; both are in the graph, gated.
    // In a captured graph the cell-grid path sits in a conditional node that
    // the decision switches on, so a rebuild by the molecule path launches
    // none of its kernels.
    const int* gate = nullptr;
    if (mol.ok) {
        if ((e = mol_partners(mol, arr.pos, hh, rc_a, st)) != cudaSuccess) return e;
        gate = mol.flag;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (mol.ok && mol.masks && (e = cudaStreamIsCapturing(st, &cs)) != cudaSuccess) return e;
    if (cs == cudaStreamCaptureStatusActive) {
        if ((e = enqueue_fallback_conditional(st)) != cudaSuccess) return e;
        if ((e = mol_rows_half(mol, arr.pos, hh, rc2_a, arr.cap_a, cnt_a, list_a, dropped, st)) != cudaSuccess)
            return e;
        if ((e = mol_rows_incoming(mol, arr.cap_a, arr.cnt_a, arr.list_a, const_cast<int*>(arr.in_cnt),
                                   const_cast<int*>(arr.in_list), arr.in_cap, ctx->d_err, st)) != cudaSuccess)
            return e;
        if (prune.ok) return lj_prune_mark(prune, st);
        return cudaSuccess;
    }
    if ((e = cells_build(cells_a, arr.pos, arr.n, hh, rc_a, ctx->d_err, st, arr.mol_id, gate)) != cudaSuccess) return e;
    if ((e = nlist_build(cells_a, LIST_HALF, arr.pos, arr.mol_id, arr.n, hh, rc2_a, arr.cap_a, cnt_a, list_a,
                         dropped, ctx->d_err, st, gate)) != cudaSuccess)
        return e;
    if (mol.ok && (e = mol_rows_half(mol, arr.pos, hh, rc2_a, arr.cap_a, cnt_a, list_a, dropped, st)) != cudaSuccess)
        return e;
    // the gather's full rows: from the molecule builder's candidate bitmaps
    // when it ran (equal molecules of 32-64 atoms), else the transpose of
    // whichever half list was built (gated the other way; its clear of the
    // row counts is not gated, so it goes first)
    if (mol.ok && mol.masks) {
        if ((e = nlist_transpose(arr.cnt_a, arr.list_a, arr.cap_a, arr.n, const_cast<int*>(arr.in_cnt),
                                 const_cast<int*>(arr.in_list), arr.in_cap, ctx->d_err, st, gate)) != cudaSuccess)
            return e;
        if ((e = mol_rows_incoming(mol, arr.cap_a, arr.cnt_a, arr.list_a, const_cast<int*>(arr.in_cnt),
                                   const_cast<int*>(arr.in_list), arr.in_cap, ctx->d_err, st)) != cudaSuccess)
            return e;
    } else if ((e = nlist_transpose(arr.cnt_a, arr.list_a, arr.cap_a, arr.n, const_cast<int*>(arr.in_cnt),
                                    const_cast<int*>(arr.in_list), arr.in_cap, ctx->d_err, st)) != cudaSuccess) {
        return e;
    }
    if (prune.ok) return lj_prune_mark(prune, st);     // new rows: the next evaluation prunes them
    return cudaSuccess;
}

cudaError_t System::enqueue_fallback_conditional(cudaStream_t st) {
    cudaError_t e;
    if (!side && (e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking)) != cudaSuccess) return e;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd)) != cudaSuccess) return e;
    if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureUnsupported;
    cudaGraphConditionalHandle cond;
    if ((e = cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
    k_fallback_cond<<<1, 32, 0, st>>>(mol.flag, cond);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd)) != cudaSuccess) return e;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if ((e = cudaGraphAddNode(&node, g, deps, nd, &cp)) != cudaSuccess) return e;
    if ((e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
        return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
        cudaSuccess)
        return e;
    const cudaError_t ef = enqueue_rebuild_fallback(side);
    cudaGraph_t got = nullptr;
    if ((e = cudaStreamEndCapture(side, &got)) != cudaSuccess) return e;
    return ef;
}

cudaError_t System::enqueue_rebuild_fallback(cudaStream_t st) {
    if (!(mol.ok && mol.masks) || arr.kind == FMD_SYS_RIGID) return cudaErrorInvalidValue;
    double* hh = arr.S->h;
    int* cnt_a = const_cast<int*>(arr.cnt_a);
    int* list_a = const_cast<int*>(arr.list_a);
    const int* gate = mol.flag;
    cudaError_t e;
    if ((e = cells_build(cells_a, arr.pos, arr.n, hh, rc_a, ctx->d_err, st, arr.mol_id, gate)) != cudaSuccess) return e;
    if ((e = nlist_build(cells_a, LIST_HALF, arr.pos, arr.mol_id, arr.n, hh, rc2_a, arr.cap_a, cnt_a, list_a,
                         dropped, ctx->d_err, st, gate)) != cudaSuccess)
        return e;
    return nlist_transpose(arr.cnt_a, arr.list_a, arr.cap_a, arr.n, const_cast<int*>(arr.in_cnt),
                           const_cast<int*>(arr.in_list), arr.in_cap, ctx->d_err, st, gate);
}

// Times every launch shape of the atomistic LJ gather and returns the
// fastest.  Each candidate is timed as the step runs it: right after a write
// larger than L2 (the step's other kernels have evicted the rows), behind the
// short-range term it follows (programmatic launch edge), writing F from the
// accumulator.  pruned: the gather of a system with pruned rows, which walks
// the pruned rows on most evaluations and the full rows (writing new pruned
// rows) on the rest; its cost is the walk plus one prune evaluation per
// kPruneEvery walks (the prune rate of the bench workload).  Otherwise the
// gather over the full rows alone.  The timed launches leave the accumulator
// zero and F holding the plain short-range term plus LJ (the caller
// recomputes F when it must hold the system's forces); a forced prune
// evaluation rewrites the pruned rows as they are (same positions).
LJShape System::pick_lj_shape(bool pruned, int& rc) {
    constexpr int kPruneEvery = 8;
    const int ff = arr.kind == FMD_SYS_AIREBO ? FMD_FF_AIREBO : FMD_FF_MM;
    cudaStream_t st = ctx->stream;
    void* flush = nullptr;
    const size_t flush_bytes = 160u << 20;
    if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
        cudaGetLastError();
        flush = nullptr;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto short_range = [&]() -> cudaError_t {
        const double* hh = arr.S->h;
        if (arr.kind == FMD_SYS_MM) return mm_bonded_launch(arr.topo, arr.pos, hh, arr.Facc, arr.part_f1, st);
        if (arr.rebo_slots)
            return rebo_slots_launch(arr.pos, hh, arr.cnt_b, arr.list_b, arr.cap_b, arr.n, arr.rebo_slots, arr.Facc,
                                     arr.part_f1, kForceBlocks, nullptr, 0, st, arr.rebo_ids, arr.rebo_phys != 0);
        return rebo_launch(arr.pos, hh, arr.cnt_b, arr.list_b, arr.cap_b, arr.n, arr.Facc, arr.part_f1, st);
    };
    const LJPruneOut walk = pruned ? lj_prune_out(prune) : LJPruneOut{};
    LJPruneOut full = walk;
    full.words = nullptr;                // no decision: the full rows, pruned rows written
    auto time_one = [&](const LJShape& sh, const LJPruneOut& po, int r) {
        if (flush) cudaMemsetAsync(flush, r, flush_bytes, st);
        cudaEventRecord(e0, st);
        short_range();
        lj_gather_launch(ff, arr.pos, arr.S->h, arr.cnt_a, arr.list_a, arr.cap_a, arr.in_cnt, arr.in_list, arr.in_cap,
                         arr.n, arr.F, arr.Facc, arr.part_f2, st, arr.precision, sh, ctx->d_err, po);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    float best = 1e30f;
    LJShape pick;
    for (int contig : {0, 1})
    for (int nt : {128, 256})
        for (int u : {2, 4})
            for (int pipe : {0, 1, 2}) {
                const LJShape sh{nt, u, pipe, contig};
                if (lj_gather_blocks(ff, arr.precision, sh, arr.in_cap) < 1) continue;
                time_one(sh, walk, 0);           // untimed: first launch of this shape
                float tot = 0.f;
                for (int r = 0; r < 3; r++) tot += time_one(sh, walk, r);
                if (pruned) {
                    float tp = 0.f;
                    for (int r = 0; r < 2; r++) tp += time_one(sh, full, r);
                    tot += 3.f * tp / (2.f * kPruneEvery);
                }
                if (tot < best) { best = tot; pick = sh; }
            }
    if (flush) cudaFree(flush);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemsetAsync(arr.Facc, 0, sizeof(double) * 3 * (size_t)arr.n, st);
    rc = ctx->sync_check("LJ launch-shape tuning");
    return pick;
}

// Partial records of the LJ term: the larger grid of the two gathers (the
// smaller one zero-fills the rest).
void System::set_lj_blocks() {
    const int ff = arr.kind == FMD_SYS_AIREBO ? FMD_FF_AIREBO : FMD_FF_MM;
    arr.lj_blocks = std::max(lj_gather_blocks(ff, arr.precision, arr.lj_shape, arr.in_cap),
                             lj_gather_blocks(ff, arr.precision, arr.lj_shape_p, arr.in_cap));
}

// Launch shape of the atomistic LJ gather over the full rows: every candidate
// (threads per block, list entries in flight per lane, row feed) is timed on
// this system's own rows at set-up and the fastest kept; the choice is cached
// per (device, kind, atoms, list width, precision) for the process.  The
// gather over the pruned rows is tuned the same way once those rows exist
// (tune_lj_pruned).
int System::tune_lj() {
    static std::map<std::tuple<int, int, int, int, int>, LJShape> cache;
    const int ff = arr.kind == FMD_SYS_AIREBO ? FMD_FF_AIREBO : FMD_FF_MM;
    // FMD_LJ_SHAPE="threads,unroll,feed" pins the shape of both gathers (no
    // trial launches), for reproducible runs and profiler captures; feed is
    // 0..2, plus 4 for contiguous atom runs per block.  A second triple after
    // ';' pins the gather over the pruned rows separately.
    if (const char* env = std::getenv("FMD_LJ_SHAPE")) {
        auto parse = [&](const char* t, LJShape& sh) {
            int feed = -1;
            if (std::sscanf(t, "%d,%d,%d", &sh.threads, &sh.unroll, &feed) != 3 ||
                !(sh.threads == 128 || sh.threads == 256) || !(sh.unroll == 2 || sh.unroll == 4) ||
                !lj_feed_valid(feed))
                return false;
            sh.pipe = feed & 3;
            sh.contig = feed >> 2;
            return lj_gather_blocks(ff, arr.precision, sh, arr.in_cap) > 0;
        };
        LJShape sh, shp;
        const char* second = std::strchr(env, ';');
        if (parse(env, sh) && (second ? parse(second + 1, shp) : (shp = sh, true))) {
            arr.lj_shape = sh;
            arr.lj_shape_p = shp;
            set_lj_blocks();
            return FMD_OK;
        }
        return ctx->fail(FMD_ERR_ARG, "FMD_LJ_SHAPE: expected threads,unroll,feed[;threads,unroll,feed] with "
                                      "threads 128|256, unroll 2|4, feed 0..2 or 4..6");
    }
    const auto key = std::make_tuple(ctx->device, arr.kind, arr.n, arr.cap_a, arr.precision);
    auto it = cache.find(key);
    if (it != cache.end()) {
        arr.lj_shape = it->second;
    } else {
        int rc = FMD_OK;
        const LJShape pick = pick_lj_shape(false, rc);
        if (rc != FMD_OK) return rc;
        cache[key] = pick;
        arr.lj_shape = pick;
    }
    arr.lj_shape_p = arr.lj_shape;
    set_lj_blocks();
    return FMD_OK;
}

// run_tuner false: only a shape cached by an earlier system of the same size
// is applied, and *pending tells whether the tuner still has to run (after
// the first evaluation has written the pruned rows).
int System::tune_lj_pruned(bool run_tuner, bool* pending) {
    static std::map<std::tuple<int, int, int, int, int>, LJShape> cache;
    if (pending) *pending = false;
    if (!prune.ok || prune.delta <= 0.0 || std::getenv("FMD_LJ_SHAPE")) return FMD_OK;
    const auto key = std::make_tuple(ctx->device, arr.kind, arr.n, arr.cap_a, arr.precision);
    auto it = cache.find(key);
    if (it != cache.end()) {
        arr.lj_shape_p = it->second;
    } else if (!run_tuner) {
        if (pending) *pending = true;
        return FMD_OK;
    } else {
        int rc = FMD_OK;
        const LJShape pick = pick_lj_shape(true, rc);
        if (rc != FMD_OK) return rc;
        cache[key] = pick;
        arr.lj_shape_p = pick;
        // the trials timed the plain short-range term: F again from the
        // system's own terms (REBO-II, the learned term, the LJ switch)
        if (enqueue_forces(arr, ctx->stream) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "force launch failed");
        if ((rc = ctx->sync_check("LJ launch-shape tuning")) != FMD_OK) return rc;
    }
    set_lj_blocks();
    return FMD_OK;
}

// Launch shape of the rigid pair kernel, timed on this system's own list at
// set-up (the pair kernel writes F, T and partials only, which the first
// force evaluation below recomputes); cached per (device, molecules, sites,
// precision).
int System::tune_rigid() {
    static std::map<std::tuple<int, int, int, int>, int> cache;
    const auto key = std::make_tuple(ctx->device, arr.n, arr.natom, arr.precision);
    auto it = cache.find(key);
    if (it != cache.end()) {
        arr.rigid_shape = it->second;
        return FMD_OK;
    }
    cudaStream_t st = ctx->stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int pick = 0;
    for (int shape : {0, 1, 2}) {
        auto go = [&]() {
            return rigid_launch(arr.precision, arr.pos, arr.qv, arr.body, arr.S->h, arr.cnt_a, arr.list_a, arr.cap_a,
                                arr.n, arr.natom, arr.rmcut2, arr.F, arr.T, arr.part_f1, st, arr.rigid_lab, shape);
        };
        go();
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3; r++) go();
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; pick = shape; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int rc = ctx->sync_check("rigid launch-shape tuning");
    if (rc != FMD_OK) return rc;
    cache[key] = pick;
    arr.rigid_shape = pick;
    return FMD_OK;
}

int System::init() {
    cudaStream_t st = ctx->stream;
    // Pre-loop order of the reference: lists from the unwrapped positions,
    // then apply_pbc, then the first forces (LJ:813-828, AI:830-853).
    if (enqueue_rebuild(st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "list build launch failed");
    if (apply_pbc_launch(arr.pos, arr.n, arr.S->h, st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "apply_pbc failed");
    if (arr.kind != FMD_SYS_RIGID) {
        const int rc = tune_lj();
        if (rc != FMD_OK) return rc;
    } else {
        const int rc = tune_rigid();
        if (rc != FMD_OK) return rc;
    }
    if (enqueue_forces(arr, st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "force launch failed");
    if (enqueue_force_reduce(arr, st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "reduce launch failed");
    if (enqueue_ke(arr, st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "kinetic launch failed");
    // The gather shape over the pruned rows, when an earlier system of this
    // size has tuned it; else the tuner runs once the first evaluation has
    // pruned the rows.
    int rc = FMD_OK;
    bool pending = false;
    if (arr.kind != FMD_SYS_RIGID && (rc = tune_lj_pruned(false, &pending)) != FMD_OK) return rc;
    // Capture the step variants the schedule can reach (the cold/warm phase
    // ones only with coldstart + warmup > 0) now, so no host-side capture
    // ever sits between two steps of a run; the host captures while the
    // device runs the set-up work enqueued above.
    auto capture_all = [&]() -> int {
        if (p.use_graphs)
            for (int r = 0; r < 2; r++)
                for (int ph = 0; ph < 2; ph++)
                    if ((ph == 0 || p.coldstart + p.warmup > 0) && (rc = capture(r != 0, ph != 0)) != FMD_OK)
                        return rc;
        return FMD_OK;
    };
    if ((rc = capture_all()) != FMD_OK) return rc;
    if ((rc = ctx->sync_check("system init")) != FMD_OK) return rc;
    if (pending) {
        // the graphs hold the launch shapes: capture again with the tuned one
        if ((rc = tune_lj_pruned(true, nullptr)) != FMD_OK) return rc;
        drop_graphs();
        if ((rc = capture_all()) != FMD_OK) return rc;
    }
    initialized = true;
    return FMD_OK;
}

int System::capture(bool rebuild, bool phase, bool judge) {
    cudaGraphExec_t& ge = graphs[rebuild ? 1 : 0][phase ? 1 : 0][judge ? 1 : 0];
    if (ge) return FMD_OK;
    cudaStream_t st = ctx->stream;
    cudaGraph_t graph;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "graph capture failed to start");
    cudaError_t e = enqueue_variant(rebuild, phase, st, judge);
    cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, std::string("graph capture failed: ") +
                                           cudaGetErrorString(e != cudaSuccess ? e : e2));
    e = cudaGraphInstantiate(&ge, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, cudaGetErrorString(e));
    return FMD_OK;
}

cudaError_t System::enqueue_variant(bool rebuild, bool phase, cudaStream_t st, bool judge) {
    cudaError_t e;
    if (rebuild && (e = enqueue_rebuild(st)) != cudaSuccess) return e;
    return enqueue_step(arr, sp, phase, st, judge);
}

cudaError_t System::enqueue_one(int g, cudaStream_t st) {
    return enqueue_variant((g % p.nlup) == 0, g <= p.coldstart + p.warmup, st, judge_step(g));
}

int System::run(int first, int last, fmd_obs* obs) {
    int rc = enqueue(first, last);
    if (rc != FMD_OK) return rc;
    rc = ctx->sync_check("system run");
    if (rc != FMD_OK) return rc;
    if (obs) {
        if (cudaMemcpy(obs, &arr.S->obs, sizeof(fmd_obs), cudaMemcpyDeviceToHost) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "observable copy failed");
    }
    return FMD_OK;
}

int System::enqueue(int first, int last) {
    if (!initialized) return ctx->fail(FMD_ERR_STATE, "fmd_system_run before fmd_system_init");
    if (last < first) return FMD_OK;
    cudaStream_t st = ctx->stream;
    const int g0 = first - 1;
    cudaMemcpyAsync(&arr.S->gstep, &g0, sizeof(int), cudaMemcpyHostToDevice, st);
    for (int g = first; g <= last; g++) {
        if (p.use_graphs) {
            const int r = (g % p.nlup) == 0, ph = g <= p.coldstart + p.warmup, j = judge_step(g);
            int rc = capture(r != 0, ph != 0, j != 0);
            if (rc != FMD_OK) return rc;
            if (cudaGraphLaunch(graphs[r][ph][j], st) != cudaSuccess)
                return ctx->fail(FMD_ERR_CUDA, "graph launch failed");
        } else {
            if (enqueue_one(g, st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "step launch failed");
        }
    }
    return FMD_OK;
}

int System::nonfinite_check() {
    // Cheap watchdog on the scalars only; kernels never trap.
    SysScal s;
    if (cudaMemcpy(&s, arr.S, sizeof(s), cudaMemcpyDeviceToHost) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "scalar copy failed");
    if (!std::isfinite(s.KE) || !std::isfinite(s.E[0]) || !std::isfinite(s.h[0]))
        return ctx->fail(FMD_ERR_NONFINITE, "non-finite energy or cell");
    return FMD_OK;
}

}  // namespace fmd

// ------------------------------------------------------------------ C-ABI --

static int make_params(const fmd_run_params* p, fmd::System& s) {
    s.p = *p;
    if (s.p.nlup <= 0) return FMD_ERR_ARG;
    s.sp.dt = p->dt; s.sp.T = p->T; s.sp.T_cold = p->T_cold;
    s.sp.coldstart = p->coldstart; s.sp.warmup = p->warmup;
    s.sp.gavg_from = p->gavg_from; s.sp.gavg_to = p->gavg_to;
    s.sp.nc = p->nc > 0 ? p->nc : 1; s.sp.nmol = p->nmol > 0 ? p->nmol : 1;
    s.sp.schedule = 1;
    return FMD_OK;
}

extern "C" int fmd_system_create_rigid(fmd_ctx* ctx, const fmd_run_params* p, int n, int natom,
                                       const double* body, double I0, double Mmol, double rmcut,
                                       int max_neigh, const double* pos, const double* vel,
                                       const double* qv, const double* omg, const double* h,
                                       const fmd_npt* npt, fmd_system** out) {
    if (!ctx || !p || !out || !body || !pos || !vel || !qv || !omg || !h || !npt || n < 1 || natom < 1 ||
        natom > 96 || max_neigh < 1)
        return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_system_create_rigid: bad argument") : FMD_ERR_ARG;
    auto s = std::make_unique<fmd::System>();
    s->ctx = ctx;
    if (make_params(p, *s) != FMD_OK) return ctx->fail(FMD_ERR_ARG, "bad run parameters");
    s->arr.kind = FMD_SYS_RIGID;
    s->arr.n = n;
    s->arr.natom = natom;
    s->arr.Mmol = Mmol;
    s->arr.I0 = I0;
    s->arr.precision = p->precision;
    const double rmc = rmcut + 3.0;
    s->arr.rmcut2 = rmcut * rmcut;
    int rc = s->alloc_common(pos, vel, h, npt);
    if (rc != FMD_OK) return rc;
    double* bd; double* q; double* w; double* T;
    if (s->alloc(&bd, 3 * (size_t)natom, body) || s->alloc(&q, 4 * (size_t)n, qv) ||
        s->alloc(&w, 3 * (size_t)n, omg) || s->alloc(&T, 3 * (size_t)n, (const double*)nullptr))
        return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
    cudaMemsetAsync(T, 0, sizeof(double) * 3 * n, ctx->stream);
    s->arr.body = bd; s->arr.qv = q; s->arr.omg = w; s->arr.T = T;
    double* lab;
    if (s->alloc(&lab, (size_t)n * natom * kRigidLabDoubles, (const double*)nullptr))
        return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
    s->arr.rigid_lab = lab;
    // The list radius is rmcut+3 (LJ:259); the force kernel skips pairs
    // beyond rmcut (LJ:320).
    if ((rc = s->alloc_lists(rmc, max_neigh, 0.0, 0, false)) != FMD_OK) return rc;
    s->rc2_a = rmc * rmc;
    out[0] = new fmd_system{std::move(s)};
    return FMD_OK;
}

extern "C" int fmd_system_create_airebo(fmd_ctx* ctx, const fmd_run_params* p, int na, const double* pos,
                                        const double* vel, const double* mass, const int* mol_id,
                                        const double* h, const fmd_npt* npt, fmd_system** out) {
    if (!ctx || !p || !out || !pos || !vel || !mass || !mol_id || !h || !npt || na < 2)
        return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_system_create_airebo: bad argument") : FMD_ERR_ARG;
    auto s = std::make_unique<fmd::System>();
    s->ctx = ctx;
    if (make_params(p, *s) != FMD_OK) return ctx->fail(FMD_ERR_ARG, "bad run parameters");
    s->arr.kind = FMD_SYS_AIREBO;
    s->arr.n = na;
    s->arr.precision = p->precision;
    s->arr.lj_blocks = lj_gather_blocks(FMD_FF_AIREBO, p->precision, s->arr.lj_shape, 0);
    int rc = s->alloc_common(pos, vel, h, npt);
    if (rc != FMD_OK) return rc;
    double* m; int* mid;
    if (s->alloc(&m, na, mass) || s->alloc(&mid, na, mol_id)) return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
    s->arr.mass = m; s->arr.mol_id = mid;
    const double lj_rcut = 3.0 * 3.40;          // AI:120
    const double rebo_rcut = 2.0 + 0.3;         // AI:116
    if ((rc = s->alloc_lists(lj_rcut + 2.0, 400, rebo_rcut, 12, true)) != FMD_OK) return rc;
    if (fmd::mol_lists_alloc(s->mol, na, mol_id, s->owned_alloc()) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "list allocation failed");
    if ((rc = s->alloc_prune(lj_rcut)) != FMD_OK) return rc;
    out[0] = new fmd_system{std::move(s)};
    return FMD_OK;
}

namespace {
// An MM system; its topology comes from the full flat topology t, or when t
// is null from one molecule's topology t1 replicated over nmol molecules of
// natom_mol atoms on the device.
int create_mm(fmd_ctx* ctx, const fmd_run_params* p, int na, const double* pos, const double* vel,
              const int* mol_id, const fmd_mm_topology* t, const fmd_mm_topology* t1, int nmol, int natom_mol,
              const double* charge, const double* h, const fmd_npt* npt, fmd_system** out) {
    auto s = std::make_unique<fmd::System>();
    s->ctx = ctx;
    if (make_params(p, *s) != FMD_OK) return ctx->fail(FMD_ERR_ARG, "bad run parameters");
    s->arr.kind = FMD_SYS_MM;
    s->arr.n = na;
    s->arr.precision = p->precision;
    s->arr.lj_blocks = lj_gather_blocks(FMD_FF_MM, p->precision, s->arr.lj_shape, 0);
    int rc = s->alloc_common(pos, vel, h, npt);
    if (rc != FMD_OK) return rc;
    int* mid;
    if (s->alloc(&mid, na, mol_id)) return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
    s->arr.mol_id = mid;
    if ((rc = t ? s->upload_topology(t) : s->replicate_topology(t1, nmol, natom_mol)) != FMD_OK) return rc;
    bool has_charge = false;
    if (charge)
        for (int i = 0; i < na && !has_charge; i++) has_charge = std::fabs(charge[i]) > 1e-10;   // MM:1110
    s->arr.has_charge = has_charge ? 1 : 0;
    if (has_charge) {
        double* q;
        if (s->alloc(&q, na, charge)) return ctx->fail(FMD_ERR_CUDA, "device allocation failed");
        s->arr.charge = q;
    }
    const double rcut = 3.0 * 3.431;            // MM:114
    if ((rc = s->alloc_lists(rcut + 2.0, 400, 0.0, 0, true)) != FMD_OK) return rc;
    if (fmd::mol_lists_alloc(s->mol, na, mol_id, s->owned_alloc()) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "list allocation failed");
    if ((rc = s->alloc_prune(rcut)) != FMD_OK) return rc;
    out[0] = new fmd_system{std::move(s)};
    return FMD_OK;
}
}  // namespace

extern "C" int fmd_system_create_mm(fmd_ctx* ctx, const fmd_run_params* p, int na, const double* pos,
                                    const double* vel, const int* mol_id, const fmd_mm_topology* t,
                                    const double* charge, const double* h, const fmd_npt* npt,
                                    fmd_system** out) {
    if (!ctx || !p || !out || !pos || !vel || !mol_id || !t || !h || !npt || na < 2)
        return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_system_create_mm: bad argument") : FMD_ERR_ARG;
    return create_mm(ctx, p, na, pos, vel, mol_id, t, nullptr, 0, 0, charge, h, npt, out);
}

extern "C" int fmd_system_create_mm_replicated(fmd_ctx* ctx, const fmd_run_params* p, int nmol, int natom_mol,
                                               const double* pos, const double* vel, const fmd_mm_topology* t1,
                                               const double* h, const fmd_npt* npt, fmd_system** out) {
    if (!ctx || !p || !out || !pos || !vel || !t1 || !h || !npt || nmol < 1 || natom_mol < 1 ||
        (long long)nmol * natom_mol < 2 || (long long)nmol * natom_mol > (1LL << 30))
        return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_system_create_mm_replicated: bad argument") : FMD_ERR_ARG;
    const int na = nmol * natom_mol;
    std::vector<int> mol_id((size_t)na);
    for (int i = 0; i < na; i++) mol_id[i] = i / natom_mol;     // contiguous molecules, 0-based
    return create_mm(ctx, p, na, pos, vel, mol_id.data(), nullptr, t1, nmol, natom_mol, nullptr, h, npt, out);
}

int fmd::System::replicate_topology(const fmd_mm_topology* t, int nmol, int natom) {
    // One molecule's indices address its own atoms: check them on the host.
    auto ok = [&](const int* a, int m) {
        if (m > 0 && !a) return false;
        for (int k = 0; k < m; k++)
            if (a[k] < 0 || a[k] >= natom) return false;
        return true;
    };
    if (t->nb < 0 || t->nang < 0 || t->ndih < 0 || t->nimp < 0 || !ok(t->b_i0, t->nb) || !ok(t->b_i1, t->nb) ||
        !ok(t->ang_i0, t->nang) || !ok(t->ang_i1, t->nang) || !ok(t->ang_i2, t->nang) ||
        !ok(t->dih_i0, t->ndih) || !ok(t->dih_i1, t->ndih) || !ok(t->dih_i2, t->ndih) || !ok(t->dih_i3, t->ndih) ||
        !ok(t->imp_i0, t->nimp) || !ok(t->imp_i1, t->nimp) || !ok(t->imp_i2, t->nimp) || !ok(t->imp_i3, t->nimp))
        return ctx->fail(FMD_ERR_ARG, "MM molecule topology: index out of range");
    if (upload_topology_arrays(t) != FMD_OK) return FMD_ERR_CUDA;   // the molecule's terms
    const MMTopoDev mol = arr.topo;
    MMTopoOut o{};
    const size_t nb = (size_t)nmol * t->nb, na = (size_t)nmol * t->nang, nd = (size_t)nmol * t->ndih,
                 ni = (size_t)nmol * t->nimp;
    if (alloc(&o.b_i0, nb, (const int*)nullptr) || alloc(&o.b_i1, nb, (const int*)nullptr) ||
        alloc(&o.b_kb, nb, (const double*)nullptr) || alloc(&o.b_r0, nb, (const double*)nullptr) ||
        alloc(&o.a_i0, na, (const int*)nullptr) || alloc(&o.a_i1, na, (const int*)nullptr) ||
        alloc(&o.a_i2, na, (const int*)nullptr) || alloc(&o.a_kth, na, (const double*)nullptr) ||
        alloc(&o.a_th0, na, (const double*)nullptr) || alloc(&o.d_i0, nd, (const int*)nullptr) ||
        alloc(&o.d_i1, nd, (const int*)nullptr) || alloc(&o.d_i2, nd, (const int*)nullptr) ||
        alloc(&o.d_i3, nd, (const int*)nullptr) || alloc(&o.d_vn, nd, (const double*)nullptr) ||
        alloc(&o.d_mult, nd, (const int*)nullptr) || alloc(&o.d_gamma, nd, (const double*)nullptr) ||
        alloc(&o.m_i0, ni, (const int*)nullptr) || alloc(&o.m_i1, ni, (const int*)nullptr) ||
        alloc(&o.m_i2, ni, (const int*)nullptr) || alloc(&o.m_i3, ni, (const int*)nullptr) ||
        alloc(&o.m_ki, ni, (const double*)nullptr) || alloc(&o.m_gamma, ni, (const double*)nullptr))
        return ctx->fail(FMD_ERR_CUDA, "topology allocation failed");
    if (mm_replicate_launch(mol, nmol, natom, o, ctx->stream) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "topology replication failed");
    MMTopoDev d{};
    d.nb = (int)nb; d.nang = (int)na; d.ndih = (int)nd; d.nimp = (int)ni;
    d.b_i0 = o.b_i0; d.b_i1 = o.b_i1; d.b_kb = o.b_kb; d.b_r0 = o.b_r0;
    d.a_i0 = o.a_i0; d.a_i1 = o.a_i1; d.a_i2 = o.a_i2; d.a_kth = o.a_kth; d.a_th0 = o.a_th0;
    d.d_i0 = o.d_i0; d.d_i1 = o.d_i1; d.d_i2 = o.d_i2; d.d_i3 = o.d_i3; d.d_vn = o.d_vn; d.d_mult = o.d_mult;
    d.d_gamma = o.d_gamma;
    d.m_i0 = o.m_i0; d.m_i1 = o.m_i1; d.m_i2 = o.m_i2; d.m_i3 = o.m_i3; d.m_ki = o.m_ki; d.m_gamma = o.m_gamma;
    arr.topo = d;
    return ctx->sync_check("topology replication");
}

int fmd::System::upload_topology(const fmd_mm_topology* t) {
    // Topology indices address device arrays: check them before any launch.
    auto ok = [&](const int* a, int m) {
        if (m > 0 && !a) return false;
        for (int k = 0; k < m; k++)
            if (a[k] < 0 || a[k] >= arr.n) return false;
        return true;
    };
    if (t->nb < 0 || t->nang < 0 || t->ndih < 0 || t->nimp < 0 || !ok(t->b_i0, t->nb) || !ok(t->b_i1, t->nb) ||
        !ok(t->ang_i0, t->nang) || !ok(t->ang_i1, t->nang) || !ok(t->ang_i2, t->nang) ||
        !ok(t->dih_i0, t->ndih) || !ok(t->dih_i1, t->ndih) || !ok(t->dih_i2, t->ndih) || !ok(t->dih_i3, t->ndih) ||
        !ok(t->imp_i0, t->nimp) || !ok(t->imp_i1, t->nimp) || !ok(t->imp_i2, t->nimp) || !ok(t->imp_i3, t->nimp))
        return ctx->fail(FMD_ERR_ARG, "MM topology: index out of range");
    return upload_topology_arrays(t);
}

// Copies the topology arrays of t to the device as the system's topology
// (indices already checked).
int fmd::System::upload_topology_arrays(const fmd_mm_topology* t) {
    MMTopoDev d{};
    d.nb = t->nb; d.nang = t->nang; d.ndih = t->ndih; d.nimp = t->nimp;
    int *i0, *i1, *i2, *i3, *mult;
    double *x0, *x1, *x2;
    if (alloc(&i0, t->nb, t->b_i0) || alloc(&i1, t->nb, t->b_i1) || alloc(&x0, t->nb, t->b_kb) ||
        alloc(&x1, t->nb, t->b_r0))
        return ctx->fail(FMD_ERR_CUDA, "topology upload failed");
    d.b_i0 = i0; d.b_i1 = i1; d.b_kb = x0; d.b_r0 = x1;
    if (alloc(&i0, t->nang, t->ang_i0) || alloc(&i1, t->nang, t->ang_i1) || alloc(&i2, t->nang, t->ang_i2) ||
        alloc(&x0, t->nang, t->ang_kth) || alloc(&x1, t->nang, t->ang_th0))
        return ctx->fail(FMD_ERR_CUDA, "topology upload failed");
    d.a_i0 = i0; d.a_i1 = i1; d.a_i2 = i2; d.a_kth = x0; d.a_th0 = x1;
    if (alloc(&i0, t->ndih, t->dih_i0) || alloc(&i1, t->ndih, t->dih_i1) || alloc(&i2, t->ndih, t->dih_i2) ||
        alloc(&i3, t->ndih, t->dih_i3) || alloc(&x0, t->ndih, t->dih_vn) || alloc(&mult, t->ndih, t->dih_mult) ||
        alloc(&x2, t->ndih, t->dih_gamma))
        return ctx->fail(FMD_ERR_CUDA, "topology upload failed");
    d.d_i0 = i0; d.d_i1 = i1; d.d_i2 = i2; d.d_i3 = i3; d.d_vn = x0; d.d_mult = mult; d.d_gamma = x2;
    if (alloc(&i0, t->nimp, t->imp_i0) || alloc(&i1, t->nimp, t->imp_i1) || alloc(&i2, t->nimp, t->imp_i2) ||
        alloc(&i3, t->nimp, t->imp_i3) || alloc(&x0, t->nimp, t->imp_ki) || alloc(&x1, t->nimp, t->imp_gamma))
        return ctx->fail(FMD_ERR_CUDA, "topology upload failed");
    d.m_i0 = i0; d.m_i1 = i1; d.m_i2 = i2; d.m_i3 = i3; d.m_ki = x0; d.m_gamma = x1;
    arr.topo = d;
    return FMD_OK;
}

extern "C" int fmd_system_init(fmd_system* s) {
    if (!s) return FMD_ERR_ARG;
    return s->sys->init();
}

extern "C" int fmd_system_run(fmd_system* s, int first, int last, fmd_obs* obs) {
    if (!s) return FMD_ERR_ARG;
    return s->sys->run(first, last, obs);
}

extern "C" int fmd_system_enqueue(fmd_system* s, int first, int last) {
    if (!s) return FMD_ERR_ARG;
    return s->sys->enqueue(first, last);
}

extern "C" int fmd_system_enqueue_obs(fmd_system* s, int first, int last, fmd_obs* obs) {
    if (!s || !s->sys || !obs) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    int rc = y.enqueue(first, last);
    if (rc != FMD_OK) return rc;
    cudaEvent_t& ev = y.obs_ev[last & 1];
    if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_enqueue_obs: event creation failed");
    if (cudaMemcpyAsync(obs, &y.arr.S->obs, sizeof(fmd_obs), cudaMemcpyDeviceToHost, y.ctx->stream) != cudaSuccess ||
        cudaEventRecord(ev, y.ctx->stream) != cudaSuccess)
        return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_enqueue_obs: copy failed");
    return FMD_OK;
}

extern "C" int fmd_system_wait_obs(fmd_system* s, int step) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    cudaEvent_t ev = y.obs_ev[step & 1];
    if (!ev) return y.ctx->fail(FMD_ERR_STATE, "fmd_system_wait_obs: no copy enqueued for this step");
    const cudaError_t e = cudaEventSynchronize(ev);
    if (e != cudaSuccess) return y.ctx->fail(FMD_ERR_CUDA, std::string("fmd_system_wait_obs: ") + cudaGetErrorString(e));
    return FMD_OK;
}

extern "C" int fmd_system_averages(fmd_system* s, fmd_avg* avg) {
    if (!s || !avg) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (cudaMemcpy(avg, &y.arr.S->avg, sizeof(fmd_avg), cudaMemcpyDeviceToHost) != cudaSuccess)
        return y.ctx->fail(FMD_ERR_CUDA, "average copy failed");
    return FMD_OK;
}

extern "C" int fmd_system_download(fmd_system* s, double* pos, double* vel, double* qv, double* omg, double* h,
                                   fmd_npt* npt) {
    if (!s) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    cudaStream_t st = y.ctx->stream;
    const size_t n = y.arr.n;
    if (pos) cudaMemcpyAsync(pos, y.arr.pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st);
    if (vel) cudaMemcpyAsync(vel, y.arr.vel, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st);
    if (qv && y.arr.qv) cudaMemcpyAsync(qv, y.arr.qv, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st);
    if (omg && y.arr.omg) cudaMemcpyAsync(omg, y.arr.omg, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st);
    if (h) cudaMemcpyAsync(h, y.arr.S->h, sizeof(double) * 9, cudaMemcpyDeviceToHost, st);
    if (npt) cudaMemcpyAsync(npt, &y.arr.S->npt, sizeof(fmd_npt), cudaMemcpyDeviceToHost, st);
    return y.ctx->sync_check("system download");
}

extern "C" int fmd_system_forces(fmd_system* s, double* F, double* T, double* E) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    cudaStream_t st = y.ctx->stream;
    const size_t n = y.arr.n;
    if (F) cudaMemcpyAsync(F, y.arr.F, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st);
    if (T && y.arr.T) cudaMemcpyAsync(T, y.arr.T, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st);
    if (E) cudaMemcpyAsync(E, y.arr.S->E, sizeof(double) * 8, cudaMemcpyDeviceToHost, st);
    return y.ctx->sync_check("system forces");
}

extern "C" int fmd_system_lj_rows(fmd_system* s, int* full_cnt, int* pruned_cnt) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    cudaStream_t st = y.ctx->stream;
    const size_t n = y.arr.n;
    if (full_cnt && y.arr.in_cnt) cudaMemcpyAsync(full_cnt, y.arr.in_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    if (pruned_cnt && y.prune.ok) cudaMemcpyAsync(pruned_cnt, y.prune.cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    return y.ctx->sync_check("system LJ rows");
}

extern "C" int fmd_system_set_physics(fmd_system* s, int flags) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (y.initialized) return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_physics: call before fmd_system_init");
    if (flags & ~(FMD_PHYS_MM_BONDED | FMD_PHYS_REBO | FMD_PHYS_QUAT))
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_physics: unknown flag");
    if ((flags & FMD_PHYS_QUAT) && y.arr.kind != FMD_SYS_RIGID)
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_physics: FMD_PHYS_QUAT needs a rigid system");
    if ((flags & FMD_PHYS_MM_BONDED) && y.arr.kind != FMD_SYS_MM)
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_physics: FMD_PHYS_MM_BONDED needs an MM system");
    if ((flags & FMD_PHYS_REBO) && (y.arr.kind != FMD_SYS_AIREBO || !y.arr.rebo_slots))
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_physics: FMD_PHYS_REBO needs an AIREBO system");
    y.arr.topo.physical = (flags & FMD_PHYS_MM_BONDED) ? 1 : 0;
    y.arr.rebo_phys = (flags & FMD_PHYS_REBO) ? 1 : 0;
    y.arr.quat_left = (flags & FMD_PHYS_QUAT) ? 1 : 0;
    return FMD_OK;
}

extern "C" int fmd_system_set_rebo2(fmd_system* s, const fmd_rebo2_knots* kn, int flags) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (y.initialized) return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_rebo2: call before fmd_system_init");
    if (flags & ~(FMD_REBO2_BOND_ORDER | FMD_REBO2_LJ_SWITCH))
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_rebo2: unknown flag");
    if (flags && y.arr.kind != FMD_SYS_AIREBO)
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_rebo2: needs an AIREBO system");
    if (flags && !kn) return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_rebo2: no knots");
    if ((flags & FMD_REBO2_BOND_ORDER) && y.arr.sg)
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_rebo2: the system uses a learned REBO term");
    if (flags) {
        static_assert(sizeof(fmd_rebo2_knots) == sizeof(double) * fmd::kRebo2Knots, "knot layout");
        std::vector<double> c(fmd::kRebo2PccCoef + 2 * (size_t)fmd::kRebo2TriCoef);
        fmd::rebo2_coeffs(&kn->pcc[0][0], c.data(), c.data() + fmd::kRebo2PccCoef,
                          c.data() + fmd::kRebo2PccCoef + fmd::kRebo2TriCoef);
        if (!y.arr.rebo2.pcc) {
            const size_t n = (size_t)y.arr.n;
            double *tab, *nc, *sw;
            int2 *bonds, *pairs;
            int* counts;
            if (y.alloc(&tab, c.size(), (const double*)nullptr) || y.alloc(&nc, n, (const double*)nullptr) ||
                y.alloc(&sw, (size_t)fmd::kForceBlocks * fmd::kNV, (const double*)nullptr) ||
                y.alloc(&bonds, n * y.arr.cap_b, (const int2*)nullptr) ||
                y.alloc(&pairs, n * fmd::kRebo2SwitchPerAtom, (const int2*)nullptr) ||
                y.alloc(&counts, 2, (const int*)nullptr))
                return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_set_rebo2: allocation failed");
            fmd::Rebo2Dev& t = y.arr.rebo2;
            t.pcc = tab;
            t.pirc = tab + fmd::kRebo2PccCoef;
            t.tcc = tab + fmd::kRebo2PccCoef + fmd::kRebo2TriCoef;
            t.ncoord = nc;
            t.bonds = bonds;
            t.sw_pairs = pairs;
            t.counts = counts;
            t.sw_cap = (int)(n * fmd::kRebo2SwitchPerAtom);
            t.err = y.ctx->d_err;
            y.arr.part_sw = sw;
        }
        if (cudaMemcpyAsync(const_cast<double*>(y.arr.rebo2.pcc), c.data(), sizeof(double) * c.size(),
                            cudaMemcpyHostToDevice, y.ctx->stream) != cudaSuccess)
            return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_set_rebo2: copy failed");
    }
    y.arr.rebo2_flags = flags;
    return y.ctx->sync_check("fmd_system_set_rebo2");
}

extern "C" int fmd_system_lj_full_rows(fmd_system* s, int* cnt, int* list, int* stride) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (stride) *stride = y.arr.in_list ? y.arr.in_cap : 0;
    if (!y.arr.in_list) return FMD_OK;
    cudaStream_t st = y.ctx->stream;
    const size_t n = y.arr.n;
    if (cnt) cudaMemcpyAsync(cnt, y.arr.in_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    if (list) cudaMemcpyAsync(list, y.arr.in_list, sizeof(int) * n * y.arr.in_cap, cudaMemcpyDeviceToHost, st);
    return y.ctx->sync_check("system LJ full rows");
}

extern "C" int fmd_system_lists(fmd_system* s, int* cnt_a, int* list_a, int* cnt_b, int* list_b) {
    if (!s) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    cudaStream_t st = y.ctx->stream;
    const size_t n = y.arr.n;
    if (cnt_a) cudaMemcpyAsync(cnt_a, y.arr.cnt_a, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    if (list_a) cudaMemcpyAsync(list_a, y.arr.list_a, sizeof(int) * n * y.arr.cap_a, cudaMemcpyDeviceToHost, st);
    if (cnt_b && y.arr.cnt_b) cudaMemcpyAsync(cnt_b, y.arr.cnt_b, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    if (list_b && y.arr.list_b)
        cudaMemcpyAsync(list_b, y.arr.list_b, sizeof(int) * n * y.arr.cap_b, cudaMemcpyDeviceToHost, st);
    return y.ctx->sync_check("system lists");
}

extern "C" int fmd_system_kernel_ms(fmd_system* s, int stage, int reps, double* ms) {
    if (!s || !ms || reps < 1 || stage < 0 || stage > 5) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (!y.initialized) return y.ctx->fail(FMD_ERR_STATE, "kernel timing before init");
    cudaStream_t st = y.ctx->stream;
    const StepArrays& a = y.arr;
    const double* hh = a.S->h;
    auto launch = [&]() -> cudaError_t {
        switch (stage) {
            case 0:
                if (a.kind == FMD_SYS_RIGID)
                    return rigid_launch(a.precision, a.pos, a.qv, a.body, hh, a.cnt_a, a.list_a, a.cap_a, a.n,
                                        a.natom, a.rmcut2, a.F, a.T, a.part_f1, st, a.rigid_lab, a.rigid_shape);
                // Timed into the scratch accumulator (F itself is left alone).
                return lj_gather_launch(a.kind == FMD_SYS_AIREBO ? FMD_FF_AIREBO : FMD_FF_MM, a.pos, hh, a.cnt_a,
                                        a.list_a, a.cap_a, a.in_cnt, a.in_list, a.in_cap, a.n, a.Facc, a.Facc,
                                        a.part_f2, st, a.precision, a.lj_shape, a.err);
            case 1:
                if (a.kind == FMD_SYS_AIREBO && (a.rebo2_flags & FMD_REBO2_BOND_ORDER))   // the REBO term the step uses
                    return rebo2_launch(a.rebo2, a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.Facc, a.part_f1,
                                        a.rebo_blocks, st);
                if (a.kind == FMD_SYS_AIREBO && a.sg)
                    return sg_enqueue_rebo(*a.sg, a, false, st);
                if (a.kind == FMD_SYS_AIREBO)
                    return rebo_slots_launch(a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.rebo_slots, a.Facc,
                                             a.part_f1, kForceBlocks, nullptr, 0, st, a.rebo_ids, a.rebo_phys != 0);
                if (a.kind == FMD_SYS_MM) return mm_bonded_launch(a.topo, a.pos, hh, a.Facc, a.part_f1, st);
                return rigid_launch(a.precision, a.pos, a.qv, a.body, hh, a.cnt_a, a.list_a, a.cap_a, a.n, a.natom,
                                    a.rmcut2, a.F, a.T, a.part_f1, st, a.rigid_lab, a.rigid_shape);
            case 2:
                return y.enqueue_rebuild(st);
            case 4:
                // the gather over the pruned rows of the last prune, into the scratch accumulator
                if (!a.prune) return cudaErrorInvalidValue;
                return lj_gather_launch(a.kind == FMD_SYS_AIREBO ? FMD_FF_AIREBO : FMD_FF_MM, a.pos, hh, a.cnt_a,
                                        a.list_a, a.cap_a, a.prune->cnt, a.prune->list, a.in_cap, a.n, a.Facc,
                                        a.Facc, a.part_f2, st, a.precision, a.lj_shape_p, a.err);
            case 5:
                // the switched-LJ correction, into the scratch accumulator
                if (!(a.rebo2_flags & FMD_REBO2_LJ_SWITCH)) return cudaErrorInvalidValue;
                return lj_switch_launch(a.rebo2, a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.cnt_a, a.list_a, a.cap_a,
                                        a.n, a.Facc, a.part_sw, kForceBlocks, false, st);
            default:
                return enqueue_forces(a, st);
        }
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();   // warm
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; r++) launch();
    cudaEventRecord(e1, st);
    cudaError_t err = cudaEventSynchronize(e1);
    float tot = 0.f;
    cudaEventElapsedTime(&tot, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // Restore the invariant that the accumulator is zero between steps and
    // that F holds the forces of the current positions.
    cudaMemsetAsync(a.Facc, 0, sizeof(double) * 3 * a.n, st);
    if (stage != 2) {
        enqueue_forces(a, st);
        enqueue_force_reduce(a, st);
    }
    int rc = y.ctx->sync_check("kernel timing");
    if (err != cudaSuccess) return y.ctx->fail(FMD_ERR_CUDA, cudaGetErrorString(err));
    *ms = (double)tot / reps;
    return rc;
}

extern "C" int fmd_system_virial(fmd_system* s, double* W9, double* KE) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    SysScal h;
    if (cudaMemcpyAsync(&h, y.arr.S, sizeof(h), cudaMemcpyDeviceToHost, y.ctx->stream) != cudaSuccess)
        return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_virial: copy failed");
    const int rc = y.ctx->sync_check("fmd_system_virial");
    if (rc != FMD_OK) return rc;
    if (W9) std::memcpy(W9, h.W9, sizeof(double) * 9);
    if (KE) *KE = h.KE;
    return FMD_OK;
}

extern "C" int fmd_system_set_lj_shape(fmd_system* s, int threads, int unroll, int feed) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (y.arr.kind == FMD_SYS_RIGID || (threads != 128 && threads != 256) || (unroll != 2 && unroll != 4) ||
        !lj_feed_valid(feed))
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_lj_shape: bad shape");
    const LJShape sh{threads, unroll, feed & 3, feed >> 2};
    const int ff = y.arr.kind == FMD_SYS_AIREBO ? FMD_FF_AIREBO : FMD_FF_MM;
    const int nb = lj_gather_blocks(ff, y.arr.precision, sh, y.arr.in_cap);
    if (nb < 1) return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_lj_shape: shape cannot run with this list");
    if (cudaStreamSynchronize(y.ctx->stream) != cudaSuccess) return y.ctx->fail(FMD_ERR_CUDA, "sync failed");
    y.drop_graphs();                     // captured graphs hold the old launch
    y.arr.lj_shape = sh;
    y.arr.lj_shape_p = sh;
    y.arr.lj_blocks = nb;
    if (y.arr.sg) {                      // keep the learned term's graph variants too
        int rc = FMD_OK;
        for (int r = 0; r < 2 && rc == FMD_OK; r++)
            for (int ph = 0; ph < 2 && rc == FMD_OK; ph++)
                for (int j = 0; j < 2 && rc == FMD_OK; j++) rc = y.capture(r != 0, ph != 0, j != 0);
        return rc;
    }
    return FMD_OK;
}

extern "C" int fmd_system_set_lj_prune(fmd_system* s, double delta) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (!(delta >= 0.0 && delta <= 10.0))
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_lj_prune: delta must lie in [0, 10] A");
    if (!y.prune.ok) {
        if (delta == 0.0) return FMD_OK;
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_set_lj_prune: the system has no LJ gather rows");
    }
    if (y.prune.delta == delta) return FMD_OK;
    if (cudaStreamSynchronize(y.ctx->stream) != cudaSuccess) return y.ctx->fail(FMD_ERR_CUDA, "sync failed");
    y.drop_graphs();                     // captured graphs hold the old launches
    y.prune.delta = delta;
    y.arr.prune_delta = delta;
    if (lj_prune_mark(y.prune, y.ctx->stream) != cudaSuccess) return y.ctx->fail(FMD_ERR_CUDA, "prune mark failed");
    if (y.initialized && y.p.use_graphs) {
        int rc = FMD_OK;
        const int nj = y.arr.sg ? 2 : 1;
        for (int r = 0; r < 2 && rc == FMD_OK; r++)
            for (int ph = 0; ph < 2 && rc == FMD_OK; ph++)
                for (int j = 0; j < nj && rc == FMD_OK; j++) rc = y.capture(r != 0, ph != 0, j != 0);
        return rc;
    }
    return FMD_OK;
}

extern "C" int fmd_system_lj_prune(fmd_system* s, double* delta, long long* evaluations, long long* prunes) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (delta) *delta = y.prune.ok ? y.prune.delta : 0.0;
    unsigned long long st[2] = {0ull, 0ull};
    if (y.prune.ok && (evaluations || prunes)) {
        if (cudaStreamSynchronize(y.ctx->stream) != cudaSuccess ||
            cudaMemcpy(st, y.prune.stats, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess)
            return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_lj_prune: read failed");
    }
    if (evaluations) *evaluations = (long long)st[0];
    if (prunes) *prunes = (long long)st[1];
    return FMD_OK;
}

extern "C" int fmd_system_lj_shape_pruned(fmd_system* s, int* threads, int* unroll, int* feed) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    const StepArrays& a = s->sys->arr;
    if (threads) *threads = a.lj_shape_p.threads;
    if (unroll) *unroll = a.lj_shape_p.unroll;
    if (feed) *feed = a.lj_shape_p.pipe | (a.lj_shape_p.contig << 2);
    return FMD_OK;
}

extern "C" int fmd_system_lj_shape(fmd_system* s, int* threads, int* unroll, int* pipelined, int* blocks) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    const StepArrays& a = s->sys->arr;
    if (threads) *threads = a.lj_shape.threads;
    if (unroll) *unroll = a.lj_shape.unroll;
    if (pipelined) *pipelined = a.lj_shape.pipe | (a.lj_shape.contig << 2);
    if (blocks) *blocks = a.lj_blocks;
    return FMD_OK;
}

extern "C" int fmd_system_site_pairs(fmd_system* s, long long* pairs) {
    if (!s || !s->sys || !pairs) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    const StepArrays& a = y.arr;
    if (a.kind != FMD_SYS_RIGID) return y.ctx->fail(FMD_ERR_ARG, "fmd_system_site_pairs: not a rigid system");
    if (!y.initialized) return y.ctx->fail(FMD_ERR_STATE, "fmd_system_site_pairs before init");
    unsigned long long* d = nullptr;
    unsigned long long h = 0;
    if (cudaMalloc(&d, sizeof(unsigned long long)) != cudaSuccess)
        return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_site_pairs: allocation failed");
    cudaStream_t st = y.ctx->stream;
    cudaError_t e = rigid_count_pairs(a.pos, a.qv, a.body, a.S->h, a.cnt_a, a.list_a, a.cap_a, a.n, a.natom,
                                      a.rmcut2, a.rigid_lab, d, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return y.ctx->fail(FMD_ERR_CUDA, cudaGetErrorString(e));
    *pairs = (long long)h;
    return FMD_OK;
}

extern "C" int fmd_system_step_kernels(fmd_system* s, int rebuild, int phase, int* nk) {
    if (!s || !nk) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    cudaStream_t st = y.ctx->stream;
    cudaGraph_t graph;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return y.ctx->fail(FMD_ERR_CUDA, "capture failed");
    cudaError_t e = y.enqueue_variant(rebuild != 0, phase != 0, st, (phase & 2) != 0);
    cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) return y.ctx->fail(FMD_ERR_CUDA, "capture failed");
    size_t n = 0;
    int k = 0;
    if (cudaGraphGetNodes(graph, nullptr, &n) == cudaSuccess) {
        std::vector<cudaGraphNode_t> nodes(n);
        if (n && cudaGraphGetNodes(graph, nodes.data(), &n) != cudaSuccess) n = 0;
        for (size_t q = 0; q < n; q++) {
            cudaGraphNodeType t = cudaGraphNodeTypeEmpty;
            if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
        }
    }
    cudaGraphDestroy(graph);
    cudaGetLastError();          // a failed graph query leaves no error for the next launch check
    *nk = k;
    return FMD_OK;
}

extern "C" int fmd_system_destroy(fmd_system* s) {
    if (!s) return FMD_OK;
    if (s->sys) {
        cudaStreamSynchronize(s->sys->ctx->stream);
        s->sys->release();
    }
    delete s;
    return FMD_OK;
}

// ------------------------------------------------- learned REBO term ------
int fmd::System::use_surrogate(fmd_sg* model, int judge_every, double rmse_max) {
    cudaStream_t st = ctx->stream;
    if (cudaStreamSynchronize(st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "fmd_system_use_surrogate: sync");
    drop_graphs();                       // captured graphs hold the old REBO term
    if (!model) {
        arr.sg = nullptr;
        arr.rebo_blocks = kForceBlocks;
    } else {
        if (arr.rebo2_flags & FMD_REBO2_BOND_ORDER)
            return ctx->fail(FMD_ERR_ARG, "fmd_system_use_surrogate: the system uses the REBO-II bond order");
        if (!sg) {
            auto g = std::make_unique<SgStep>();
            if (sg::work_alloc(g->work, arr.n, arr.cap_b) != cudaSuccess)
                return ctx->fail(FMD_ERR_CUDA, "fmd_system_use_surrogate: workspace allocation failed");
            if (alloc(&g->Fj, 3 * (size_t)arr.n, (const double*)nullptr) ||
                alloc(&g->part_j, (size_t)sg::kRowBlocks * kNV, (const double*)nullptr)) {
                sg::work_free(g->work);
                return ctx->fail(FMD_ERR_CUDA, "fmd_system_use_surrogate: allocation failed");
            }
            sg = std::move(g);
        }
        sg_model_images(model, &sg->img, &sg->vec);
        sg->judge_every = judge_every;
        sg->rmse_max = rmse_max;
        arr.sg = sg.get();
        arr.rebo_blocks = sg::kRowBlocks;
        // part_f1 holds max(kForceBlocks, n) records; the learned term writes kRowBlocks.
        if (std::max(kForceBlocks, arr.n) < sg::kRowBlocks) {
            double* p1;
            if (alloc(&p1, (size_t)sg::kRowBlocks * kNV, (const double*)nullptr))
                return ctx->fail(FMD_ERR_CUDA, "fmd_system_use_surrogate: allocation failed");
            arr.part_f1 = p1;
        }
    }
    // fresh judge record: the learned term is active again
    SysScal z;
    std::memset(&z, 0, sizeof(z));
    const size_t off = offsetof(SysScal, sg_off);
    if (cudaMemcpyAsync(reinterpret_cast<char*>(arr.S) + off, reinterpret_cast<const char*>(&z) + off,
                        sizeof(SysScal) - off, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "fmd_system_use_surrogate: copy failed");
    int rc = ctx->sync_check("fmd_system_use_surrogate");
    if (rc != FMD_OK || !initialized) return rc;
    // The forces of the current state come from the new REBO term.
    if (enqueue_forces(arr, st) != cudaSuccess || enqueue_force_reduce(arr, st) != cudaSuccess)
        return ctx->fail(FMD_ERR_CUDA, "fmd_system_use_surrogate: force launch failed");
    if ((rc = ctx->sync_check("fmd_system_use_surrogate")) != FMD_OK) return rc;
    if (p.use_graphs)
        for (int r = 0; r < 2; r++)
            for (int ph = 0; ph < 2; ph++)
                for (int j = 0; j < 2; j++)
                    if ((j == 0 || arr.sg) && (rc = capture(r != 0, ph != 0, j != 0)) != FMD_OK) return rc;
    return FMD_OK;
}

extern "C" int fmd_system_use_surrogate(fmd_system* s, fmd_sg* model, int judge_every, double rmse_max) {
    if (!s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (y.arr.kind != FMD_SYS_AIREBO)
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_use_surrogate: not an AIREBO system");
    if (model && (judge_every < 0 || !(rmse_max > 0.0)))
        return y.ctx->fail(FMD_ERR_ARG, "fmd_system_use_surrogate: judge_every < 0 or rmse_max <= 0");
    return y.use_surrogate(model, judge_every, rmse_max);
}

extern "C" int fmd_system_surrogate_status(fmd_system* s, fmd_sg_status* out) {
    if (!s || !s->sys || !out) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    SysScal h;
    if (cudaMemcpyAsync(&h, y.arr.S, sizeof(h), cudaMemcpyDeviceToHost, y.ctx->stream) != cudaSuccess)
        return y.ctx->fail(FMD_ERR_CUDA, "fmd_system_surrogate_status: copy failed");
    int rc = y.ctx->sync_check("fmd_system_surrogate_status");
    if (rc != FMD_OK) return rc;
    out->attached = y.arr.sg != nullptr;
    out->active = y.arr.sg != nullptr && h.sg_off == 0;
    out->judged = h.sg_judged;
    out->takeover_step = h.sg_takeover;
    out->rmse_last = h.sg_rmse_last;
    out->rmse_max = h.sg_rmse_max;
    return FMD_OK;
}

// Training snapshot of an AIREBO system: its positions, cell and current REBO
// list, with reference values from the plain REBO kernel (sg_abi.cu).
extern "C" int fmd_sg_data_add_system(fmd_sg_data* d, fmd_system* s) {
    if (!d || !s || !s->sys) return FMD_ERR_ARG;
    fmd::System& y = *s->sys;
    if (y.arr.kind != FMD_SYS_AIREBO)
        return y.ctx->fail(FMD_ERR_ARG, "fmd_sg_data_add_system: not an AIREBO system");
    if (!y.initialized) return y.ctx->fail(FMD_ERR_STATE, "fmd_sg_data_add_system: system not initialised");
    return fmd::sg_data_add_device(d, y.arr.pos, y.arr.S->h, y.arr.cnt_b, y.arr.list_b, y.arr.cap_b, y.arr.n,
                                   y.ctx->stream);
}
