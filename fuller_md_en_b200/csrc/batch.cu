// batch.cu -- many independent replicas advanced together (no counterpart in
// the reference, whose programs run one system each).
//
// A batch bundles R device-resident systems of one kind (MM) that may differ
// in size, cell, temperature and pressure.  Each phase of the step -- the
// scalar half-steps, the kicks, the bonded terms, the LJ gather, the
// reductions -- is ONE launch over all replicas: a block-offset table maps
// block b to (replica, local block), so every replica keeps its own grid and
// partial records and its results are those of the same kernels run on that
// system alone.  List rebuilds (every nlup steps) run per replica on forked
// streams that the graph captures as parallel branches.  Each step variant
// {rebuild, cold/warm phase} is one CUDA graph covering the whole batch.
//
// An autotuner times the LJ gather (threads per block, atoms per block,
// list entries in flight per lane) and the bonded kernel (threads per block,
// terms per block) on the batch itself at creation and keeps the fastest;
// results are cached per (device, replicas, atoms) for the process.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "molnlist.h"
#include "step.h"
#include "system.h"

using namespace fmd;

namespace {

constexpr int kAtomThreads = 256;   // per-particle kernels (kicks, rescale)
constexpr int kSideStreams = 8;     // parallel branches of a rebuild

struct Tune {
    int lj_threads = 256, lj_unroll = 4, lj_apb = 16;   // apb: atoms per block
    int lj_staged = 0;                                   // rows staged in shared memory
    int f1_threads = 128, f1_tpb = 512;                  // tpb: terms per block
    double lj_ms = 0, f1_ms = 0;
};

std::map<std::tuple<int, int, long long>, Tune>& tune_cache() {
    static std::map<std::tuple<int, int, long long>, Tune> m;
    return m;
}

int blocks_for(long long work, int per_block) {
    const long long b = (work + per_block - 1) / per_block;
    return (int)std::max(1LL, std::min<long long>(b, kForceBlocks));
}

}  // namespace

struct fmd_batch {
    fmd_ctx* ctx = nullptr;
    std::vector<System*> sys;
    int R = 0;
    long long natoms = 0;
    StepArrays* dA = nullptr;
    StepParams* dP = nullptr;
    int* dOff = nullptr;                 // [3 * (R + 1)]: atom, lj, f1 block offsets
    BatchDev bd;
    Tune tune;
    cudaGraphExec_t graphs[2][2] = {};
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kSideStreams] = {};
    // Batched list rebuild (every replica on the candidate-bitmap molecule
    // path): replica table and block offsets on the device.
    bool molb = false;
    MolRep* dReps = nullptr;
    int* dMolOff = nullptr;
    MolBatch mb;

    // Replica table and block offsets of the batched rebuild; leaves molb
    // false (per-replica rebuild branches) unless every replica has equal
    // molecules of 32-64 atoms, the path the batched kernels implement.
    int setup_mol_batch() {
        for (System* s : sys)
            if (!(s->mol.ok && s->mol.masks) || s->arr.kind != FMD_SYS_MM) return FMD_OK;
        std::vector<MolRep> reps(R);
        std::vector<int> off(3 * (R + 1), 0);
        long long ntot = 0;
        for (System* s : sys) ntot += s->arr.n;
        constexpr int kRowBlocks = kSMs * 8;     // the single-system row kernels' grid
        for (int r = 0; r < R; r++) {
            System* s = sys[r];
            MolRep& q = reps[r];
            q.m = s->mol;
            q.pos = s->arr.pos;
            q.hh = s->arr.S->h;
            q.rc = s->rc_a;
            q.rc2 = s->rc2_a;
            q.cap = s->arr.cap_a;
            q.in_cap = s->arr.in_cap;
            q.cnt = const_cast<int*>(s->arr.cnt_a);
            q.list = const_cast<int*>(s->arr.list_a);
            q.dropped = s->dropped;
            q.in_cnt = const_cast<int*>(s->arr.in_cnt);
            q.in_list = const_cast<int*>(s->arr.in_list);
            q.err = ctx->d_err;
            q.prune_words = s->prune.ok ? s->prune.words : nullptr;
            const int M = s->mol.M;
            const int share = (int)std::max(1LL, (kRowBlocks * (long long)s->arr.n + ntot / 2) / ntot);
            off[r + 1] = off[r] + (M * 32 + 255) / 256;
            off[(R + 1) + r + 1] = off[(R + 1) + r] + share;
            off[2 * (R + 1) + r + 1] = off[2 * (R + 1) + r] + std::min(2 * M, share);
        }
        if (cudaMalloc(&dReps, sizeof(MolRep) * R) != cudaSuccess ||
            cudaMalloc(&dMolOff, sizeof(int) * off.size()) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "batch: allocation failed");
        if (cudaMemcpyAsync(dReps, reps.data(), sizeof(MolRep) * R, cudaMemcpyHostToDevice, ctx->stream) !=
                cudaSuccess ||
            cudaMemcpyAsync(dMolOff, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, ctx->stream) !=
                cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "batch: upload failed");
        mb.reps = dReps;
        mb.R = R;
        mb.off_w = dMolOff;
        mb.off_rows = dMolOff + (R + 1);
        mb.off_in = dMolOff + 2 * (R + 1);
        mb.nblk_w = off[R];
        mb.nblk_rows = off[(R + 1) + R];
        mb.nblk_in = off[2 * (R + 1) + R];
        molb = true;
        int rc = ctx->sync_check("batch rebuild tables");
        if (rc) return rc;
        // kernels of the conditional fallback body: the same launches captured
        // once into a graph of their own and counted
        cudaGraph_t fb = nullptr;
        if (cudaStreamBeginCapture(side[0], cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "batch: fallback capture failed to start");
        cudaError_t ef = cudaSuccess;
        for (System* s : sys)
            if ((ef = s->enqueue_rebuild_fallback(side[0])) != cudaSuccess) break;
        const cudaError_t e2 = cudaStreamEndCapture(side[0], &fb);
        if (ef != cudaSuccess || e2 != cudaSuccess) {
            cudaGetLastError();
            return ctx->fail(FMD_ERR_CUDA, "batch: fallback capture failed");
        }
        body_kernels = count_kernel_nodes(fb, nullptr);
        cudaGraphDestroy(fb);
        return pending("after counting the fallback's kernels");
    }

    // The batched rebuild, inside a stream capture: one launch per phase for
    // all replicas, and between the path decision and the half rows a
    // conditional node whose body -- every replica's cell-grid fallback,
    // gated per replica on the device -- runs only when some replica's
    // molecule path was rejected for this build.
    cudaError_t enqueue_rebuild_batched(cudaStream_t st) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        cudaError_t e;
        where = "an error pending before the rebuild";
        if ((e = cudaPeekAtLastError()) != cudaSuccess) return e;
        where = "capture info";
        if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd)) != cudaSuccess) return e;
        if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureUnsupported;
        where = "conditional handle";
        cudaGraphConditionalHandle cond;
        if ((e = cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
        where = "batched partner tables";
        if ((e = mol_rebuild_batch_pre(mb, cond, st, &where)) != cudaSuccess) return e;
        where = "capture info";
        if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd)) != cudaSuccess) return e;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        where = "conditional node";
        if ((e = cudaGraphAddNode(&node, g, deps, nd, &cp)) != cudaSuccess) return e;
        where = "capture dependencies";
        if ((e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
            return e;
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        where = "fallback capture";
        if ((e = cudaStreamBeginCaptureToGraph(side[0], body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
            cudaSuccess)
            return e;
        cudaError_t ef = cudaSuccess;
        for (System* s : sys)
            if ((ef = s->enqueue_rebuild_fallback(side[0])) != cudaSuccess) break;
        cudaGraph_t got = nullptr;
        if ((e = cudaStreamEndCapture(side[0], &got)) != cudaSuccess) return e;
        if (ef != cudaSuccess) return ef;
        where = "batched rows";
        return mol_rebuild_batch_rows(mb, st);
    }
    const char* where = "";

    int set_offsets(const Tune& t) {
        std::vector<int> off(3 * (R + 1), 0);
        for (int r = 0; r < R; r++) {
            const StepArrays& a = sys[r]->arr;
            const long long terms = (long long)a.topo.nb + a.topo.nang + a.topo.ndih + a.topo.nimp;
            off[r + 1] = off[r] + blocks_for(a.n, kAtomThreads);
            off[(R + 1) + r + 1] = off[(R + 1) + r] + blocks_for(a.n, t.lj_apb);
            off[2 * (R + 1) + r + 1] = off[2 * (R + 1) + r] + blocks_for(std::max(terms, 1LL), t.f1_tpb);
        }
        if (cudaMemcpyAsync(dOff, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "batch: offset upload failed");
        bd.off_atom = dOff;
        bd.off_lj = dOff + (R + 1);
        bd.off_f1 = dOff + 2 * (R + 1);
        bd.nblk_atom = off[R];
        bd.nblk_lj = off[(R + 1) + R];
        bd.nblk_f1 = off[2 * (R + 1) + R];
        bd.lj_threads = t.lj_threads;
        bd.lj_unroll = t.lj_unroll;
        bd.lj_staged_in_cap = t.lj_staged ? sys[0]->arr.in_cap : 0;
        bd.f1_threads = t.f1_threads;
        return ctx->sync_check("batch offsets");
    }

    void drop_graphs() {
        for (auto& row : graphs)
            for (auto& g : row)
                if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    // Forces of the current state through each replica's own launches (after
    // tuning runs have consumed the accumulators).
    int refresh_forces() {
        cudaStream_t st = ctx->stream;
        for (System* s : sys) {
            if (cudaMemsetAsync(s->arr.Facc, 0, sizeof(double) * 3 * (size_t)s->arr.n, st) != cudaSuccess ||
                enqueue_forces(s->arr, st) != cudaSuccess || enqueue_force_reduce(s->arr, st) != cudaSuccess)
                return ctx->fail(FMD_ERR_CUDA, "batch: force refresh failed");
        }
        return ctx->sync_check("batch force refresh");
    }

    double time_ms(int reps, const std::function<cudaError_t()>& f) {
        cudaStream_t st = ctx->stream;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        f();
        cudaEventRecord(e0, st);
        for (int k = 0; k < reps; k++) f();
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return ms / reps;
    }

    int autotune() {
        const int dev = ctx->device;
        const auto key = std::make_tuple(dev, R, natoms);
        auto it = tune_cache().find(key);
        if (it != tune_cache().end()) {
            tune = it->second;
            return set_offsets(tune);
        }
        Tune best = tune;
        best.lj_ms = 1e30;
        cudaStream_t st = ctx->stream;
        // staged rows need one row stride (16-byte multiple) across replicas
        bool can_stage = sys[0]->arr.in_cap % 4 == 0;
        for (System* s : sys) can_stage = can_stage && s->arr.in_cap == sys[0]->arr.in_cap;
        for (int staged : {0, 1})
            for (int nt : {128, 256})
                for (int u : {2, 4})
                    for (int apb : {8, 16, 32, 64}) {
                        if (staged && !can_stage) continue;
                        Tune t = best;
                        t.lj_threads = nt; t.lj_unroll = u; t.lj_apb = apb; t.lj_staged = staged;
                        int rc = set_offsets(t);
                        if (rc) return rc;
                        const int icap = staged ? sys[0]->arr.in_cap : 0;
                        const double ms = time_ms(3, [&]() {
                            return batch_lj_launch(dA, bd.off_lj, R, bd.nblk_lj, bd.ff, bd.precision, nt, u, st, icap);
                        });
                        if (ms < best.lj_ms) { best = t; best.lj_ms = ms; }
                    }
        if (bd.kind == FMD_SYS_MM) {
            best.f1_ms = 1e30;
            Tune b2 = best;
            for (int nt : {128, 256})
                for (int tpb : {256, 512, 1024, 2048}) {
                    Tune t = b2;
                    t.f1_threads = nt; t.f1_tpb = tpb;
                    int rc = set_offsets(t);
                    if (rc) return rc;
                    const double ms = time_ms(3, [&]() {
                        return batch_mm_bonded_launch(dA, bd.off_f1, R, bd.nblk_f1, nt, st);
                    });
                    if (ms < best.f1_ms) { best.f1_threads = nt; best.f1_tpb = tpb; best.f1_ms = ms; }
                }
        }
        int rc = ctx->sync_check("batch autotune");
        if (rc) return rc;
        tune = best;
        tune_cache()[key] = best;
        if ((rc = set_offsets(tune))) return rc;
        return refresh_forces();
    }

    cudaError_t enqueue_variant(bool rebuild, bool phase, cudaStream_t st) {
        cudaError_t e;
        if (rebuild && molb) {
            if ((e = enqueue_rebuild_batched(st)) != cudaSuccess) return e;
        } else if (rebuild) {
            // per-replica rebuilds as parallel branches
            if ((e = cudaEventRecord(ev_fork, st)) != cudaSuccess) return e;
            for (int k = 0; k < kSideStreams; k++)
                if ((e = cudaStreamWaitEvent(side[k], ev_fork, 0)) != cudaSuccess) return e;
            for (int r = 0; r < R; r++)
                if ((e = sys[r]->enqueue_rebuild(side[r % kSideStreams])) != cudaSuccess) return e;
            for (int k = 0; k < kSideStreams; k++) {
                if ((e = cudaEventRecord(ev_join[k], side[k])) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(st, ev_join[k], 0)) != cudaSuccess) return e;
            }
        }
        return enqueue_batch_step(bd, phase, st);
    }

    int capture(bool rebuild, bool phase) {
        cudaGraphExec_t& ge = graphs[rebuild ? 1 : 0][phase ? 1 : 0];
        if (ge) return FMD_OK;
        cudaStream_t st = ctx->stream;
        cudaGraph_t graph;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return ctx->fail(FMD_ERR_CUDA, "batch: graph capture failed to start");
        cudaError_t e = enqueue_variant(rebuild, phase, st);
        cudaError_t e2 = cudaStreamEndCapture(st, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            cudaGetLastError();
            if (e2 == cudaSuccess && graph) cudaGraphDestroy(graph);
            return ctx->fail(FMD_ERR_CUDA, std::string("batch: graph capture failed: ") + where + ": " +
                                               cudaGetErrorName(e != cudaSuccess ? e : e2) + " (" +
                                               cudaGetErrorString(e != cudaSuccess ? e : e2) + ")");
        }
        if (int rc = pending("after the capture")) return rc;
        count_kernels(graph, rebuild, nkern[rebuild ? 1 : 0][phase ? 1 : 0], nkern_cond[rebuild ? 1 : 0][phase ? 1 : 0]);
        if (int rc = pending("after counting the graph's kernels")) return rc;
        e = cudaGraphInstantiate(&ge, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, cudaGetErrorString(e));
        if (int rc = pending("after instantiation")) return rc;
        // upload now, so the first launch of this variant does no set-up work
        if ((e = cudaGraphUpload(ge, st)) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, cudaGetErrorString(e));
        if (int rc = pending("after the upload")) return rc;
        return FMD_OK;
    }

    // Kernel nodes of a captured step graph: launched every replay (top
    // level), and inside conditional bodies (launched only when the body runs).
    int nkern[2][2] = {}, nkern_cond[2][2] = {};
    int body_kernels = 0;               // kernel nodes of the conditional fallback body
    std::string count_note;             // a graph query that failed while counting (diagnostic)
    int count_kernel_nodes(cudaGraph_t g, int* conditionals) {
        size_t n = 0;
        cudaError_t e;
        if ((e = cudaGraphGetNodes(g, nullptr, &n)) != cudaSuccess) {
            count_note = std::string("cudaGraphGetNodes(count): ") + cudaGetErrorName(e);
            cudaGetLastError();
            return 0;
        }
        std::vector<cudaGraphNode_t> nodes(n);
        if (n && (e = cudaGraphGetNodes(g, nodes.data(), &n)) != cudaSuccess) {
            count_note = std::string("cudaGraphGetNodes: ") + cudaGetErrorName(e);
            cudaGetLastError();
            return 0;
        }
        int k = 0, c = 0;
        for (size_t q = 0; q < n; q++) {
            cudaGraphNodeType t = cudaGraphNodeTypeEmpty;
            if ((e = cudaGraphNodeGetType(nodes[q], &t)) != cudaSuccess) {
                count_note = std::string("cudaGraphNodeGetType: ") + cudaGetErrorName(e);
                cudaGetLastError();
                continue;
            }
            k += t == cudaGraphNodeTypeKernel;
            c += t == cudaGraphNodeTypeConditional;
        }
        if (conditionals) *conditionals = c;
        return k;
    }
    // (A conditional node's type query fails on this runtime, so the rebuild
    // variant's one conditional body is counted from the fallback's own
    // capture at set-up.)
    void count_kernels(cudaGraph_t g, bool rebuild, int& top, int& cond) {
        top = count_kernel_nodes(g, nullptr);
        cond = rebuild && molb ? body_kernels : 0;
    }

    // Fails when a CUDA error is pending (left by an earlier runtime call).
    int pending(const char* stage) {
        const cudaError_t e = cudaPeekAtLastError();
        if (e == cudaSuccess) return FMD_OK;
        cudaGetLastError();
        return ctx->fail(FMD_ERR_CUDA, std::string("batch: ") + cudaGetErrorName(e) + " pending " + stage +
                                           (count_note.empty() ? std::string() : " [" + count_note + "]"));
    }

    // All four step variants, captured and uploaded at creation (as a system
    // does in its init), so no host-side capture sits between two steps.
    int capture_all() {
        for (int r = 0; r < 2; r++)
            for (int ph = 0; ph < 2; ph++) {
                const int rc = capture(r != 0, ph != 0);
                if (rc != FMD_OK) return rc;
            }
        return ctx->sync_check("batch graph capture");
    }

    int enqueue(int first, int last) {
        if (last < first) return FMD_OK;
        cudaStream_t st = ctx->stream;
        const int g0 = first - 1;
        for (System* s : sys)
            if (cudaMemcpyAsync(&s->arr.S->gstep, &g0, sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess)
                return ctx->fail(FMD_ERR_CUDA, "batch: step counter upload failed");
        const fmd_run_params& p = sys[0]->p;
        for (int g = first; g <= last; g++) {
            const int r = (g % p.nlup) == 0, ph = g <= p.coldstart + p.warmup;
            int rc = capture(r != 0, ph != 0);
            if (rc != FMD_OK) return rc;
            if (cudaGraphLaunch(graphs[r][ph], st) != cudaSuccess) return ctx->fail(FMD_ERR_CUDA, "batch: graph launch failed");
        }
        return FMD_OK;
    }

    void release() {
        drop_graphs();
        for (auto& s : side)
            if (s) { cudaStreamDestroy(s); s = nullptr; }
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (auto& e : ev_join)
            if (e) cudaEventDestroy(e);
        cudaFree(dA); cudaFree(dP); cudaFree(dOff); cudaFree(dReps); cudaFree(dMolOff);
        dA = nullptr; dP = nullptr; dOff = nullptr; dReps = nullptr; dMolOff = nullptr;
    }
};

extern "C" int fmd_batch_create(fmd_ctx* ctx, int R, fmd_system* const* systems, int autotune, fmd_batch** out) {
    if (!ctx || !systems || !out || R < 1) return ctx ? ctx->fail(FMD_ERR_ARG, "fmd_batch_create: bad argument") : FMD_ERR_ARG;
    *out = nullptr;
    auto* b = new fmd_batch();
    b->ctx = ctx;
    b->R = R;
    for (int r = 0; r < R; r++) {
        if (!systems[r] || !systems[r]->sys) { delete b; return ctx->fail(FMD_ERR_ARG, "fmd_batch_create: null system"); }
        System* s = systems[r]->sys.get();
        const fmd_run_params& p0 = systems[0]->sys->p;
        if (s->ctx != ctx || s->arr.kind != FMD_SYS_MM || s->arr.has_charge || s->arr.sg != nullptr ||
            s->p.nlup != p0.nlup || s->p.coldstart != p0.coldstart || s->p.warmup != p0.warmup ||
            s->arr.precision != systems[0]->sys->arr.precision) {
            delete b;
            return ctx->fail(FMD_ERR_ARG, "fmd_batch_create: replicas must be MM systems of this context without "
                                          "charges, with one list cadence, schedule and precision");
        }
        for (int q = 0; q < r; q++)
            if (systems[q] == systems[r]) { delete b; return ctx->fail(FMD_ERR_ARG, "fmd_batch_create: a system appears twice"); }
        b->sys.push_back(s);
        b->natoms += s->arr.n;
    }
    for (System* s : b->sys)
        if (!s->initialized) {
            const int rc = s->init();
            if (rc) { delete b; return rc; }
        }
    std::vector<StepArrays> A(R);
    std::vector<StepParams> P(R);
    for (int r = 0; r < R; r++) { A[r] = b->sys[r]->arr; P[r] = b->sys[r]->sp; }
    cudaStream_t st = ctx->stream;
    if (cudaMalloc(&b->dA, sizeof(StepArrays) * R) != cudaSuccess ||
        cudaMalloc(&b->dP, sizeof(StepParams) * R) != cudaSuccess ||
        cudaMalloc(&b->dOff, sizeof(int) * 3 * (R + 1)) != cudaSuccess) {
        b->release();
        delete b;
        return ctx->fail(FMD_ERR_CUDA, "fmd_batch_create: allocation failed");
    }
    cudaMemcpyAsync(b->dA, A.data(), sizeof(StepArrays) * R, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->dP, P.data(), sizeof(StepParams) * R, cudaMemcpyHostToDevice, st);
    for (auto& s : b->side)
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
            b->release();
            delete b;
            return ctx->fail(FMD_ERR_CUDA, "fmd_batch_create: stream creation failed");
        }
    cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    for (auto& e : b->ev_join) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    b->bd.R = R;
    b->bd.A = b->dA;
    b->bd.P = b->dP;
    b->bd.kind = FMD_SYS_MM;
    b->bd.ff = FMD_FF_MM;
    b->bd.precision = b->sys[0]->arr.precision;
    int rc = b->pending("before the batch set-up");
    if (!rc) rc = autotune ? b->autotune() : b->set_offsets(b->tune);
    if (!rc) rc = b->pending("after the launch-shape set-up");
    if (!rc) rc = b->setup_mol_batch();
    if (!rc) rc = b->pending("after the rebuild tables");
    if (!rc) rc = b->capture_all();
    if (rc) { b->release(); delete b; return rc; }
    *out = b;
    return FMD_OK;
}

extern "C" int fmd_batch_enqueue(fmd_batch* b, int first, int last) {
    if (!b) return FMD_ERR_ARG;
    return b->enqueue(first, last);
}

extern "C" int fmd_batch_run(fmd_batch* b, int first, int last) {
    if (!b) return FMD_ERR_ARG;
    const int rc = b->enqueue(first, last);
    if (rc) return rc;
    return b->ctx->sync_check("fmd_batch_run");
}

extern "C" int fmd_batch_observables(fmd_batch* b, fmd_obs* obs) {
    if (!b || !obs) return FMD_ERR_ARG;
    for (int r = 0; r < b->R; r++)
        if (cudaMemcpyAsync(obs + r, &b->sys[r]->arr.S->obs, sizeof(fmd_obs), cudaMemcpyDeviceToHost,
                            b->ctx->stream) != cudaSuccess)
            return b->ctx->fail(FMD_ERR_CUDA, "fmd_batch_observables: copy failed");
    return b->ctx->sync_check("fmd_batch_observables");
}

extern "C" int fmd_batch_get_tuning(fmd_batch* b, fmd_batch_tuning* t) {
    if (!b || !t) return FMD_ERR_ARG;
    t->lj_threads = b->tune.lj_threads;
    t->lj_unroll = b->tune.lj_unroll;
    t->lj_atoms_per_block = b->tune.lj_apb;
    t->lj_staged = b->tune.lj_staged;
    t->bonded_threads = b->tune.f1_threads;
    t->bonded_terms_per_block = b->tune.f1_tpb;
    t->lj_ms = b->tune.lj_ms;
    t->bonded_ms = b->tune.f1_ms;
    t->blocks_lj = b->bd.nblk_lj;
    t->blocks_bonded = b->bd.nblk_f1;
    t->blocks_atom = b->bd.nblk_atom;
    return FMD_OK;
}

extern "C" int fmd_batch_step_kernels(fmd_batch* b, int rebuild, int phase, int* nk) {
    if (!b || !nk) return FMD_ERR_ARG;
    *nk = b->nkern[rebuild ? 1 : 0][phase ? 1 : 0];
    return FMD_OK;
}

extern "C" int fmd_batch_step_kernels_conditional(fmd_batch* b, int rebuild, int phase, int* nk) {
    if (!b || !nk) return FMD_ERR_ARG;
    *nk = b->nkern_cond[rebuild ? 1 : 0][phase ? 1 : 0];
    return FMD_OK;
}

extern "C" int fmd_batch_destroy(fmd_batch* b) {
    if (!b) return FMD_OK;
    cudaStreamSynchronize(b->ctx->stream);
    b->release();
    delete b;
    return FMD_OK;
}
