// fmd_internal.h -- shared declarations of the B200 library (device state,
// launch helpers, error plumbing).  Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/fullermd.h"

namespace fmd {

constexpr int kSMs = 148;            // B200: 2 dies x 74 SMs
constexpr int kNptDoubles = 15;      // {xi,Q,Vg[9],W,Pe,Tt,Nf}

// ---- error handling ------------------------------------------------------
struct Status {
    int code = FMD_OK;
    std::string msg;
};

#define FMD_CUDA_TRY(ctx, expr)                                                   \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess) return (ctx)->fail(FMD_ERR_CUDA,                   \
            std::string(#expr) + ": " + cudaGetErrorString(_e));                  \
    } while (0)

// ---- growable device buffer ------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// ---- device-side error word --------------------------------------------------
// Kernels never trap; they record the first problem here and the host turns
// it into a status code after the next synchronisation point.
struct DevErr {
    int code;      // FMD_OK or FMD_ERR_*
    int where;     // kernel id
    int index;     // offending particle / entry
    int value;     // offending count
};

enum KernelId {
    K_NLIST = 1, K_TRANSPOSE = 2, K_REBO = 3, K_LJ = 4, K_RIGID = 5, K_MM = 6, K_INTEGRATE = 7,
    K_CELLS = 8, K_REBO2 = 9,
};

}  // namespace fmd

// The context: one device, one stream, a pool of scratch buffers.
struct fmd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int last_code = FMD_OK;
    std::string last_msg;
    fmd::DevErr* d_err = nullptr;   // device error word
    fmd::DevErr* h_err = nullptr;   // pinned mirror
    // named scratch buffers, grown on demand (never inside a captured graph)
    std::vector<fmd::DevBuf> scratch;
    // pinned staging for scalars
    double* h_scalars = nullptr;
    // pair arithmetic of the atomistic LJ terms in host-pointer calls (fmd_precision)
    int precision = FMD_PREC_FP64;
    // Device blocks released by systems of this context, by size: the next
    // system of the same size takes them instead of mapping fresh memory
    // (cudaMalloc of a few hundred MB costs milliseconds and varies with the
    // process's allocation history).  Freed with the context.
    std::multimap<size_t, void*> mem_cache;
    cudaError_t dev_alloc(void** p, size_t bytes) {
        auto it = mem_cache.find(bytes);
        if (it != mem_cache.end()) {
            *p = it->second;
            mem_cache.erase(it);
            return cudaSuccess;
        }
        return cudaMalloc(p, bytes);
    }
    // The caller has synchronised every stream that used the block.
    void dev_release(void* p, size_t bytes) {
        if (p) mem_cache.emplace(bytes, p);
    }

    int fail(int code, const std::string& m) {
        last_code = code;
        last_msg = m;
        return code;
    }
    int ok() { return FMD_OK; }
    // Ensures scratch slot `slot` holds at least `bytes`.
    int need(int slot, size_t bytes, void** out);
    // Synchronises the stream and converts a recorded device error into a status.
    int sync_check(const char* what);
};
