// noalloc.cu -- a REBO force entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc: host programs that hand all device
// memory to a pool or allocator of their own and forbid side allocations,
// and embedded or real-time drivers that must not touch the allocator after
// start-up.  The regular entry points allocate device scratch through an
// fmd_ctx (and creating a context allocates too), so they are unusable there.
//
// This variant takes device pointers from the caller for every input and
// output, and keeps its only scratch -- the cell matrix and one partial
// {energy, virial} record per thread block -- in the file-scope array below.
// The array is a fixed size, reserved on every GPU that loads this library,
// for as long as the process lives.  The cell matrix reaches the GPU as a
// kernel argument (by value), so the call issues no host-to-device copy.
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>
#include "kernels.h"
#include "geom.cuh"

namespace fmd {
namespace {

// k_rebo runs 128 threads per block with four threads per atom and a
// grid-stride loop, so any number of atoms is covered by a capped grid.
constexpr int kNoAllocThreads = 128;
constexpr int kNoAllocLanes = 4;
constexpr int kNoAllocMaxBlocks = 1024;         // partial records the array holds
// Largest na accepted: the 122,880-atom nc=8 crystal fits, and at most four
// grid-stride passes of the capped grid are needed.
constexpr int kNoAllocMaxAtoms = 131072;
constexpr int kScratchDoubles = 18 + kNoAllocMaxBlocks * kNV;           // {h, hi} + partials

// 82 KB per GPU.  Shared by every call in the process; see the header for
// the consequences.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch per device, looked up once per device.
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// h then h^-1, passed by value: kernel arguments are copied when the launch
// is enqueued, so the caller's arrays may change as soon as the call returns.
struct CellArg {
    double v[18];
};

__global__ void k_noalloc_cell(CellArg c, double* __restrict__ hh) {
    if (threadIdx.x < 18) hh[threadIdx.x] = c.v[threadIdx.x];
}

// Sums the nblk partial records and adds them into the caller's virial;
// writes the energy.  Every record it reads was written by this call's REBO
// launch, so nothing in the array needs to start at zero.
__global__ void k_noalloc_reduce(const double* __restrict__ part, int nblk, double* __restrict__ vir9,
                                 double* __restrict__ E) {
    __shared__ double sm[32 * kNV];
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < kNV; k++) acc[k] += part[(size_t)b * kNV + k];
    double tot[kNV];
    block_sum_store<kNV>(acc, sm, tot);
    if (threadIdx.x == 0) {
        *E = tot[0];
        for (int q = 0; q < 9; q++) vir9[q] += tot[1 + q];
    }
}

// Puts the caller's current device back on every return path.
struct DeviceRestore {
    int dev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    }
    ~DeviceRestore() {
        if (dev >= 0) cudaSetDevice(dev);
    }
};

}  // namespace
}  // namespace fmd

extern "C" int fmd_rebo_forces_noalloc(const double* d_pos, const double* h, const double* hi, const int* d_nlc,
                                       const int* d_nll, int max_neigh, int na, double* d_F, double* d_vir9,
                                       double* d_E, void* stream) {
    using namespace fmd;
    if (!d_pos || !h || !hi || !d_nlc || !d_nll || !d_F || !d_vir9 || !d_E || max_neigh < 1 || na < 1)
        return FMD_ERR_ARG;
    if (na > kNoAllocMaxAtoms) return FMD_ERR_CAPACITY;
    DeviceRestore keep;
    // The positions decide the device; the scratch address is per device.
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, d_pos) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return FMD_ERR_ARG;
    }
    const int dev = attr.device;
    if (dev < 0 || dev >= kMaxDevices) return FMD_ERR_ARG;
    if (dev != keep.dev && cudaSetDevice(dev) != cudaSuccess) return FMD_ERR_CUDA;
    double* scratch;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            // In host code the array's name is only a host-side stand-in; the
            // device address must be looked up with that device current.
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return FMD_ERR_CUDA;
            g_scratch_addr[dev] = (double*)p;
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    CellArg cell;
    for (int k = 0; k < 9; k++) { cell.v[k] = h[k]; cell.v[9 + k] = hi[k]; }
    k_noalloc_cell<<<1, 32, 0, st>>>(cell, scratch);
    if (cudaGetLastError() != cudaSuccess) return FMD_ERR_CUDA;
    const long long threads = (long long)na * kNoAllocLanes;
    const int nblk = (int)std::min<long long>((threads + kNoAllocThreads - 1) / kNoAllocThreads, kNoAllocMaxBlocks);
    double* part = scratch + 18;
    if (rebo_launch_grid(d_pos, scratch, d_nlc, d_nll, max_neigh, na, d_F, part, nblk, st) != cudaSuccess)
        return FMD_ERR_CUDA;
    k_noalloc_reduce<<<1, 256, 0, st>>>(part, nblk, d_vir9, d_E);
    return cudaGetLastError() == cudaSuccess ? FMD_OK : FMD_ERR_CUDA;
}
