// sg_host.h -- internal hooks between the learned-potential C-ABI and the
// device-resident systems.  Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>

#include "fmd_internal.h"

struct fmd_sg_data;
struct fmd_sg;

namespace fmd {

// Adds a snapshot whose positions, {h, hi} and REBO list are device arrays;
// its reference REBO energy, forces and virial come from the plain kernel.
int sg_data_add_device(fmd_sg_data* d, const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                       int na, cudaStream_t st);

}  // namespace fmd
