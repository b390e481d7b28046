// rm_device.h -- device generation from a .rm descriptor (CUDA translation units only).
#pragma once

#include <cuda_runtime.h>

#include "rm.h"

// the C ABI's opaque descriptor handle
struct dsgdpp_rm {
  dsgdpp::RmDesc d;
};

namespace dsgdpp {

// Worig (size1 x rank) and Horig (size2 x rank), both row-major FP64, into
// device memory.
void rm_factors_device(const RmDesc& d, double* W, double* H, cudaStream_t st);

// The data (which = 0) or test (which = 1) matrix into device arrays of
// rm_count(d, which) entries: chunk by chunk in row-major chunk order, each
// chunk's cells in generator order.  Returns the count.
uint64_t rm_data_device(const RmDesc& d, int which, uint32_t* rows, uint32_t* cols, double* vals,
                        cudaStream_t st);

uint64_t rm_count(const RmDesc& d, int which);

}  // namespace dsgdpp
