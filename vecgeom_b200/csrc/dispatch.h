// dispatch.h -- launchers shared between the C-ABI layer and the kernel files.
#pragma once
#include <cuda_runtime.h>

#include "batch.cuh"

namespace vgb {
vgb_status launch_batch_f64(const vgb_geometry *g, int32_t placed, int op, const BatchIO &io,
                            cudaStream_t s);
vgb_status launch_fused_f64(const vgb_geometry *g, int32_t placed, const FusedIO &io,
                            cudaStream_t s);
}  // namespace vgb
