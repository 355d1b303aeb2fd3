// dispatch.h -- launchers shared between the C-ABI layer and the kernel files.
#pragma once
#include <cuda_runtime.h>

#include "batch.cuh"

namespace vgb {
// precision: VGB_PREC_FP64 or VGB_PREC_FP32_REFINE; for single-volume batches
// both run the FP64 kernels (a float screen in front of them was measured to
// cost more than it saves here: only ~20% of the mixed rays are certified
// misses).  The navigator uses the float screen on its daughter loops.
vgb_status launch_batch_f64(const vgb_geometry *g, int32_t placed, int op, const BatchIO &io,
                            cudaStream_t s, int precision = VGB_PREC_FP64);
vgb_status launch_fused_f64(const vgb_geometry *g, int32_t placed, const FusedIO &io,
                            cudaStream_t s);
}  // namespace vgb
