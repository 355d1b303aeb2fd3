// shapes.cuh -- every shape's parameter record and device arithmetic.
#pragma once
#include "../../include/vgb.h"
#include "box.cuh"

struct vgb_geometry;

namespace vgb {
// Called by vgb_geometry_close() once the device parameter pool is allocated:
// shape records that point into the pool (section tables etc.) store device
// addresses here before the pool is copied.
vgb_status finalize_shapes(vgb_geometry *g);
}  // namespace vgb
