// shapes.cuh -- every shape's parameter record and device arithmetic.
#pragma once
#include "../../include/vgb.h"
#include "box.cuh"
#include "tube.cuh"
#include "cone.cuh"
#include "sphere.cuh"
#include "trd.cuh"
#include "torus.cuh"

struct vgb_geometry;

// (type, ops template, parameter record) of every shape with batch kernels
#define VGB_FOR_EACH_SHAPE(X)            \
  X(VGB_SHAPE_BOX, vgb::BoxOps, vgb::BoxP) \
  X(VGB_SHAPE_TUBE, vgb::TubeOps, vgb::TubeP) \
  X(VGB_SHAPE_CONE, vgb::ConeOps, vgb::ConeP) \
  X(VGB_SHAPE_SPHERE, vgb::SphereOps, vgb::SphereP) \
  X(VGB_SHAPE_TRD, vgb::TrdOps, vgb::TrdP) \
  X(VGB_SHAPE_TORUS, vgb::TorusOps, vgb::TorusP)

namespace vgb {
// Called by vgb_geometry_close() once the device parameter pool is allocated:
// shape records that point into the pool (section tables etc.) store device
// addresses here before the pool is copied.
vgb_status finalize_shapes(vgb_geometry *g);
}  // namespace vgb
