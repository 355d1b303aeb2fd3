// shapes.cuh -- every shape's parameter record and device arithmetic.
#pragma once
#include "../../include/vgb.h"
#include "box.cuh"
#include "tube.cuh"
#include "cone.cuh"
#include "sphere.cuh"
#include "trd.cuh"
#include "torus.cuh"
#include "polycone.cuh"
#include "polyhedron.cuh"

struct vgb_geometry;

// (type, ops template, parameter record) of every shape with batch kernels
#define VGB_FOR_EACH_SHAPE(X)                                 \
  X(VGB_SHAPE_BOX, vgb::BoxOps, vgb::BoxP)                    \
  X(VGB_SHAPE_TUBE, vgb::TubeOps, vgb::TubeP)                 \
  X(VGB_SHAPE_CONE, vgb::ConeOps, vgb::ConeP)                 \
  X(VGB_SHAPE_SPHERE, vgb::SphereOps, vgb::SphereP)           \
  X(VGB_SHAPE_TRD, vgb::TrdOps, vgb::TrdP)                    \
  X(VGB_SHAPE_TORUS, vgb::TorusOps, vgb::TorusP)              \
  X(VGB_SHAPE_POLYCONE, vgb::PolyconeOps, vgb::PolyconeP)    \
  X(VGB_SHAPE_POLYHEDRON, vgb::PolyhedronOps, vgb::PolyhedronP)

namespace vgb {

// Records with variable-length tables (polycone sections, ...) reach them
// through the record's own address, bound when a kernel is launched: the
// device copy of the parameter pool, or the host copy for host-side callers.
template <class P> VGB_HD P bind_params(P p, const double *) { return p; }
VGB_HD PolyconeP bind_params(PolyconeP p, const double *rec) {
  p.base = rec;
  return p;
}
VGB_HD PolyhedronP bind_params(PolyhedronP p, const double *rec) {
  p.base = rec;
  return p;
}

// Called by vgb_geometry_close() once the device parameter pool is allocated.
vgb_status finalize_shapes(vgb_geometry *g);
}  // namespace vgb
