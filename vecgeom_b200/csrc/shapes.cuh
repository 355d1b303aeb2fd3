// shapes.cuh -- every shape's parameter record and device arithmetic.
#pragma once
#include <type_traits>

#include "../../include/vgb.h"
#include "box.cuh"
#include "tube.cuh"
#include "cone.cuh"
#include "sphere.cuh"
#include "trd.cuh"
#include "torus.cuh"
#include "polycone.cuh"
#include "polyhedron.cuh"
#include "orb.cuh"
#include "parallelepiped.cuh"
#include "paraboloid.cuh"
#include "trapezoid.cuh"

struct vgb_geometry;

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

// Shapes whose reference DistanceToIn moves the direction with the point
// transform (TorusImplementation.h:906) declare kDirectionAsPoint.
template <class Ops, class = void> struct DirAsPoint : std::false_type {};
template <class Ops>
struct DirAsPoint<Ops, std::void_t<decltype(Ops::kDirectionAsPoint)>>
    : std::integral_constant<bool, Ops::kDirectionAsPoint> {};

template <class Ops, class R>
VGB_HD V3<R> dti_dir(const DXform &X, const V3<R> &d) {
  if constexpr (DirAsPoint<Ops>::value)
    return xf_point(X, d);
  else
    return xf_dir(X, d);
}

}  // namespace vgb

#include "boolean.cuh"

namespace vgb {
VGB_HD BooleanP bind_params(BooleanP p, const double *rec) {
  p.base = rec;
  return p;
}

// Called by vgb_geometry_close() once the device parameter pool is allocated.
vgb_status finalize_shapes(vgb_geometry *g);
}  // namespace vgb

// (type, ops template, parameter record) of every shape with batch kernels
#define VGB_FOR_EACH_SHAPE(X)                                 \
  VGB_FOR_EACH_PRIMITIVE(X)                                   \
  X(VGB_SHAPE_BOOLEAN, vgb::BoolOps, vgb::BooleanP)
