// parallelepiped.cuh -- Parallelepiped arithmetic (device), templated on the
// arithmetic type; follows volumes/kernel/ParallelepipedImplementation.h as the
// reference Scalar backend runs it: the point is sheared into the frame of an
// axis-aligned box and the box kernels answer, except DistanceToOut, which has
// its own face walk.
#pragma once
#include "box.cuh"

namespace vgb {

// UnplacedParallelepiped (volumes/UnplacedParallelepiped.h:20-26,
// source/UnplacedParallelepiped.cpp:40-65) with the two factors the safeties
// compute per point, constant per shape.
struct ParaP {
  BoxP dims;  // fDimensions (half lengths)
  double tanAlpha, tanThetaSinPhi, tanThetaCosPhi;
  double ctx;  // 1 / sqrt(1 + tanAlpha^2 + tanThetaCosPhi^2)
  double cty;  // 1 / sqrt(1 + tanThetaSinPhi^2)
};

template <class R> struct ParaOps {
  using B = BoxOps<R>;

  // Transform (ParallelepipedImplementation.h:96-104)
  static VGB_HD V3<R> shear(const ParaP &a, V3<R> p) {
    p.y = p.y - (R)a.tanThetaSinPhi * p.z;
    p.x = p.x - ((R)a.tanThetaCosPhi * p.z + (R)a.tanAlpha * p.y);
    return p;
  }
  static VGB_HD bool contains(const ParaP &a, const V3<R> &p) {
    return B::contains(a.dims, shear(a, p));
  }
  static VGB_HD int inside(const ParaP &a, const V3<R> &p) { return B::inside(a.dims, shear(a, p)); }
  static VGB_HD R distance_to_in(const ParaP &a, const V3<R> &p, const V3<R> &v, R step_max) {
    return B::distance_to_in(a.dims, shear(a, p), shear(a, v), step_max);
  }

  // DistanceToOut (:165-250): the z faces, then the y faces along the sheared
  // y, then the x faces along the sheared x; a face the point is beyond while
  // moving out of it ends the walk with 0
  static VGB_HD R distance_to_out(const ParaP &a, const V3<R> &p, const V3<R> &v, R) {
    const R hz = (R)a.dims.d[2], hy = (R)a.dims.d[1], hx = (R)a.dims.d[0];
    const R ht = (R)kHalfTolerance;
    R distance = Lim<R>::inf();
    // +z
    bool inDir = v.z > 0;
    R max = hz - p.z;
    bool inPoint = max > ht;
    if (inDir && !inPoint) return (R)0;
    if (inPoint && inDir) distance = max / v.z;
    // -z
    inDir = v.z < 0;
    max = -hz - p.z;
    inPoint = max < -ht;
    if (inDir && !inPoint) return (R)0;
    if (inPoint && inDir) distance = max / v.z;
    // +y, -y
    const R py = p.y - (R)a.tanThetaSinPhi * p.z;
    const R vy = v.y - (R)a.tanThetaSinPhi * v.z;
    inDir = vy > 0;
    max = hy - py;
    inPoint = max > ht;
    max = max / vy;
    if (inDir && !inPoint) return (R)0;
    if (inPoint && inDir && max < distance) distance = max;
    inDir = vy < 0;
    max = -hy - py;
    inPoint = max < -ht;
    max = max / vy;
    if (inDir && !inPoint) return (R)0;
    if (inPoint && inDir && max < distance) distance = max;
    // +x, -x
    const R px = p.x - (R)a.tanThetaCosPhi * p.z - (R)a.tanAlpha * py;
    const R vx = v.x - (R)a.tanThetaCosPhi * v.z - (R)a.tanAlpha * vy;
    inDir = vx > 0;
    max = hx - px;
    inPoint = max > ht;
    max = max / vx;
    if (inDir && !inPoint) return (R)0;
    if (inPoint && inDir && max < distance) distance = max;
    inDir = vx < 0;
    max = -hx - px;
    inPoint = max < -ht;
    max = max / vx;
    if (inDir && !inPoint) return (R)0;
    if (inPoint && inDir && max < distance) distance = max;
    return distance;
  }

  // SafetyToIn / SafetyToOut (:255-300)
  static VGB_HD R safety_to_in(const ParaP &a, const V3<R> &p) {
    const V3<R> l = shear(a, p);
    const R s0 = (fabs(l.x) - (R)a.dims.d[0]) * (R)a.ctx;
    const R s1 = (fabs(l.y) - (R)a.dims.d[1]) * (R)a.cty;
    const R s2 = fabs(l.z) - (R)a.dims.d[2];
    R s = s0;
    if (s1 > s) s = s1;
    if (s2 > s) s = s2;
    return s;
  }
  static VGB_HD R safety_to_out(const ParaP &a, const V3<R> &p) {
    const V3<R> l = shear(a, p);
    const R s0 = ((R)a.dims.d[0] - fabs(l.x)) * (R)a.ctx;
    const R s1 = ((R)a.dims.d[1] - fabs(l.y)) * (R)a.cty;
    const R s2 = (R)a.dims.d[2] - fabs(l.z);
    R s = s0;
    if (s1 < s) s = s1;
    if (s2 < s) s = s2;
    return s;
  }
};

}  // namespace vgb
