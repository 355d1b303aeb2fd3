// box.cuh -- Box shape arithmetic (device), templated on the arithmetic type.
//
// Follows volumes/kernel/BoxImplementation.h operation by operation so the FP64
// instantiation (compiled with -fmad=false) rounds like the reference Scalar
// backend.  Branches are folded into selects: every point of a warp runs the
// same instruction stream, which suits the one-point-per-thread batch kernels.
#pragma once
#include "vgb_core.cuh"

namespace vgb {

// UnplacedBox: the three half-lengths (volumes/UnplacedBox.h:20-31).
struct BoxP {
  double d[3];
};

template <class R> struct BoxOps {
  // :607-666 GenericKernelForContainsAndInside<ForInside=false>
  static VGB_HD bool contains(const BoxP &b, const V3<R> &p) {
    bool out = fabs(p.x) > (R)b.d[0];
    out |= fabs(p.y) > (R)b.d[1];
    out |= fabs(p.z) > (R)b.d[2];
    return !out;
  }

  // :607-666 with ForInside=true, :653-666 InsideKernel
  static VGB_HD int inside(const BoxP &b, const V3<R> &p) {
    const R ht = (R)kHalfTolerance;
    const R ax = fabs(p.x), ay = fabs(p.y), az = fabs(p.z);
    bool out = ax > (R)b.d[0] + ht;
    bool in = ax < (R)b.d[0] - ht;
    out |= ay > (R)b.d[1] + ht;
    in &= ay < (R)b.d[1] - ht;
    out |= az > (R)b.d[2] + ht;
    in &= az < (R)b.d[2] - ht;
    return in ? kInside : (out ? kOutside : kSurface);
  }

  // :668-746 DistanceToInKernel.  Returns kInfinity on a miss (the value the
  // reference's caller starts `distance` at, volumes/ShapeImplementationHelper.h:199-220).
  static VGB_HD R distance_to_in(const BoxP &b, const V3<R> &p, const V3<R> &v, R step_max) {
    const R s0 = fabs(p.x) - (R)b.d[0];
    const R s1 = fabs(p.y) - (R)b.d[1];
    const R s2 = fabs(p.z) - (R)b.d[2];
    const R mtol = (R)0. - (R)kHalfTolerance;
    const R kmin = Lim<R>::minimum();
    if (s0 >= step_max || s1 >= step_max || s2 >= step_max) return Lim<R>::inf();
    if (s0 < 0 && s1 < 0 && s2 < 0) return (R)-1.;
    R next = s0 / fabs(v.x + kmin);
    R c1 = p.y + next * v.y;
    R c2 = p.z + next * v.z;
    if (s0 >= mtol && p.x * v.x < 0 && fabs(c1) <= (R)b.d[1] && fabs(c2) <= (R)b.d[2]) return next;
    next = s1 / fabs(v.y + kmin);
    c1 = p.x + next * v.x;
    c2 = p.z + next * v.z;
    if (s1 >= mtol && p.y * v.y < 0 && fabs(c1) <= (R)b.d[0] && fabs(c2) <= (R)b.d[2]) return next;
    next = s2 / fabs(v.z + kmin);
    c1 = p.x + next * v.x;
    c2 = p.y + next * v.y;
    if (s2 >= mtol && p.z * v.z < 0 && fabs(c1) <= (R)b.d[0] && fabs(c2) <= (R)b.d[1]) return next;
    return Lim<R>::inf();
  }

  // :748-799 DistanceToOutKernel
  static VGB_HD R distance_to_out(const BoxP &b, const V3<R> &p, const V3<R> &v, R) {
    const R kmin = Lim<R>::minimum();
    const R i0 = (R)1. / (v.x + kmin), i1 = (R)1. / (v.y + kmin), i2 = (R)1. / (v.z + kmin);
    const R d0 = ((v.x < 0 ? -(R)b.d[0] : (R)b.d[0]) - p.x) * i0;
    const R d1 = ((v.y < 0 ? -(R)b.d[1] : (R)b.d[1]) - p.y) * i1;
    const R d2 = ((v.z < 0 ? -(R)b.d[2] : (R)b.d[2]) - p.z) * i2;
    R dist = d0;
    if (d1 < dist) dist = d1;
    if (d2 < dist) dist = d2;
    return dist;
  }

  // :801-818 SafetyToInKernel
  static VGB_HD R safety_to_in(const BoxP &b, const V3<R> &p) {
    R s = -(R)b.d[0] + fabs(p.x);
    const R sy = -(R)b.d[1] + fabs(p.y);
    const R sz = -(R)b.d[2] + fabs(p.z);
    if (sy > s) s = sy;
    if (sz > s) s = sz;
    return s;
  }

  // :820-837 SafetyToOutKernel
  static VGB_HD R safety_to_out(const BoxP &b, const V3<R> &p) {
    R s = (R)b.d[0] - fabs(p.x);
    const R sy = (R)b.d[1] - fabs(p.y);
    const R sz = (R)b.d[2] - fabs(p.z);
    if (sy < s) s = sy;
    if (sz < s) s = sz;
    return s;
  }
};

}  // namespace vgb
