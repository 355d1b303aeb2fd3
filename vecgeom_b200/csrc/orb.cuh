// orb.cuh -- Orb (full solid sphere) arithmetic (device), templated on the
// arithmetic type; follows volumes/kernel/OrbImplementation.h as the reference
// Scalar backend runs it.
#pragma once
#include "vgb_core.cuh"

namespace vgb {

// UnplacedOrb (volumes/UnplacedOrb.h:27-35, source/UnplacedOrb.cpp:33-44).
struct OrbP {
  double r;
  double rTolerance;  // fRTolerance
  double rTolI;       // fR - fRTolerance
  double rTolO;       // fR + fRTolerance
};

template <class R> struct OrbOps {
  // GenericKernelForContainsAndInside (OrbImplementation.h:312-334)
  static VGB_HD void kernel(const OrbP &o, const V3<R> &p, bool &cin, bool &cout) {
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const R tolRMax = (R)o.rTolO, tolRMin = (R)o.rTolI;
    cout = rad2 > tolRMax * tolRMax;
    cin = rad2 < tolRMin * tolRMin;
  }
  static VGB_HD bool contains(const OrbP &o, const V3<R> &p) {
    bool ci, co;
    kernel(o, p, ci, co);
    return !co;
  }
  static VGB_HD int inside(const OrbP &o, const V3<R> &p) {
    bool ci, co;
    kernel(o, p, ci, co);
    return co ? kOutside : (ci ? kInside : kSurface);
  }

  // DistanceToInKernel (:352-405).  A ray from outside the outer tolerance
  // moving in takes -p.v - sqrt(d2) without checking d2, so a ray that misses
  // the orb gets NaN, as in the reference.
  static VGB_HD R distance_to_in(const OrbP &o, const V3<R> &p, const V3<R> &v, R) {
    const R inf = Lim<R>::inf();
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const R rad = sqrt(rad2);
    const R pDotV3d = p.x * v.x + p.y * v.y + p.z * v.z;
    const R radius2 = (R)o.r * (R)o.r;
    const R c = rad2 - radius2;
    const R d2 = pDotV3d * pDotV3d - c;
    const R tolI = (R)o.rTolI, tolO = (R)o.rTolO;
    if (rad < tolI) return inf;
    if ((rad >= tolI) && (rad <= tolO) && (pDotV3d < 0)) return (R)0;
    if ((rad >= tolI) && (rad <= tolO) && (pDotV3d >= 0)) return inf;
    if ((rad > tolO) && (pDotV3d < 0)) return -pDotV3d - sqrt(d2);
    return inf;
  }

  // DistanceToOutKernel (:410-462): 0 outside the outer tolerance and on the
  // tolerant surface moving out, the far root inside, and 0 for a point just
  // outside the radius within the tolerance that is neither (the reference
  // leaves its initial zero there)
  static VGB_HD R distance_to_out(const OrbP &o, const V3<R> &p, const V3<R> &v, R) {
    const R zero = 0;
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const R rad = sqrt(rad2);
    const R pDotV3d = p.x * v.x + p.y * v.y + p.z * v.z;
    const R radius = (R)o.r;
    const R radius2 = radius * radius;
    const R c = rad2 - radius2;
    const R d2 = pDotV3d * pDotV3d - c;
    const R tolRMax = (R)o.rTolO;
    const R tolRMax2 = tolRMax * tolRMax;
    if (rad2 > tolRMax2) return zero;
    const bool within = (rad <= tolRMax) && (c < ((R)kTolerance * radius));
    const bool onsurf = (c > (-2 * (R)kTolerance * radius)) && ((pDotV3d >= 0) || (d2 < 0));
    if (within && onsurf) return zero;
    if (within && !onsurf) return -pDotV3d + sqrt(d2);
    return zero;
  }

  // SafetyToInKernel / SafetyToOutKernel (:467-505)
  static VGB_HD R safety_to_in(const OrbP &o, const V3<R> &p) {
    const R rad = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    const R safe = rad - (R)o.r;
    return safe < (R)0 ? (R)0 : safe;
  }
  static VGB_HD R safety_to_out(const OrbP &o, const V3<R> &p) {
    const R rad = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    const R safe = (R)o.r - rad;
    return safe < (R)0 ? (R)0 : safe;
  }
};

}  // namespace vgb
