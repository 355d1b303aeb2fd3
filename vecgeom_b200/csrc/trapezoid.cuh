// trapezoid.cuh -- general Trapezoid (G4Trap-like) arithmetic (device),
// templated on the arithmetic type; follows volumes/kernel/TrapezoidImplementation.h
// with the four side planes held as a plane shell (base/PlaneShell.h), the
// reference's default build (CMake option PLANESHELL ON), as the Scalar backend
// runs it.  The z faces are handled apart from the four side planes.
#pragma once
#include "vgb_core.cuh"

namespace vgb {

// UnplacedTrapezoid (volumes/UnplacedTrapezoid.h:31-60): the four side planes
// a x + b y + c z + d = 0 with outward unit normals (-Y, +Y, -X, +X faces, in
// that order, source/UnplacedTrapezoid.cpp:215-262), then the parameters the
// Extent is computed from.
struct TrapezoidP {
  double a[4], b[4], c[4], d[4];
  double dz;
  double tthetaCphi, tthetaSphi;  // tan(theta) cos(phi), tan(theta) sin(phi)
  double dy1, dx1, dx2, tanAlpha1;
  double dy2, dx3, dx4, tanAlpha2;
  double theta, phi;
};

template <class R> struct TrapezoidOps {
  // signed distance of p to side plane i (PlaneShell.h DistanceToPoint)
  static VGB_HD R plane(const TrapezoidP &t, int i, const V3<R> &p) {
    return (R)t.a[i] * p.x + (R)t.b[i] * p.y + (R)t.c[i] * p.z + (R)t.d[i];
  }
  static VGB_HD R proj(const TrapezoidP &t, int i, const V3<R> &v) {
    return (R)t.a[i] * v.x + (R)t.b[i] * v.y + (R)t.c[i] * v.z;
  }

  // GenericKernelForContainsAndInside<ForInside = false>
  // (TrapezoidImplementation.h:118-156, PlaneShell.h:134-160)
  static VGB_HD bool contains(const TrapezoidP &t, const V3<R> &p) {
    if (fabs(p.z) > (R)t.dz) return false;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (plane(t, i, p) > (R)0) return false;
    return true;
  }

  // the same kernel with ForInside = true: half-tolerant on both sides
  static VGB_HD int inside(const TrapezoidP &t, const V3<R> &p) {
    const R ht = (R)kHalfTolerance;
    const R az = fabs(p.z);
    if (az > (R)t.dz + ht) return kOutside;
    bool in = az < (R)t.dz - ht;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const R d = plane(t, i, p);
      if (d > (R)0 + ht) return kOutside;
      in = in && d < (R)0 - ht;
    }
    return in ? kInside : kSurface;
  }

  // DistanceToIn (TrapezoidImplementation.h:232-379): the z slab gives
  // [smin, smax], the plane shell (PlaneShell.h:169-236) the entry along the
  // ray from smin on; an entry equal to the slab's exit falls back to smin.
  static VGB_HD R distance_to_in(const TrapezoidP &t, const V3<R> &p, const V3<R> &v, R) {
    const R inf = Lim<R>::inf();
    const R ht = (R)kHalfTolerance;
    const R dz = (R)t.dz;
    const bool posZ = v.z > (R)0, negZ = v.z < (R)0;
    const R zsign = negZ ? (R)-1 : (R)1;
    const R zmax = zsign * dz - p.z;
    if ((posZ && zmax < (R)0 + ht) || (negZ && zmax > (R)0 - ht)) return inf;
    const R dirFactor = (R)1 / v.z;
    R smax = zmax * dirFactor;
    R smin = (-zsign * dz - p.z) * dirFactor;
    const bool flat = !posZ && !negZ;
    if (flat) {
      if (!(fabs(p.z) < dz - ht)) return inf;
      smin = (R)0;
      smax = inf;
    }
    // the plane shell, starting from smin with its own open far end
    R pd[4], pr[4], vd[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      pd[i] = plane(t, i, p);
      pr[i] = proj(t, i, v);
      vd[i] = -pd[i] / pr[i];
    }
    R s = smin, sfar = inf;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const bool posPoint = pd[i] >= -(R)kHalfTolerance;
      const bool posDir = pr[i] > (R)0;
      if (posPoint && posDir) return inf;
      const bool fromInside = !posPoint && posDir;
      if (fromInside && vd[i] < s) return inf;
      const bool fromOutside = posPoint && !posDir;
      if (fromOutside && vd[i] > sfar) return inf;
      const bool valid = s < vd[i] && vd[i] < sfar;
      if (fromOutside && valid) s = vd[i];
      if (fromInside && valid) sfar = vd[i];
    }
    const V3<R> e{p.x + v.x * s, p.y + v.y * s, p.z + v.z * s};
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (!(plane(t, i, e) <= (R)0 + ht)) return inf;
    // back in the trapezoid kernel with the shell's answer s
    if (s == inf || s > smax) return inf;
    R distance = (s > smin && s < smax) ? s : smin;
    if (distance < (R)0) distance = (R)0;
    return distance;
  }

  // DistanceToOut (TrapezoidImplementation.h:385-463, PlaneShell.h:238-277)
  static VGB_HD R distance_to_out(const TrapezoidP &t, const V3<R> &p, const V3<R> &v, R) {
    const R ht = (R)kHalfTolerance;
    const bool posZ = v.z > (R)0, negZ = v.z < (R)0;
    const R zsign = negZ ? (R)-1 : (R)1;
    const R zmax = zsign * (R)t.dz - p.z;
    if ((posZ && zmax <= (R)0 + ht) || (negZ && zmax >= (R)0 - ht)) return (R)0;
    R distance = zmax / v.z;
    R shell = Lim<R>::inf();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const R pr = proj(t, i, v);
      const R vd = -plane(t, i, p) / pr;
      if (vd >= (R)0 && pr > (R)0 && vd < shell) shell = vd;
    }
    if (shell < distance) distance = shell;
    return distance;
  }

  // SafetyToIn (TrapezoidImplementation.h:469-499, PlaneShell.h:279-302): no
  // clamp at zero
  static VGB_HD R safety_to_in(const TrapezoidP &t, const V3<R> &p) {
    R s = fabs(p.z) - (R)t.dz;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const R d = plane(t, i, p);
      if (d > s) s = d;
    }
    return s;
  }

  // SafetyToOut (:504-541, PlaneShell.h:304-320): zero on and beyond the z
  // faces, else the side planes may take it below zero
  static VGB_HD R safety_to_out(const TrapezoidP &t, const V3<R> &p) {
    R s = (R)t.dz - fabs(p.z);
    if (s < (R)0) s = (R)0;
    if (s == (R)0) return s;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const R d = -plane(t, i, p);
      if (d < s) s = d;
    }
    return s;
  }
};

}  // namespace vgb
