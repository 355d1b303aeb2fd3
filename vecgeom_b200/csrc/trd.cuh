// trd.cuh -- Trd shape arithmetic (device), templated on the arithmetic type.
//
// Follows volumes/kernel/TrdImplementation.h as the reference Scalar backend
// runs it: the placed volume is specialised as Trd1 (dy1 == dy2, y not
// varying) or Trd2 (source/UnplacedTrd.cpp:221-236); here that choice is the
// record's varying_y flag, a warp-uniform branch.
#pragma once
#include "vgb_core.cuh"

namespace vgb {

// UnplacedTrd with its cached values (volumes/UnplacedTrd.h:20-51).
struct TrdP {
  double dx1, dx2, dy1, dy2, dz;
  double x2minusx1, y2minusy1, dztimes2, halfx1plusx2, halfy1plusy2;
  double fx, fy, calfx, calfy;
  int32_t varying_y;  // dy1 != dy2 (Trd2)
  int32_t pad;
};

template <class R> struct TrdOps {
  // TrdUtilities::UnplacedInside<surfaceT> (:112-140)
  template <bool Surface>
  static VGB_HD void kernel(const TrdP &t, const V3<R> &p, bool &cin, bool &cout) {
    const R ht = (R)kHalfTolerance;
    const R pzPlusDz = p.z + (R)t.dz;
    cout = fabs(p.z) > (Surface ? (R)t.dz + ht : (R)t.dz);
    if (Surface) cin = fabs(p.z) < (R)t.dz - ht;
    // PointLineOrientation: cross = vx*py - vy*px
    R cross = (R)t.x2minusx1 * pzPlusDz - (R)t.dztimes2 * (fabs(p.x) - (R)t.dx1);
    cout |= (Surface ? cross + ht : cross) < 0;
    if (Surface) cin &= cross - ht > 0;
    if (t.varying_y) {
      cross = (R)t.y2minusy1 * pzPlusDz - (R)t.dztimes2 * (fabs(p.y) - (R)t.dy1);
      cout |= (Surface ? cross + ht : cross) < 0;
      if (Surface) cin &= cross - ht > 0;
    } else {
      cout |= fabs(p.y) > (Surface ? (R)t.dy1 + ht : (R)t.dy1);
      if (Surface) cin &= fabs(p.y) < (R)t.dy1 - ht;
    }
  }

  static VGB_HD bool contains(const TrdP &t, const V3<R> &p) {
    bool ci, co;
    kernel<false>(t, p, ci, co);
    return !co;
  }

  // :186-200: kSurface, then kInside, then kOutside (outside wins)
  static VGB_HD int inside(const TrdP &t, const V3<R> &p) {
    bool ci, co;
    kernel<true>(t, p, ci, co);
    return co ? kOutside : (ci ? kInside : kSurface);
  }

  // FaceTrajectoryIntersection<forY, mirroredPoint> (:62-96)
  template <bool ForY, bool Mirrored>
  static VGB_HD void face(const TrdP &t, const V3<R> &pos, const V3<R> &dir, R &dist, bool &ok) {
    R alongV, posV, dirV, posK, dirK, fK, halfKplus, v1;
    if (ForY) {
      alongV = (R)t.y2minusy1; v1 = (R)t.dy1; posV = pos.y; posK = pos.x; dirV = dir.y;
      dirK = dir.x; fK = (R)t.fx; halfKplus = (R)t.halfx1plusx2;
    } else {
      alongV = (R)t.x2minusx1; v1 = (R)t.dx1; posV = pos.x; posK = pos.y; dirV = dir.x;
      dirK = dir.y; fK = (R)t.fy; halfKplus = (R)t.halfy1plusy2;
    }
    if (Mirrored) {
      posV *= -1;
      dirV *= -1;
    }
    const R alongZ = (R)t.dztimes2;
    dist = (alongZ * (posV - v1) - alongV * (pos.z + (R)t.dz)) / (dir.z * alongV - dirV * alongZ);
    ok = dist > 0;
    if (ok) {
      const R hitz = pos.z + dist * dir.z;
      ok &= fabs(hitz) <= (R)t.dz;
      const R hitk = posK + dist * dirK;
      const R dK = halfKplus - fK * hitz;
      ok &= fabs(hitk) <= dK;
    }
  }

  // DistanceToIn (:202-262); no early return in the reference's flow
  static VGB_HD R distance_to_in(const TrdP &t, const V3<R> &p, const V3<R> &v, R) {
    R distance = Lim<R>::inf();
    bool okz = p.z * v.z < 0;
    if (okz) {
      const R distz = (fabs(p.z) - (R)t.dz) / fabs(v.z);
      const R hitx = fabs(p.x + distz * v.x);
      const R hity = fabs(p.y + distz * v.y);
      const bool okzt = p.z > (R)t.dz && hitx <= (R)t.dx2 && hity <= (R)t.dy2;
      const bool okzb = p.z < -(R)t.dz && hitx <= (R)t.dx1 && hity <= (R)t.dy1;
      okz &= (okzt | okzb);
      if (okz) distance = distz;
    }
    R d;
    bool ok;
    face<false, false>(t, p, v, d, ok);
    if (ok && d < distance) distance = d;
    face<false, true>(t, p, v, d, ok);
    if (ok && d < distance) distance = d;
    if (t.varying_y) {
      face<true, false>(t, p, v, d, ok);
      if (ok && d < distance) distance = d;
      face<true, true>(t, p, v, d, ok);
      if (ok && d < distance) distance = d;
    } else {
      const R disty = (fabs(p.y) - (R)t.dy1) / fabs(v.y);
      const R zhit = p.z + disty * v.z;
      const R xhit = p.x + disty * v.x;
      const R dx = (R)t.halfx1plusx2 - (R)t.fx * zhit;
      const bool oky = p.y * v.y < 0 && disty > 0 && fabs(xhit) < dx && fabs(zhit) < (R)t.dz;
      if (oky && disty < distance) distance = disty;
    }
    return distance;
  }

  // DistanceToOut (:264-336), Scalar backend (early returns taken)
  static VGB_HD R distance_to_out(const TrdP &t, const V3<R> &p, const V3<R> &v, R) {
    R distance = Lim<R>::inf();
    if (v.z > 0) {
      const R distz = ((R)t.dz - p.z) / fabs(v.z);
      const R hitx = fabs(p.x + distz * v.x);
      const R hity = fabs(p.y + distz * v.y);
      if (hitx <= (R)t.dx2 && hity <= (R)t.dy2) return distz;
    }
    if (v.z < 0) {
      const R distz = (p.z - (-(R)t.dz)) / fabs(v.z);
      const R hitx = fabs(p.x + distz * v.x);
      const R hity = fabs(p.y + distz * v.y);
      if (hitx <= (R)t.dx1 && hity <= (R)t.dy1) return distz;
    }
    R d;
    bool ok;
    face<false, false>(t, p, v, d, ok);
    if (ok) return d;
    face<false, true>(t, p, v, d, ok);
    if (ok) return d;
    if (t.varying_y) {
      face<true, false>(t, p, v, d, ok);
      if (ok) return d;
      face<true, true>(t, p, v, d, ok);
      if (ok) distance = d;
    } else {
      const R plane = v.y < 0 ? -(R)t.dy1 : (R)t.dy1;
      const R disty = (plane - p.y) / v.y;
      const R zhit = p.z + disty * v.z;
      const R xhit = p.x + disty * v.x;
      const R dx = (R)t.halfx1plusx2 - (R)t.fx * zhit;
      if (fabs(xhit) < dx && fabs(zhit) < (R)t.dz) distance = disty;
    }
    return distance;
  }

  // TrdUtilities::Safety<inside> (:98-110)
  template <bool Inside>
  static VGB_HD R safety(const TrdP &t, const V3<R> &p) {
    const R safz = (R)t.dz - fabs(p.z);
    R dist = safz;
    const R distx = (R)t.halfx1plusx2 - (R)t.fx * p.z;
    const bool okx = distx >= 0;
    const R safx = (distx - fabs(p.x)) * (R)t.calfx;
    if (okx && safx < dist) dist = safx;
    if (t.varying_y) {
      const R disty = (R)t.halfy1plusy2 - (R)t.fy * p.z;
      const bool oky = disty >= 0;
      const R safy = (disty - fabs(p.y)) * (R)t.calfy;
      if (oky && safy < dist) dist = safy;
    } else {
      const R safy = (R)t.dy1 - fabs(p.y);
      if (safy < dist) dist = safy;
    }
    return Inside ? dist : -dist;
  }

  static VGB_HD R safety_to_in(const TrdP &t, const V3<R> &p) { return safety<false>(t, p); }
  static VGB_HD R safety_to_out(const TrdP &t, const V3<R> &p) { return safety<true>(t, p); }
};

}  // namespace vgb
