// tube.cuh -- Tube shape arithmetic (device), templated on the arithmetic type.
//
// Follows volumes/kernel/TubeImplementation.h as the reference Scalar backend
// runs it: UniversalTube (source/UnplacedTube.cpp:52-70, rmin and phi handled
// at run time) with the scalar early returns of DistanceToIn.
#pragma once
#include "wedge.cuh"

namespace vgb {

// UnplacedTube with its cached values (volumes/UnplacedTube.h:26-80).
struct TubeP {
  double rmin, rmax, z, sphi, dphi;
  double rmin2, rmax2;
  double a1x, a1y, a2x, a2y;  // fAlongPhi{1,2}{x,y}
  double tolIrmin2, tolOrmin2, tolIrmax2, tolOrmax2, tolIz, tolOz;
  WedgeP wedge;
  int32_t has_rmin;    // checkRminTreatment: rmin > 0
  int32_t has_phi;     // checkPhiTreatment: dphi < 2 pi
  int32_t le_pi;       // PointInCyclicalSector: dphi <= M_PI
  int32_t pad;
};

template <class R> struct TubeOps {
  static constexpr int kDistanceBlocks = 5;  // resident blocks of the distance kernels
  using W = WedgeOps<R>;

  // TubeUtilities::PointInCyclicalSector<onSurface=false> (:55-92)
  static VGB_HD bool in_sector(const TubeP &t, R x, R y) {
    const R startCheck = (-x * (R)t.a1y + y * (R)t.a1x);
    const R endCheck = (-(R)t.a2x * y + (R)t.a2y * x);
    const R mt = -(R)kTolerance;
    if (t.le_pi) return (startCheck >= mt) & (endCheck >= mt);
    return (startCheck >= mt) | (endCheck >= mt);
  }

  // GenericKernelForContainsAndInside (:287-350)
  template <bool ForInside>
  static VGB_HD void contains_inside(const TubeP &t, const V3<R> &p, bool &cin, bool &cout) {
    const R absz = fabs(p.z);
    const R tol = (R)kTolerance;
    cout = absz > (ForInside ? (R)t.z + (R)kHalfTolerance : (R)t.z);
    if (ForInside) cin = absz < (R)t.z - (R)kHalfTolerance;
    const R r2 = p.x * p.x + p.y * p.y;
    cout |= r2 > (ForInside ? (R)t.rmax2 + tol * (R)t.rmax : (R)t.rmax2);
    if (ForInside) cin &= r2 < (R)t.rmax2 - tol * (R)t.rmax;
    if (t.has_rmin) {
      cout |= r2 <= (ForInside ? (R)t.rmin2 - tol * (R)t.rmin : (R)t.rmin2);
      if (ForInside) cin &= r2 > (R)t.rmin2 + tol * (R)t.rmin;
    }
    if (t.has_phi) {
      bool wi, wo;
      W::template contains_inside<ForInside>(t.wedge, p.x, p.y, wi, wo);
      cout |= wo;
      if (ForInside) cin &= wi;
    }
  }

  static VGB_HD bool contains(const TubeP &t, const V3<R> &p) {
    bool ci, co;
    contains_inside<false>(t, p, ci, co);
    return !co;
  }

  static VGB_HD int inside(const TubeP &t, const V3<R> &p) {
    bool ci, co;
    contains_inside<true>(t, p, ci, co);
    return ci ? kInside : (co ? kOutside : kSurface);
  }

  // CircleTrajectoryIntersection (:94-137)
  template <bool Largest, bool SectorCheck>
  static VGB_HD void circle_hit(R b, R c, const TubeP &t, const V3<R> &p, const V3<R> &v, R &dist,
                                bool &ok) {
    R delta = b * b - c;
    const bool dmask = Largest ? (delta >= (R)0.) : (delta > (R)0.);
    if (!dmask) delta = (R)0.;
    delta = sqrt(delta);
    if (!Largest) delta = -delta;
    dist = -b + delta;
    if (SectorCheck) {
      const R hitz = p.z + dist * v.z;
      const R hity = p.y + dist * v.y;
      const R hitx = p.x + dist * v.x;
      bool insector = true;
      if (t.has_phi) insector = W::contains_with_boundary(t.wedge, hitx, hity);
      ok = dmask & (dist >= (R)0) & (fabs(hitz) <= (R)t.z) & insector;
    } else {
      ok = dmask;
    }
  }

  // PhiPlaneTrajectoryIntersection<.., PositiveDirectionOfPhiVector, insectorCheck> (:231-267)
  template <bool PositiveDir, bool SectorCheck>
  static VGB_HD void phi_plane_hit(double alongX, double alongY, const TubeP &t, const V3<R> &p,
                                   const V3<R> &v, R &dist, bool &ok) {
    const R ax = (R)alongX, ay = (R)alongY;
    dist = (ay * p.x - ax * p.y) / (v.y * ax - v.x * ay);
    if (SectorCheck) {
      const R hitx = p.x + dist * v.x;
      const R hity = p.y + dist * v.y;
      const R hitz = p.z + dist * v.z;
      const R r2 = hitx * hitx + hity * hity;
      ok = fabs(hitz) <= (R)t.tolIz && (r2 >= (R)t.tolIrmin2) && (r2 <= (R)t.tolIrmax2) &&
           dist > 0;
      if (PositiveDir) ok = ok && (hitx * ax + hity * ay) > (R)0.;
    } else if (PositiveDir) {
      const R hitx = p.x + dist * v.x;
      const R hity = p.y + dist * v.y;
      ok = (hitx * ax + hity * ay) >= (R)0.;
    }
  }

  // DistanceToIn (:401-554), Scalar backend (early returns taken)
  static VGB_HD R distance_to_in(const TubeP &t, const V3<R> &p, const V3<R> &v, R /*step_max*/) {
    R distance = Lim<R>::inf();
    const R rsq = p.x * p.x + p.y * p.y;
    const R pdx = p.x * v.x;
    const R pdy = p.y * v.y;
    const R abspz = fabs(p.z);
    const R distz = (abspz - (R)t.z) / fabs(v.z);
    bool okz = (p.z * v.z) < 0;
    if (abspz > (R)t.z && !okz) return distance;
    if (fabs(p.x) > (R)t.rmax && pdx >= 0) return distance;
    if (fabs(p.y) > (R)t.rmax && pdy >= 0) return distance;
    const R hitx = p.x + distz * v.x;
    const R hity = p.y + distz * v.y;
    const R r2 = hitx * hitx + hity * hity;
    okz = okz & (distz > 0) & (r2 <= (R)t.tolIrmax2);
    if (t.has_rmin) okz = okz && ((R)t.tolIrmin2 <= r2);
    if (t.has_phi) okz = okz & in_sector(t, hitx, hity);
    if (okz) return distz;

    const R invnsq = (R)1 / ((R)1 - v.z * v.z);
    const R rdotn = pdx + pdy;
    const R b = invnsq * rdotn;
    const R crmax = invnsq * (rsq - (R)t.rmax2);
    R dist_rmax;
    bool ok_rmax;
    circle_hit<false, true>(b, crmax, t, p, v, dist_rmax, ok_rmax);
    if (ok_rmax) return dist_rmax;

    R dist_rmin = 0;
    bool ok_rmin = false;
    if (t.has_rmin) {
      const R crmin = invnsq * (rsq - (R)t.rmin2);
      circle_hit<true, true>(b, crmin, t, p, v, dist_rmin, ok_rmin);
      if (ok_rmin) distance = dist_rmin;
    }
    // ok_rmax and okz are false here (early returns above)
    if (t.has_phi) {
      R dist_phi;
      bool ok_phi;
      phi_plane_hit<true, true>(t.a1x, t.a1y, t, p, v, dist_phi, ok_phi);
      if (ok_phi && dist_phi < distance) distance = dist_phi;
      phi_plane_hit<true, true>(t.a2x, t.a2y, t, p, v, dist_phi, ok_phi);
      if (ok_phi && dist_phi < distance) distance = dist_phi;
    }
    return distance;
  }

  // DistanceToOut (:556-655); UniversalTube takes the "bigger than pi or
  // unknown" phi branch (positive-direction checks on both planes).
  static VGB_HD R distance_to_out(const TubeP &t, const V3<R> &p, const V3<R> &v, R /*step*/) {
    R distance = Lim<R>::inf();
    const R dirzsign = v.z < 0 ? (R)-1. : (R)1.;
    const R distz = ((R)t.z * dirzsign - p.z) / v.z;
    if (distz >= 0) distance = distz;
    const R invnsq = (R)1 / (v.x * v.x + v.y * v.y);
    const R rdotn = v.x * p.x + v.y * p.y;
    const R rsq = p.x * p.x + p.y * p.y;
    const R b = invnsq * rdotn;
    if (t.has_rmin) {
      const R crmin = invnsq * (rsq - (R)t.rmin2);
      R d;
      bool ok;
      circle_hit<false, false>(b, crmin, t, p, v, d, ok);
      if (ok && d >= 0 && d < distance) distance = d;
    }
    {
      const R crmax = invnsq * (rsq - (R)t.rmax2);
      R d;
      bool ok;
      circle_hit<true, false>(b, crmax, t, p, v, d, ok);
      if (ok && d >= 0 && d < distance) distance = d;
    }
    if (t.has_phi) {
      R d;
      bool ok = false;
      phi_plane_hit<true, false>(t.a1x, t.a1y, t, p, v, d, ok);
      if (ok && d > 0 && d < distance) distance = d;
      phi_plane_hit<true, false>(t.a2x, t.a2y, t, p, v, d, ok);
      if (ok && d > 0 && d < distance) distance = d;
    }
    return distance;
  }

  // PhiPlaneSafety<inside> (:183-214), SectorType kUnknownAngle
  template <bool Inside>
  static VGB_HD R phi_plane_safety(const TubeP &t, const V3<R> &p) {
    R phi1 = p.x * (R)t.a1y - p.y * (R)t.a1x;
    if (Inside) phi1 *= -1;
    const R inf = Lim<R>::inf();
    if (phi1 < 0 || p.x * (R)t.a1x + p.y * (R)t.a1y < 0) phi1 = inf;
    R phi2 = p.x * (R)t.a2y - p.y * (R)t.a2x;
    if (Inside) phi2 *= -1;
    phi2 *= -1;
    if (phi2 < 0 || p.x * (R)t.a2x + p.y * (R)t.a2y < 0) phi2 = inf;
    R safety = vmin(phi1, phi2);
    if (safety == inf) safety = (R)-1;
    return safety;
  }

  // SafetyToIn (:657-697)
  static VGB_HD R safety_to_in(const TubeP &t, const V3<R> &p) {
    const R r = sqrt(p.x * p.x + p.y * p.y);
    const R safez = fabs(p.z) - (R)t.z;
    const R safermax = r - (R)t.rmax;
    R safety = vmax(safez, safermax);
    if (t.has_rmin) safety = vmax(safety, (R)t.rmin - r);
    if (t.has_phi) {
      if (in_sector(t, p.x, p.y)) return safety;
      R safephi = phi_plane_safety<false>(t, p);
      safety = vmax(safety, safephi);
    }
    return safety;
  }

  // SafetyToOut (:699-730)
  static VGB_HD R safety_to_out(const TubeP &t, const V3<R> &p) {
    const R r = sqrt(p.x * p.x + p.y * p.y);
    const R safez = (R)t.z - fabs(p.z);
    const R safermax = (R)t.rmax - r;
    R safety = vmin(safez, safermax);
    if (t.has_rmin) safety = vmin(safety, r - (R)t.rmin);
    if (t.has_phi) {
      R safephi = phi_plane_safety<true>(t, p);
      if (safephi < 0) safephi = Lim<R>::inf();
      safety = vmin(safety, safephi);
    }
    return safety;
  }
};

}  // namespace vgb
