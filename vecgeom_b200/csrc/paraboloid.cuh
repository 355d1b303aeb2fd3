// paraboloid.cuh -- Paraboloid arithmetic (device), templated on the arithmetic
// type; follows volumes/kernel/ParaboloidImplementation.h as the reference
// Scalar backend runs it (early returns taken).  The surface is
// z = A rho^2 + B, cut at |z| = dz, with radius rlo at z = -dz and rhi at +dz.
#pragma once
#include "vgb_core.cuh"

namespace vgb {

// UnplacedParaboloid::SetRloAndRhiAndDz (source/UnplacedParaboloid.cpp:90-128)
struct ParaboloidP {
  double rlo, rhi, dz;
  double a, b, ainv, a2;
  double rlo2, rhi2;
  double tolOz;
  double dx;  // fDx = fDy = Max(fRhi, fRlo) (ComputeBoundingBox, :242-245)
};

template <class R> struct ParaboloidOps {
  // UnplacedInside (:87-132).  The inner z test compares with fTolOz, as the
  // reference does.
  static VGB_HD int inside(const ParaboloidP &q, const V3<R> &p) {
    const R rho2 = p.x * p.x + p.y * p.y;
    const R absZ = fabs(p.z);
    if (absZ > (R)q.tolOz) return kOutside;
    const R value = (R)q.a * rho2 + (R)q.b - p.z;
    if (value > (R)kHalfTolerance) return kOutside;
    if ((absZ < (R)q.tolOz) && (value < -(R)kHalfTolerance)) return kInside;
    return kSurface;
  }
  // UnplacedContains (:134-158): beyond |z| > dz it returns without writing
  // its result, which the single-point call initialises to false
  static VGB_HD bool contains(const ParaboloidP &q, const V3<R> &p) {
    if (fabs(p.z) > (R)q.dz) return false;
    const R aa = (R)q.a * (p.z - (R)q.b);
    const R rho2 = p.x * p.x + p.y * p.y;
    return !(aa < 0 || aa < (R)q.a2 * rho2);
  }

  // DistanceToIn (:210-322)
  static VGB_HD R distance_to_in(const ParaboloidP &q, const V3<R> &p, const V3<R> &v, R) {
    const R inf = Lim<R>::inf();
    const R dz = (R)q.dz;
    const R absZ = fabs(p.z);
    const R absDirZ = fabs(v.z);
    const R rho2 = p.x * p.x + p.y * p.y;
    const R pdx = p.x * v.x, pdy = p.y * v.y;
    const bool checkZ = p.z * v.z > 0;
    if (absZ > dz && checkZ) return inf;
    if ((rho2 > (R)q.rhi2) && (pdx > 0 && pdy > 0)) return inf;
    if ((fabs(p.x) > (R)q.rhi) && (pdx > 0)) return inf;
    if ((fabs(p.y) > (R)q.rhi) && (pdy > 0)) return inf;
    const R distZ = (absZ - dz) / absDirZ;
    const R xHit = p.x + distZ * v.x;
    const R yHit = p.y + distZ * v.y;
    const R rhoHit2 = xHit * xHit + yHit * yHit;
    R ray2 = (R)q.rhi2;
    if (p.z < -dz && v.z > 0) ray2 = (R)q.rlo2;
    if ((absZ > dz) && (!checkZ) && (rhoHit2 <= ray2)) return distZ;
    const R dirRho2 = v.x * v.x + v.y * v.y;
    const R a = (R)q.a * dirRho2;
    const R b = (R)2. * (R)q.a * (pdx + pdy) - v.z;
    const R c = (R)q.a * rho2 + (R)q.b - p.z;
    const R ainv = (R)1. / a;
    const R t = b * (R)0.5;
    const R prod = c * a;
    R delta = t * t - prod;
    if (delta < 0) return inf;
    delta = sqrt(delta);
    const R distParab = ainv * (-t - delta);
    const R zHit = p.z + distParab * v.z;
    const bool hit = (distParab > (R)1E20) || (fabs(zHit) <= dz);
    return (hit && distParab > 0) ? distParab : inf;
  }

  // DistanceToOut (:325-380): the nearer of the z plane ahead and the
  // paraboloid root ahead (sqrt of a negative discriminant gives NaN roots,
  // which select nothing)
  static VGB_HD R distance_to_out(const ParaboloidP &q, const V3<R> &p, const V3<R> &v, R) {
    const R inf = Lim<R>::inf();
    const R dz = (R)q.dz;
    const R dirZinv = (R)1 / v.z;
    const R distZ = (v.z < 0) ? -(dz + p.z) * dirZinv : (dz - p.z) * dirZinv;
    const R rho2 = p.x * p.x + p.y * p.y;
    const R dirRho2 = v.x * v.x + v.y * v.y;
    const R a = (R)q.a * dirRho2;
    const R b = (R)2. * (R)q.a * (p.x * v.x + p.y * v.y) - v.z;
    const R c = (R)q.a * rho2 + (R)q.b - p.z;
    const R ainv = (R)1. / a;
    const R t = b * (R)0.5;
    const R prod = c * a;
    const R delta = sqrt(t * t - prod);
    const R sign = (ainv < 0) ? (R)-1. : (R)1.;
    const R d1 = ainv * (-t - sign * delta);
    const R d2 = ainv * (-t + sign * delta);
    R distParab = inf;
    if (d1 > 0) distParab = d1;
    if (d1 < 0 && d2 > 0) distParab = d2;
    if (d1 < 0 && d2 < 0) distParab = inf;
    return vmin(distParab, distZ);
  }

  // SafetyToIn (:383-527, the code outside the #ifdef variants)
  static VGB_HD R safety_to_in(const ParaboloidP &q, const V3<R> &p) {
    const R safeZ = fabs(p.z) - (R)q.dz;
    const R r = sqrt(p.x * p.x + p.y * p.y);
    const R safeRhi = r - (R)q.rhi;
    if ((safeZ > 0) || (safeRhi > 0)) return vmax(safeZ, safeRhi);
    const R r0sq = (p.z - (R)q.b) * (R)q.ainv;
    const R dr = r - sqrt(r0sq);
    const R talf = (R)-2. * (R)q.a * sqrt(r0sq);
    const R salf = talf / sqrt((R)1. + talf * talf);
    const R safR = fabs(dr * salf);
    return vmax(safR, safeZ);
  }

  // SafetyToOut (:530-550)
  static VGB_HD R safety_to_out(const ParaboloidP &q, const V3<R> &p) {
    const R safZ = (R)q.dz - fabs(p.z);
    const R r = sqrt(p.x * p.x + p.y * p.y);
    const R safRlo = (R)q.rlo - r;
    const R s = vmin(safZ, safRlo);
    return s > 0 ? s : (R)0;
  }
};

}  // namespace vgb
