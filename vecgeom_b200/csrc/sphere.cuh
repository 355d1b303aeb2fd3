// sphere.cuh -- Sphere shape arithmetic (device), templated on the arithmetic type.
//
// Inside/Contains, SafetyToIn/Out and DistanceToOut follow
// volumes/kernel/SphereImplementation.h (ROOT TGeoSphere lineage) as the
// reference Scalar backend runs them, including its flag use: the kernels ask
// IsFullPhiSphere(), which returns fFullSphere (volumes/UnplacedSphere.h:262-270),
// so a full-phi sphere with a theta cut still runs the phi-plane code.
//
// DistanceToIn is an empty stub in the reference (SphereImplementation.h:84-93);
// the vendored USolids USphere::DistanceToIn (USolids/src/USphere.cc:630-1563,
// the Geant4 G4Sphere algorithm) is the in-tree definition this restates.
#pragma once
#include "vgb_core.cuh"

namespace vgb {

// A polar-angle cut c the kernels compare theta = atan2(rho, z) with, and its
// sine and cosine (mode 1: c < 0, below every theta; mode 2: c above pi).
struct ThetaCut {
  double c, sn, cs;
  int32_t mode;
  int32_t pad;
};
// the cuts: Inside's (fSTheta -/+ half tolerance, eTheta -/+ half tolerance)
// and DistanceToIn's (tolSTheta, tolETheta, tolSTheta + kAngTolerance,
// tolETheta - kAngTolerance), each the double value the reference compares with
enum { kCutInS0, kCutInS1, kCutInE0, kCutInE1, kCutTolS, kCutTolE, kCutTolS2, kCutTolE2, kCuts };

// UnplacedSphere / USphere cached values (volumes/UnplacedSphere.h:25-215,
// source/UnplacedSphere.cpp:24-95, USolids/src/USphere.cc:30-60).
struct SphereP {
  double rmin, rmax, sphi, dphi, stheta, dtheta;
  double rminTolerance;  // fRminTolerance
  double mkTolerance;    // USphere::kTolerance = max(kRadTolerance, fEpsilon*fRmax)
  double hDPhi, cPhi, ePhi, sinCPhi, cosCPhi, cosHDPhiIT, cosHDPhiOT;
  double sinSPhi, cosSPhi, sinEPhi, cosEPhi;
  double eTheta, sinSTheta, cosSTheta, sinETheta, cosETheta, tanSTheta2, tanETheta2;
  double cosHDPhi;       // cos(hDPhi), as SafetyToIn evaluates it
  double sinPhim, cosPhim;  // sin/cos(0.5*(fSPhi + ePhi)), as DistanceToOut evaluates them
  int32_t fullPhi;    // fFullPhiSphere
  int32_t fullTheta;  // fFullThetaSphere
  int32_t full;       // fFullSphere (what IsFullPhiSphere() returns)
  int32_t pad;
  ThetaCut cut[kCuts];
};

template <class R> struct SphereOps {
  static constexpr double kHalfAngTol = 0.5 * kAngTolerance;

  // The reference compares polar angles theta = atan2(rho, z) with fixed cuts.
  // z sin c - rho cos c = r sin(c - theta) decides such a comparison without
  // atan2 when theta is more than ~3e-15 rad from the cut (the margin covers
  // the rounding of this expression and of sin c, cos c, rho), well beyond the
  // error of atan2 itself (2 ulp, < 1e-15 rad), so the outcome is the one the
  // atan2 comparison gives.  Nearer the cut the comparison evaluates atan2.
  // -1: theta < c, +1: theta > c, 0: undecided.
  static VGB_HD int cut_side(R rho, R z, const ThetaCut &k) {
    if (k.mode == 1) return 1;
    if (k.mode == 2) return -1;
    const R f = z * (R)k.sn - rho * (R)k.cs;
    const R m = (R)4e-15 * (fabs(z) + rho);
    return f > m ? -1 : (f < -m ? 1 : 0);
  }
  // atan2(rho, z) out of line: it is needed only within ~3e-15 rad of a cut,
  // and one copy instead of one per comparison keeps the kernels' code small
  static VGB_HD_NOINLINE R polar_atan2(R rho, R z) { return atan2(rho, z); }

  // theta = atan2(rho, z), evaluated only when a comparison needs its value
  struct PolarAngle {
    R rho, z, t;
    bool known;
    VGB_HD PolarAngle(R rho_, R z_) : rho(rho_), z(z_), t(0), known(false) {}
    VGB_HD R value() {
      if (!known) {
        t = polar_atan2(rho, z);
        known = true;
      }
      return t;
    }
    VGB_HD bool lt(const ThetaCut &k) {
      const int sd = cut_side(rho, z, k);
      return sd ? sd < 0 : value() < (R)k.c;
    }
    VGB_HD bool le(const ThetaCut &k) {
      const int sd = cut_side(rho, z, k);
      return sd ? sd < 0 : value() <= (R)k.c;
    }
    VGB_HD bool gt(const ThetaCut &k) {
      const int sd = cut_side(rho, z, k);
      return sd ? sd > 0 : value() > (R)k.c;
    }
    VGB_HD bool ge(const ThetaCut &k) {
      const int sd = cut_side(rho, z, k);
      return sd ? sd > 0 : value() >= (R)k.c;
    }
  };

  // :804-880 GenericKernelForContainsAndInside (both flags always computed)
  static VGB_HD void kernel(const SphereP &s, const V3<R> &p, bool &cin, bool &cout) {
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    R tolRMin = (R)s.rmin + (R)(0.5 * s.rminTolerance);
    R tolRMax = (R)s.rmax - (R)(0.5 * s.rminTolerance);
    cin = (rad2 <= tolRMax * tolRMax) && (rad2 >= tolRMin * tolRMin);
    tolRMin = (R)s.rmin - (R)(0.5 * s.rminTolerance);
    tolRMax = (R)s.rmax + (R)(0.5 * s.rminTolerance);
    cout = (rad2 <= tolRMin * tolRMin) || (rad2 >= tolRMax * tolRMax);
    if (cout) return;
    const R ht = (R)kHalfAngTol;
    // A full-phi sphere with a theta cut still runs the phi test (fFullSphere
    // is false).  With fSPhi = 0 and fDPhi = 2 pi the test only changes the
    // result for points within the half tolerance of phi = 0 (they lose
    // kInside); a point with x < 0, or with |y| > 1e-8 |x| (more than 1e-8 rad
    // from phi = 0), keeps cin and cout as they are without atan2.
    const bool phi_far = s.fullPhi && ((p.x < 0) || (fabs(p.y) > (R)1e-8 * fabs(p.x)));
    if (!s.full && !phi_far) {
      R pPhi = atan2(p.y, p.x);
      const R fSPhi = (R)s.sphi, ePhi = (R)s.sphi + (R)s.dphi;
      if (pPhi < fSPhi - ht) pPhi = pPhi + (R)(2. * kPi);
      if (pPhi > ePhi + ht) pPhi = pPhi - (R)(2. * kPi);
      cin &= (pPhi <= ePhi - ht) && (pPhi >= fSPhi + ht);
      cout |= (pPhi < fSPhi - ht) || (pPhi > ePhi + ht);
      if (cout) return;
    }
    if (!s.fullTheta) {
      // pTheta = atan2(sqrt(x^2 + y^2), z) against stheta -/+ ht, eTheta -/+ ht
      PolarAngle th(sqrt(p.x * p.x + p.y * p.y), p.z);
      cin &= th.le(s.cut[kCutInE0]) && th.ge(s.cut[kCutInS1]);
      cout |= th.lt(s.cut[kCutInS0]) || th.gt(s.cut[kCutInE1]);
    }
  }

  static VGB_HD bool contains(const SphereP &s, const V3<R> &p) {
    bool ci, co;
    kernel(s, p, ci, co);
    return !co;
  }

  static VGB_HD int inside(const SphereP &s, const V3<R> &p) {
    bool ci, co;
    kernel(s, p, ci, co);
    return ci ? kInside : (co ? kOutside : kSurface);
  }

  // ---- DistanceToIn: USolids/src/USphere.cc:630-1563 ----------------------
  // phi test at an intersection: (x*cosCPhi + y*sinCPhi)/rho >= limit
  static VGB_HD bool psi_ok(const SphereP &s, R x, R y, R rho, double limit) {
    return (x * (R)s.cosCPhi + y * (R)s.sinCPhi) / rho >= (R)limit;
  }

  // The reference splits an outer-sphere hit farther than dRmax = 100 rmax
  // (:685-689): it moves the point fTerm = sd - fmod(sd, dRmax) along the ray,
  // runs DistanceToIn again from there (without splitting again) and carries on
  // from the original point with sd = fTerm + that distance.  far_split decides
  // the split with the body's own expressions; distance_to_in then runs the one
  // body twice, from the moved point (depth 1) and from the original point with
  // the outer distance replaced (depth 0), so the kernel holds a single copy of
  // it.  The arithmetic is the reference's, in its order.
  static VGB_HD bool far_split(const SphereP &s, const V3<R> &p, const V3<R> &v, R &fTerm) {
    const R fRmax = (R)s.rmax;
    const R dRmax = (R)100. * (R)s.rmax;
    const R rad2 = (p.x * p.x + p.y * p.y) + p.z * p.z;
    const R pDotV3d = (p.x * v.x + p.y * v.y) + p.z * v.z;
    const R c = rad2 - fRmax * fRmax;
    if (!(c > (R)s.mkTolerance * fRmax)) return false;
    const R d2 = pDotV3d * pDotV3d - c;
    if (!(d2 >= 0)) return false;
    const R sd = -pDotV3d - sqrt(d2);
    if (!(sd >= 0 && sd > dRmax)) return false;
    fTerm = sd - fmod(sd, dRmax);
    return true;
  }

  // depth 1: the run from the split point (no further split); depth 0: the run
  // from the point itself, where an outer distance beyond dRmax is `outer`
  static VGB_HD R dti_core(const SphereP &s, const V3<R> &p, const V3<R> &v, int depth, R outer) {
    const R inf = Lim<R>::inf();
    R snxt = inf;
    const R dRmax = (R)100. * (R)s.rmax;
    const R halfCarTol = (R)(kTolerance * 0.5);
    const R halfAngTol = (R)kHalfAngTol;
    const R halfTol = (R)s.mkTolerance * (R)0.5;
    const R halfRminTol = (R)s.rminTolerance * (R)0.5;
    const R fRmin = (R)s.rmin, fRmax = (R)s.rmax;
    const R tolORMin2 = (fRmin > halfRminTol) ? (fRmin - halfRminTol) * (fRmin - halfRminTol) : (R)0;
    const R tolIRMin2 = (fRmin + halfRminTol) * (fRmin + halfRminTol);
    const R tolORMax2 = (fRmax + halfTol) * (fRmax + halfTol);
    const R tolIRMax2 = (fRmax - halfTol) * (fRmax - halfTol);
    const R eTheta = (R)s.eTheta, fSTheta = (R)s.stheta;
    const R piby2 = (R)(kPi / 2);
    R xi, yi, zi, rhoi, rhoi2, radi2, sd, c, d2, t1, t2, b, d;

    const R rho2 = p.x * p.x + p.y * p.y;
    const R rad2 = rho2 + p.z * p.z;
    // polar angle of the point, the reference's atan2(sqrt(rho2), z); only
    // compared with the cuts (PolarAngle)
    PolarAngle pTheta(sqrt(rho2), p.z);
    const R pDotV2d = p.x * v.x + p.y * v.y;
    const R pDotV3d = pDotV2d + p.z * v.z;
    // theta of (rho, z) within [tolSTheta, tolETheta]
    auto theta_in = [&](R rh, R zz) {
      PolarAngle th(rh, zz);
      return th.ge(s.cut[kCutTolS]) && th.le(s.cut[kCutTolE]);
    };
    // pTheta within [tolSTheta + kAng, tolETheta - kAng]
    auto strictly_theta = [&]() {
      return pTheta.ge(s.cut[kCutTolS2]) && pTheta.le(s.cut[kCutTolE2]);
    };

    // outer sphere (:667-760)
    c = rad2 - fRmax * fRmax;
    if (c > (R)s.mkTolerance * fRmax) {
      d2 = pDotV3d * pDotV3d - c;
      if (d2 >= 0) {
        sd = -pDotV3d - sqrt(d2);
        if (sd >= 0) {
          if (depth == 0 && sd > dRmax) sd = outer;  // :685-689, split and recomputed
          xi = p.x + sd * v.x;
          yi = p.y + sd * v.y;
          rhoi = sqrt(xi * xi + yi * yi);
          if (!s.fullPhi && rhoi != 0) {
            if (psi_ok(s, xi, yi, rhoi, s.cosHDPhiOT)) {
              if (!s.fullTheta) {
                zi = p.z + sd * v.z;
                if (theta_in(rhoi, zi)) return sd;
              } else {
                return sd;
              }
            }
          } else {
            if (!s.fullTheta) {
              zi = p.z + sd * v.z;
              if (theta_in(rhoi, zi)) return sd;
            } else {
              return sd;
            }
          }
        }
      } else {
        return inf;
      }
    } else {
      d2 = pDotV3d * pDotV3d - c;
      if ((rad2 > tolIRMax2) && ((d2 >= (R)s.mkTolerance * fRmax) && (pDotV3d < 0))) {
        if (!s.fullPhi) {
          if (psi_ok(s, p.x, p.y, sqrt(rho2), s.cosHDPhiIT)) {
            if (!s.fullTheta) {
              if (strictly_theta()) return (R)0;
            } else {
              return (R)0;
            }
          }
        } else {
          if (!s.fullTheta) {
            if (strictly_theta()) return (R)0;
          } else {
            return (R)0;
          }
        }
      }
    }

    // inner sphere (:790-930)
    if (s.rmin != 0) {
      c = rad2 - fRmin * fRmin;
      d2 = pDotV3d * pDotV3d - c;
      if ((c > -halfRminTol) && (rad2 < tolIRMin2) &&
          ((d2 < fRmin * (R)kTolerance) || (pDotV3d >= 0))) {
        if (!s.fullPhi) {
          if (psi_ok(s, p.x, p.y, sqrt(rho2), s.cosHDPhiIT)) {
            if (!s.fullTheta) {
              if (strictly_theta()) return (R)0;
            } else {
              return (R)0;
            }
          }
        } else {
          if (!s.fullTheta) {
            if (strictly_theta()) return (R)0;
          } else {
            return (R)0;
          }
        }
      } else if (d2 >= 0) {
        sd = -pDotV3d + sqrt(d2);
        if (sd >= halfRminTol) {
          xi = p.x + sd * v.x;
          yi = p.y + sd * v.y;
          rhoi = sqrt(xi * xi + yi * yi);
          if (!s.fullPhi && rhoi != 0) {
            if (psi_ok(s, xi, yi, rhoi, s.cosHDPhiOT)) {
              if (!s.fullTheta) {
                zi = p.z + sd * v.z;
                if (theta_in(rhoi, zi)) snxt = sd;
              } else {
                snxt = sd;
              }
            }
          } else {
            if (!s.fullTheta) {
              zi = p.z + sd * v.z;
              if (theta_in(rhoi, zi)) snxt = sd;
            } else {
              snxt = sd;
            }
          }
        }
      }
    }

    // phi planes (:934-1040)
    if (!s.fullPhi) {
      for (int plane = 0; plane < 2; ++plane) {
        const R comp = plane == 0 ? v.x * (R)s.sinSPhi - v.y * (R)s.cosSPhi
                                  : -(v.x * (R)s.sinEPhi - v.y * (R)s.cosEPhi);
        if (!(comp < 0)) continue;
        const R dist = plane == 0 ? p.y * (R)s.cosSPhi - p.x * (R)s.sinSPhi
                                  : -(p.y * (R)s.cosEPhi - p.x * (R)s.sinEPhi);
        if (!(dist < halfCarTol)) continue;
        sd = dist / comp;
        if (!(sd < snxt)) continue;
        if (sd > 0) {
          xi = p.x + sd * v.x;
          yi = p.y + sd * v.y;
          zi = p.z + sd * v.z;
          rhoi2 = xi * xi + yi * yi;
          radi2 = rhoi2 + zi * zi;
        } else {
          sd = 0;
          xi = p.x;
          yi = p.y;
          zi = p.z;
          rhoi2 = rho2;
          radi2 = rad2;
        }
        const R side = yi * (R)s.cosCPhi - xi * (R)s.sinCPhi;
        const bool half_ok = plane == 0 ? (side <= 0) : (side >= 0);
        if ((radi2 <= tolORMax2) && (radi2 >= tolORMin2) && half_ok) {
          if (!s.fullTheta) {
            if (theta_in(sqrt(rhoi2), zi) && half_ok) snxt = sd;
          } else {
            snxt = sd;
          }
        }
      }
    }

    // theta cones (:1044-1560)
    if (!s.fullTheta) {
      const R dist2STheta = (s.stheta != 0) ? rho2 - p.z * p.z * (R)s.tanSTheta2 : inf;
      const R dist2ETheta = (s.eTheta < kPi) ? rho2 - p.z * p.z * (R)s.tanETheta2 : inf;
      // candidate on one theta cone (sd given); the boundary half-space check is
      // zi * (theta - pi/2) <= 0
      auto accept = [&](R sdv, R thetaC) {
        xi = p.x + sdv * v.x;
        yi = p.y + sdv * v.y;
        zi = p.z + sdv * v.z;
        rhoi2 = xi * xi + yi * yi;
        radi2 = rhoi2 + zi * zi;
        if ((radi2 <= tolORMax2) && (radi2 >= tolORMin2) && (zi * (thetaC - piby2) <= 0)) {
          if (!s.fullPhi && rhoi2 != 0) {
            if (psi_ok(s, xi, yi, sqrt(rhoi2), s.cosHDPhiOT)) snxt = sdv;
          } else {
            snxt = sdv;
          }
        }
      };
      const R tanS2 = (R)s.tanSTheta2, tanE2 = (R)s.tanETheta2;
      // The two cones' quadratics (t1, t2, b, c, d2, d of every branch below),
      // evaluated once for each lane that reaches this point instead of inside
      // the branches: points on either side of a cut take different branches,
      // and a warp would evaluate the same quadratic once per branch group.  The
      // expressions and their order are the reference's, and a branch uses a
      // cone only where the reference goes on with it (t1 != 0, d2 >= 0), so
      // every result is unchanged.  A missing cone (stheta = 0, eTheta = pi) has
      // dist2 = inf: its c is +-inf, so it never yields a candidate, and it is
      // not evaluated.
      const bool haveS = s.stheta != 0, haveE = s.eTheta < kPi;
      R t1S = 0, t2S = 0, bS = 0, d2S = -1, dS = 0;
      R t1E = 0, t2E = 0, bE = 0, d2E = -1, dE = 0;
      if (haveS) {
        t1S = (R)1 - v.z * v.z * ((R)1 + tanS2);
        t2S = pDotV2d - p.z * v.z * tanS2;
        bS = t2S / t1S;
        c = dist2STheta / t1S;
        d2S = bS * bS - c;
        dS = sqrt(d2S);
      }
      if (haveE) {
        t1E = (R)1 - v.z * v.z * ((R)1 + tanE2);
        t2E = pDotV2d - p.z * v.z * tanE2;
        bE = t2E / t1E;
        c = dist2ETheta / t1E;
        d2E = bE * bE - c;
        dE = sqrt(d2E);
      }
      const bool realS = haveS && (t1S != 0) && (d2S >= 0);
      const bool realE = haveE && (t1E != 0) && (d2E >= 0);
      if (pTheta.lt(s.cut[kCutTolS])) {
        // (unreachable without a start cone: the cut lies below theta = 0)
        if (realS) {
          sd = -bS - dS;
          zi = p.z + sd * v.z;
          if ((sd < 0) || (zi * (fSTheta - piby2) > 0)) sd = -bS + dS;
          if ((sd >= 0) && (sd < snxt)) accept(sd, fSTheta);
        }
        if (realE) {
          sd = -bE + dE;
          if ((sd >= 0) && (sd < snxt)) accept(sd, eTheta);
        }
      } else if (pTheta.gt(s.cut[kCutTolE])) {
        // (unreachable without an end cone: the cut lies above theta = pi)
        if (realE) {
          sd = -bE - dE;
          zi = p.z + sd * v.z;
          if ((sd < 0) || (zi * (eTheta - piby2) > 0)) sd = -bE + dE;
          if ((sd >= 0) && (sd < snxt)) accept(sd, eTheta);
        }
        if (realS) {
          sd = -bS + dS;
          if ((sd >= 0) && (sd < snxt)) accept(sd, fSTheta);
        }
      } else if (pTheta.lt(s.cut[kCutTolS2]) && (fSTheta > halfAngTol)) {
        if ((t2S >= 0 && tolIRMin2 < rad2 && rad2 < tolIRMax2 && s.stheta < kPi / 2) ||
            (t2S < 0 && tolIRMin2 < rad2 && rad2 < tolIRMax2 && s.stheta > kPi / 2) ||
            (v.z < 0 && tolIRMin2 < rad2 && rad2 < tolIRMax2 && s.stheta == kPi / 2)) {
          if (!s.fullPhi && rho2 != 0) {
            if (psi_ok(s, p.x, p.y, sqrt(rho2), s.cosHDPhiIT)) return (R)0;
          } else {
            return (R)0;
          }
        }
        if (realS) {
          sd = -bS + dS;
          if ((sd >= halfCarTol) && (sd < snxt) && (s.stheta < kPi / 2)) accept(sd, fSTheta);
        }
      } else if (pTheta.gt(s.cut[kCutTolE2]) && (s.eTheta < kPi - kAngTolerance)) {
        if (((t2E < 0) && (s.eTheta < kPi / 2) && (tolIRMin2 < rad2) && (rad2 < tolIRMax2)) ||
            ((t2E >= 0) && (s.eTheta > kPi / 2) && (tolIRMin2 < rad2) && (rad2 < tolIRMax2)) ||
            ((v.z > 0) && (s.eTheta == kPi / 2) && (tolIRMin2 < rad2) && (rad2 < tolIRMax2))) {
          if (!s.fullPhi && rho2 != 0) {
            if (psi_ok(s, p.x, p.y, sqrt(rho2), s.cosHDPhiIT)) return (R)0;
          } else {
            return (R)0;
          }
        }
        if (realE) {
          sd = -bE + dE;
          if ((sd >= halfCarTol) && (sd < snxt) && (s.eTheta > kPi / 2)) accept(sd, eTheta);
        }
      } else {
        if (realS) {
          sd = -bS + dS;
          if ((sd >= 0) && (sd < snxt)) accept(sd, fSTheta);
        }
        if (realE) {
          sd = -bE + dE;
          if ((sd >= 0) && (sd < snxt)) accept(sd, eTheta);
        }
      }
    }
    return snxt;
  }

  static VGB_HD R distance_to_in(const SphereP &s, const V3<R> &p, const V3<R> &v, R) {
    R fTerm = 0;
    V3<R> from = p;
    int depth = 0;
    if (far_split(s, p, v, fTerm)) {
      from = {p.x + fTerm * v.x, p.y + fTerm * v.y, p.z + fTerm * v.z};
      depth = 1;
    }
    R outer = 0;
    // one call site, so the body is inlined once
#pragma unroll 1
    while (true) {
      const R r = dti_core(s, from, v, depth, outer);
      if (depth == 0) return r;
      outer = fTerm + r;
      from = p;
      depth = 0;
    }
  }

  // ---- DistanceToOut: SphereImplementation.h:1267-1510 and its helpers -----

  // :384-441 DistanceToSphere
  static VGB_HD R to_sphere(const SphereP &s, const V3<R> &p, const V3<R> &v, R radius, bool check,
                            bool firstcross) {
    const R inf = Lim<R>::inf();
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const R pDotV3d = p.x * v.x + p.y * v.y + p.z * v.z;
    const R c = rad2 - radius * radius;
    const R d2 = pDotV3d * pDotV3d - c;
    if (d2 <= 0) return inf;
    const R d = sqrt(d2);
    R distance;
    const bool in = (c <= 0);
    if (in)
      distance = (-pDotV3d) + d;
    else if (firstcross)
      distance = (-pDotV3d) - d;
    else
      distance = (-pDotV3d) + d;
    if (distance < 0) distance = inf;
    if (check) {
      const V3<R> pt = {p.x + distance * v.x, p.y + distance * v.y, p.z + distance * v.z};
      if (!contains(s, pt)) distance = inf;
    }
    return distance;
  }

  // :314-382 DistanceToCone
  static VGB_HD void to_cone(const V3<R> &p, const V3<R> &v, R dzv, R r1v, R r2v, R &bv, R &deltav) {
    deltav = (R)-1;
    if (dzv < 0) return;
    const R ro0v = (R)0.5 * (r1v + r2v);
    const R tzv = (R)0.5 * (r2v - r1v) / dzv;
    const R rsqv = p.x * p.x + p.y * p.y;
    const R rcv = ro0v + p.z * tzv;
    R av = v.x * v.x + v.y * v.y - tzv * tzv * v.z * v.z;
    bv = p.x * v.x + p.y * v.y - tzv * rcv * v.z;
    R cv = rsqv - rcv * rcv;
    const R temp = fabs(av), temp2 = fabs(bv);
    const R toler = (R)1.e-10;
    if ((temp < toler) && (temp2 < toler)) return;
    if (temp < toler) {
      bv = (R)0.5 * (cv / bv);
      deltav = 0;
      return;
    }
    av = (R)1 / av;
    bv *= av;
    cv *= av;
    deltav = bv * bv - cv;
    deltav = deltav > 0 ? sqrt(deltav) : (R)-1;
  }

  // :257-312 DistanceToPhiMin (in = true)
  static VGB_HD R to_phi_min(const SphereP &s, const V3<R> &p, const V3<R> &v) {
    const R s1 = (R)s.sinSPhi, c1 = (R)s.cosSPhi, s2 = (R)s.sinEPhi, c2 = (R)s.cosEPhi;
    const R sm = (R)s.sinPhim, cm = (R)s.cosPhim;
    const R inf = Lim<R>::inf();
    R sfi1 = inf, sfi2 = inf, ss = 0;
    R un = v.x * s1 - v.y * c1;
    if (un > 0) {
      ss = (R)-1 * p.x * s1 + p.y * c1;
      if (ss >= 0) {
        ss = ss / un;
        if (((p.x + ss * v.x) * sm - (p.y + ss * v.y) * cm) >= 0) sfi1 = ss;
      }
    }
    un = (R)-1 * v.x * s2 + v.y * c2;
    if (un > 0) {
      ss = p.x * s2 - p.y * c2;
      if (ss >= 0) {
        ss = ss / un;
        if (((R)-1 * (p.x + ss * v.x) * sm + (p.y + ss * v.y) * cm) >= 0) sfi2 = ss;
      }
    }
    return vmin(sfi1, sfi2);
  }

  static VGB_HD R distance_to_out(const SphereP &s, const V3<R> &p, const V3<R> &v, R) {
    const R inf = Lim<R>::inf();
    const R zero = 0, one = 1, mone = -1;
    const R toler = (R)1.E-10, toler2 = (R)1.E+10;
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const R rad = sqrt(rad2);
    const R pDotV3d = p.x * v.x + p.y * v.y + p.z * v.z;
    const R rxy2 = p.x * p.x + p.y * p.y;
    R snxt = inf, b = 0, delta = 0, xnew = 0, ynew = 0, znew = 0;
    R sn1 = inf, rn1 = inf, sn2 = inf, rn2;
    const R fPhi1 = (R)s.sphi, fPhi2 = (R)s.ePhi;
    const R fRmin = (R)s.rmin, fRmax = (R)s.rmax;

    if ((fRmin > zero) && (rad <= (fRmin + toler)) && (pDotV3d < zero)) return inf;
    if ((fRmin > zero) && (pDotV3d < zero)) rn1 = to_sphere(s, p, v, fRmin, true, true);
    if ((rad >= (fRmax - toler)) && (pDotV3d >= zero)) return inf;
    rn2 = to_sphere(s, p, v, fRmax, false, false);
    const R sr = vmin(rn1, rn2);

    const bool isFullPhiSphere = s.full;
    // the phi test of a theta-cone candidate: atan2(y, x) - fPhi1 moved into
    // [0, 2 pi) against fPhi2 - fPhi1.  For a full-phi sphere (fPhi1 = 0,
    // fPhi2 = 2 pi) every angle passes, NaN excepted.
    auto in_phi_range = [&](R x, R y) {
      if (s.fullPhi) return !(x != x || y != y);
      R d = atan2(y, x) - fPhi1;
      if (d < zero) d = d + (R)(2 * kPi);
      return d <= (fPhi2 - fPhi1);
    };
    if (!s.fullTheta) {
      // one theta cone; returns true if the point leaves through it at once
      auto theta_cone = [&](bool first, R &snside) -> bool {
        const bool cond = first ? (s.stheta > 0) : (s.eTheta < kPi);
        // without this cone (stheta = 0, or eTheta = pi) the reference still
        // evaluates its quantities, over zero radii, and then returns false
        // before using any of them; a scalar lane returns at once
        if (!cond) return false;
        const R si = (R)(first ? s.sinSTheta : s.sinETheta);
        const R ci = (R)(first ? s.cosSTheta : s.cosETheta);
        R r1, r2, z1, z2;
        if (ci > zero) {
          r1 = fRmin * si; z1 = fRmin * ci; r2 = fRmax * si; z2 = fRmax * ci;
        } else {
          r1 = fRmax * si; z1 = fRmax * ci; r2 = fRmin * si; z2 = fRmin * ci;
        }
        const R dz = (R)0.5 * (z2 - z1);
        const V3<R> pt = {p.x, p.y, p.z - (R)0.5 * (z1 + z2)};
        const R zinv = one / dz;
        const R rin = (R)0.5 * (r1 + r2 + (r2 - r1) * pt.z * zinv);
        const R sigz = p.z < zero ? mone : one;
        const bool bigequ =
            first ? ((sigz * ci > zero) && (sigz * rxy2 < sigz * rin * (rin + sigz * toler)))
                  : ((sigz * ci > zero) && (sigz * rxy2 > sigz * rin * (rin - sigz * toler)));
        if (bigequ) {
          // on or past the cone: 0 if heading out of the solid, else no candidate here
          const R ddotn = pt.x * v.x + pt.y * v.y + (R)0.5 * (r1 - r2) * v.z * zinv * sqrt(rxy2);
          return first ? (sigz * ddotn <= zero) : (sigz * ddotn >= zero);
        }
        R bv = 0, deltav = 0;
        to_cone(pt, v, dz, r1, r2, bv, deltav);
        delta = deltav;
        b = bv;
        if (!(delta > zero)) return false;
        snxt = mone * b - delta;
        znew = pt.z + snxt * v.z;
        R temp = fabs(znew);
        if ((snxt > zero) && (temp < dz)) {
          if (isFullPhiSphere) {
            snside = snxt;
          } else {
            xnew = pt.x + snxt * v.x;
            ynew = pt.y + snxt * v.y;
            if (in_phi_range(xnew, ynew)) snside = snxt;
          }
        }
        // second root: the reference tests sn > toler (end cone) / sn > toler2
        // (start cone) before moving snxt, and sn > toler2 for the rest
        if (first ? (snside > toler2) : (snside > toler)) snxt = mone * b + delta;
        if (snside > toler2) {
          znew = pt.z + snxt * v.z;
          temp = fabs(znew);
          if ((snxt > zero) && (temp < dz)) {
            if (isFullPhiSphere) {
              snside = snxt;
            } else {
              xnew = pt.x + snxt * v.x;
              ynew = pt.y + snxt * v.y;
              if (in_phi_range(xnew, ynew)) snside = snxt;
            }
          }
        }
        return false;
      };
      const double theta1Plane = fabs(s.stheta - kPi / 2);
      const double theta2Plane = fabs(s.eTheta - kPi / 2);
      if (theta1Plane < 1.e-10) {
        if ((p.z * v.z) < zero) sn1 = mone * p.z / v.z;
      } else if (theta_cone(true, sn1)) {
        return zero;
      }
      snxt = inf;
      if (theta2Plane < 1.e-10) {
        // the reference writes sn1 here (SphereImplementation.h:1398-1400)
        if ((p.z * v.z) < zero) sn1 = mone * p.z / v.z;
      } else if (theta_cone(false, sn2)) {
        return zero;
      }
    }
    const R st = vmin(sn1, sn2);
    R sp = inf;
    if (!s.full) sp = to_phi_min(s, p, v);
    const R srt = vmin(sr, st);
    return vmin(srt, sp);
  }

  // ---- safeties: SphereImplementation.h:948-1040, :1059-1140 -------------
  static VGB_HD R safety_to_in(const SphereP &s, const V3<R> &p) {
    const R zero = 0;
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const R rad = sqrt(rad2);
    const R rho2 = p.x * p.x + p.y * p.y;
    const R rho = sqrt(rho2);
    const R fRmin = (R)s.rmin;
    const R safeRMin = fRmin - rad;
    const R safeRMax = rad - (R)s.rmax;
    R safety;
    if (fRmin > zero)
      safety = (safeRMin > safeRMax) ? safeRMin : safeRMax;
    else
      safety = safeRMax;
    if (!s.full && (rho > zero)) {
      const R cosPsi = (p.x * (R)s.cosCPhi + p.y * (R)s.sinCPhi) / rho;
      R test1 = (p.x * (R)s.sinSPhi - p.y * (R)s.cosSPhi);
      if (test1 < 0) test1 = (R)-1 * test1;
      R test2 = (p.x * (R)s.sinEPhi - p.y * (R)s.cosEPhi);
      if (test2 < 0) test2 = (R)-1 * test2;
      if (cosPsi < (R)s.cosHDPhi) {
        const R safePhi = ((p.y * (R)s.cosCPhi - p.x * (R)s.sinCPhi) <= 0) ? test1 : test2;
        if (safePhi > safety) safety = safePhi;
      }
    }
    const R rds = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    if (!s.fullTheta && (rds != zero)) {
      // The reference takes pTheta = pi/2 - asin(z / rds) and, on the side of the
      // cut the point lies beyond, rds sin(stheta - pTheta) or rds sin(pTheta -
      // eTheta).  With sin pTheta = rho / rds and cos pTheta = z / rds these are
      // z sin(stheta) - rho cos(stheta) and rho cos(eTheta) - z sin(eTheta), whose
      // signs are those of the angle differences (both lie in [-pi, pi]; at most
      // one is positive, as stheta < eTheta).  Same value to ~1e-15 mm (rounding
      // of the two products against that of asin, the subtraction and sin),
      // without the two transcendental calls.
      const R toS = p.z * (R)s.sinSTheta - rho * (R)s.cosSTheta;
      const R toE = rho * (R)s.cosETheta - p.z * (R)s.sinETheta;
      const R safeTheta = toS > toE ? toS : toE;
      if (safeTheta >= zero && safety <= safeTheta) safety = safeTheta;
    }
    if (safety < zero) safety = zero;
    return safety;
  }

  static VGB_HD R safety_to_out(const SphereP &s, const V3<R> &p) {
    const R zero = 0;
    const R rad2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const R rad = sqrt(rad2);
    const R rho2 = p.x * p.x + p.y * p.y;
    const R rho = sqrt(rho2);
    const R safeRMin = rad - (R)s.rmin;
    const R safeRMax = (R)s.rmax - rad;
    R safety;
    if (s.rmin > 0)
      safety = (safeRMin < safeRMax) ? safeRMin : safeRMax;
    else
      safety = safeRMax;
    if (!s.full && (rho > 0)) {
      const R test1 = (p.y * (R)s.cosCPhi - p.x * (R)s.sinCPhi);
      const R safePhi = (test1 <= zero) ? (R)-1 * (p.x * (R)s.sinSPhi - p.y * (R)s.cosSPhi)
                                        : (p.x * (R)s.sinEPhi - p.y * (R)s.cosEPhi);
      if (safePhi < safety) safety = safePhi;
    }
    const R rds = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    if (!s.fullTheta && (rds > 0)) {
      // The reference's rds sin(pTheta - stheta) and rds sin(eTheta - pTheta)
      // (pTheta = pi/2 - asin(z / rds)), expanded as in SafetyToIn; it keeps the
      // one of the smaller angle, which for angles in [0, pi] with eTheta - stheta
      // <= pi is the smaller of the two values.
      const R fromS = rho * (R)s.cosSTheta - p.z * (R)s.sinSTheta;
      const R fromE = p.z * (R)s.sinETheta - rho * (R)s.cosETheta;
      const R safeTheta = fromS < fromE ? fromS : fromE;
      if (safety > safeTheta) safety = safeTheta;
    }
    if (safety < zero) safety = zero;
    return safety;
  }
};

}  // namespace vgb
