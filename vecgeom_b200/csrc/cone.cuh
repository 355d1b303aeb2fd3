// cone.cuh -- Cone shape arithmetic (device), templated on the arithmetic type.
//
// The reference runs the USolids/Geant4 cone algorithms for distances and
// safeties (volumes/kernel/ConeImplementation.h:237-1060 DistanceToInUSolids,
// :1221-1794 DistanceToOutUSOLIDS, :1813-1908 SafetyToInUSOLIDS, :1922-1989
// SafetyToOutUSOLIDS) and a slope/offset test for Contains/Inside (:83-158),
// as UniversalCone (source/UnplacedCone.cpp:255-270, no compile-time
// specialisation).  The branch structure and the rounding order follow those
// functions; every early return of the scalar code is kept.
#pragma once
#include "wedge.cuh"

namespace vgb {

// UnplacedCone with its cached values (volumes/UnplacedCone.h:60-170).
struct ConeP {
  double rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi;
  double innerSlope, outerSlope, innerOffset, outerOffset;
  double secRMin, secRMax, invSecRMin, invSecRMax;
  double cosCPhi, sinCPhi, cosSPhi, sinSPhi, cosEPhi, sinEPhi;
  double cosHDPhi, cosHDPhiIT, cosHDPhiOT;
  double tanRMin, tanRMax;
  WedgeP wedge;
  int32_t full_phi;  // IsFullPhi(): dphi == kTwoPi
  int32_t has_rmin;  // checkRminTreatment: rmin1 > 0 || rmin2 > 0
  int32_t has_phi;   // checkPhiTreatment: dphi < 2 pi
  int32_t pad;
};

template <class R> struct ConeOps {
  static constexpr int kDistanceBlocks = 5;  // resident blocks of the distance kernels
  using W = WedgeOps<R>;
  static constexpr double kHalfCarTol = kTolerance * 0.5;
  static constexpr double kHalfRadTol = kRadTolerance * 0.5;
  static constexpr double kHalfAngTol = kAngTolerance * 0.5;

  // :83-158 GenericKernelForContainsAndInside
  template <bool ForInside>
  static VGB_HD void contains_inside(const ConeP &c, const V3<R> &p, bool &cin, bool &cout) {
    const R tol = (R)kTolerance;
    const R absz = fabs(p.z);
    cout = absz > (ForInside ? (R)c.dz + (R)kHalfTolerance : (R)c.dz);
    if (ForInside) cin = absz < (R)c.dz - (R)kHalfTolerance;
    const R r2 = p.x * p.x + p.y * p.y;
    const R rmax = (R)c.outerSlope * p.z + (R)c.outerOffset;
    const R rmax2 = rmax * rmax;
    cout |= r2 > (ForInside ? rmax2 + tol * rmax : rmax2);
    if (ForInside) cin &= r2 < rmax2 - tol * rmax;
    if (c.has_rmin) {
      const R rmin = (R)c.innerSlope * p.z + (R)c.innerOffset;
      const R rmin2 = rmin * rmin;
      cout |= r2 <= (ForInside ? rmin2 - tol * rmin : rmin2);
      if (ForInside) cin &= r2 > rmin2 + tol * rmin;
    }
    if (c.has_phi) {
      bool wi, wo;
      W::template contains_inside<ForInside>(c.wedge, p.x, p.y, wi, wo);
      cout |= wo;
      if (ForInside) cin &= wi;
    }
  }

  static VGB_HD bool contains(const ConeP &c, const V3<R> &p) {
    bool ci, co;
    contains_inside<false>(c, p, ci, co);
    return !co;
  }

  static VGB_HD int inside(const ConeP &c, const V3<R> &p) {
    bool ci, co;
    contains_inside<true>(c, p, ci, co);
    return ci ? kInside : (co ? kOutside : kSurface);
  }

  // cosPsi = (x*cosCPhi + y*sinCPhi) / den  >=  limit
  static VGB_HD bool phi_ok(const ConeP &c, R x, R y, R den, double limit) {
    const R cosPsi = (x * (R)c.cosCPhi + y * (R)c.sinCPhi) / den;
    return cosPsi >= (R)limit;
  }

  // The two roots of t^2 + 2 b t + cc = 0 (d = b^2 - cc) in the forms the USolids
  // code writes at every use: lo = -b - sqrt(d), written cc / (-b + sqrt(d)) when
  // b <= 0; hi = -b + sqrt(d), written cc / (-b - sqrt(d)) when b > 0.  One square
  // root and one division serve both, so DistanceToOut, which takes the near root and
  // then, where that one is behind or off the cone, the far one, pays one division
  // with its lanes together (48 k against 38 k Mpoints/s measured).  DistanceToIn keeps
  // each branch's own expression: evaluating both roots ahead of its case split, where
  // most lanes need no division, measured 9 % slower.  NaN when d < 0 (used under d >= 0).
  struct Roots { R lo, hi, sq; };
  static VGB_HD Roots roots(R b, R cc, R d) {
    const R sq = sqrt(d);
    const R den = b > 0 ? -b - sq : -b + sq;
    const R q = cc / den;
    return b > 0 ? Roots{den, q, sq} : Roots{q, den, sq};
  }

  // normal of the inner cone at (x, y) dotted with v <= 0 (:620-630 and copies)
  static VGB_HD bool inner_normal_ok(const ConeP &c, R xi, R yi, const V3<R> &v) {
    const R risec = sqrt(xi * xi + yi * yi) * (R)c.secRMin;
    const R nx = -xi / risec, ny = -yi / risec, nz = (R)c.tanRMin / (R)c.secRMin;
    return nx * v.x + ny * v.y + nz * v.z <= 0;
  }

  // :237-1060 DistanceToInUSolids (p, v already in the cone frame)
  static VGB_HD R distance_to_in(const ConeP &c, const V3<R> &p, const V3<R> &v, R /*smax*/) {
    const R inf = Lim<R>::inf();
    R snxt = inf;
    R sd, xi, yi, zi, ri, rhoi2, b, cc, d;
    const R rMinAv = ((R)c.rmin1 + (R)c.rmin2) * (R)0.5;
    const R rMinOAv = rMinAv > (R)kHalfRadTol ? rMinAv - (R)kHalfRadTol : (R)0.0;
    const R rMaxAv = ((R)c.rmax1 + (R)c.rmax2) * (R)0.5;
    const R rMaxOAv = rMaxAv + (R)kHalfRadTol;
    const R tolIDz = (R)c.dz - (R)kHalfCarTol;
    const R tolODz = (R)c.dz + (R)kHalfCarTol;

    // z faces (:285-355)
    if (fabs(p.z) >= tolIDz) {
      if (p.z * v.z < 0) {
        sd = (fabs(p.z) - (R)c.dz) / fabs(v.z);
        if (sd < (R)0.0) sd = (R)0.0;
        xi = p.x + sd * v.x;
        yi = p.y + sd * v.y;
        rhoi2 = xi * xi + yi * yi;
        R tolORMin, tolIRMin, tolIRMax, tolORMax2, tolORMin2, tolIRMin2, tolIRMax2;
        if (v.z > 0) {
          tolORMin = (R)c.rmin1 - (R)kHalfRadTol * (R)c.secRMin;
          tolIRMin = (R)c.rmin1 + (R)kHalfRadTol * (R)c.secRMin;
          tolIRMax = (R)c.rmax1 - (R)kHalfRadTol * (R)c.secRMin;
          tolORMax2 = ((R)c.rmax1 + (R)kHalfRadTol * (R)c.secRMax) *
                      ((R)c.rmax1 + (R)kHalfRadTol * (R)c.secRMax);
        } else {
          tolORMin = (R)c.rmin2 - (R)kHalfRadTol * (R)c.secRMin;
          tolIRMin = (R)c.rmin2 + (R)kHalfRadTol * (R)c.secRMin;
          tolIRMax = (R)c.rmax2 - (R)kHalfRadTol * (R)c.secRMin;
          tolORMax2 = ((R)c.rmax2 + (R)kHalfRadTol * (R)c.secRMax) *
                      ((R)c.rmax2 + (R)kHalfRadTol * (R)c.secRMax);
        }
        (void)tolORMax2;
        if (tolORMin > 0) {
          tolORMin2 = tolORMin * tolORMin;
          tolIRMin2 = tolIRMin * tolIRMin;
        } else {
          tolORMin2 = (R)0.0;
          tolIRMin2 = (R)0.0;
        }
        (void)tolORMin2;
        tolIRMax2 = tolIRMax > 0 ? tolIRMax * tolIRMax : (R)0.0;
        if ((tolIRMin2 <= rhoi2) && (rhoi2 <= tolIRMax2)) {
          if (!c.full_phi && rhoi2 != 0) {
            if (phi_ok(c, xi, yi, sqrt(rhoi2), c.cosHDPhiIT)) return sd;
          } else {
            return sd;
          }
        }
      } else {
        return snxt;
      }
    }

    // outer cone (:380-505)
    const R t1 = (R)1.0 - v.z * v.z;
    const R t2 = p.x * v.x + p.y * v.y;
    const R t3 = p.x * p.x + p.y * p.y;
    const R rin = (R)c.tanRMin * p.z + rMinAv;
    const R rout = (R)c.tanRMax * p.z + rMaxAv;
    R nt1 = t1 - ((R)c.tanRMax * v.z) * ((R)c.tanRMax * v.z);
    R nt2 = t2 - (R)c.tanRMax * v.z * rout;
    R nt3 = t3 - rout * rout;

    if (fabs(nt1) > (R)kRadTolerance) {
      b = nt2 / nt1;
      cc = nt3 / nt1;
      d = b * b - cc;
      if ((nt3 > rout * rout * (R)kRadTolerance * (R)kRadTolerance * (R)c.secRMax * (R)c.secRMax) ||
          (rout < 0)) {
        if (d >= 0) {
          if ((rout < 0) && (nt3 <= 0)) {
            if (b > 0)
              sd = cc / (-b - sqrt(d));
            else
              sd = -b + sqrt(d);
          } else {
            if ((b <= 0) && (cc >= 0)) {
              sd = cc / (-b + sqrt(d));
            } else {
              if (cc <= 0)
                sd = -b + sqrt(d);
              else
                return inf;
            }
          }
          if (sd > 0) {
            zi = p.z + sd * v.z;
            if (fabs(zi) <= tolODz) {
              if (c.full_phi) return sd;
              xi = p.x + sd * v.x;
              yi = p.y + sd * v.y;
              ri = rMaxAv + zi * (R)c.tanRMax;
              if (phi_ok(c, xi, yi, ri, c.cosHDPhiIT)) return sd;
            }
          }
        }
      } else {
        // inside outer cone: on the surface heading in gives 0 (:472-502)
        if ((t3 > (rin + (R)kHalfRadTol * (R)c.secRMin) * (rin + (R)kHalfRadTol * (R)c.secRMin)) &&
            (nt2 < 0) && (d >= 0) && (fabs(p.z) <= tolIDz)) {
          const R risec = sqrt(p.x * p.x + p.y * p.y) * (R)c.secRMax;
          const R nx = p.x / risec, ny = p.y / risec, nz = -(R)c.tanRMax / (R)c.secRMax;
          const bool heading_in = nx * v.x + ny * v.y + nz * v.z <= 0;
          if (!c.full_phi) {
            if (phi_ok(c, p.x, p.y, sqrt(t3), c.cosHDPhiIT) && heading_in) return (R)0.0;
          } else if (heading_in) {
            return (R)0.0;
          }
        }
      }
    } else {
      // single root (:518-557)
      if (fabs(nt2) > (R)kRadTolerance) {
        sd = (R)-0.5 * nt3 / nt2;
        if (sd < 0) return inf;
        zi = p.z + sd * v.z;
        if ((fabs(zi) <= tolODz) && (nt2 < 0)) {
          if (c.full_phi) return sd;
          xi = p.x + sd * v.x;
          yi = p.y + sd * v.y;
          ri = rMaxAv + zi * (R)c.tanRMax;
          if (phi_ok(c, xi, yi, ri, c.cosHDPhiIT)) return sd;
        }
      } else {
        sd = inf;
      }
    }

    // inner cone (:567-900)
    if (rMinAv != 0) {
      nt1 = t1 - ((R)c.tanRMin * v.z) * ((R)c.tanRMin * v.z);
      nt2 = t2 - (R)c.tanRMin * v.z * rin;
      nt3 = t3 - rin * rin;
      if (nt1 != 0) {
        if (nt3 > rin * (R)kRadTolerance * (R)c.secRMin) {
          // outside real and imaginary inner cones: 2nd root (:576-650)
          b = nt2 / nt1;
          cc = nt3 / nt1;
          d = b * b - cc;
          if (d >= 0) {
            if (b > 0)
              sd = cc / (-b - sqrt(d));
            else
              sd = -b + sqrt(d);
            if (sd >= 0) {
              zi = p.z + sd * v.z;
              if (fabs(zi) <= tolODz) {
                xi = p.x + sd * v.x;
                yi = p.y + sd * v.y;
                if (!c.full_phi) {
                  ri = rMinAv + zi * (R)c.tanRMin;
                  if (phi_ok(c, xi, yi, ri, c.cosHDPhiIT)) {
                    if (sd > (R)kHalfRadTol) {
                      snxt = sd;
                    } else if (inner_normal_ok(c, xi, yi, v)) {
                      snxt = sd;
                    }
                  }
                } else {
                  if (sd > (R)kHalfRadTol) return sd;
                  if (inner_normal_ok(c, xi, yi, v)) return sd;
                }
              }
            }
          }
        } else if (nt3 < -rin * (R)kRadTolerance * (R)c.secRMin) {
          // within the inner cone radius (:652-806)
          b = nt2 / nt1;
          cc = nt3 / nt1;
          d = b * b - cc;
          if (d >= 0) {
            if (b > 0)
              sd = cc / (-b - sqrt(d));
            else
              sd = -b + sqrt(d);
            zi = p.z + sd * v.z;
            ri = rMinAv + zi * (R)c.tanRMin;
            if (ri > 0) {
              if ((sd >= 0) && (fabs(zi) <= tolODz)) {
                xi = p.x + sd * v.x;
                yi = p.y + sd * v.y;
                if (!c.full_phi) {
                  if (phi_ok(c, xi, yi, ri, c.cosHDPhiOT)) {
                    if (sd > (R)kHalfRadTol) {
                      snxt = sd;
                    } else if (inner_normal_ok(c, xi, yi, v)) {
                      snxt = sd;
                    }
                  }
                } else {
                  if (sd > (R)kHalfRadTol) return sd;
                  if (inner_normal_ok(c, xi, yi, v)) return sd;
                }
              }
            } else {
              if (b > 0)
                sd = -b - sqrt(d);
              else
                sd = cc / (-b + sqrt(d));
              zi = p.z + sd * v.z;
              ri = rMinAv + zi * (R)c.tanRMin;
              if ((sd >= 0) && (ri > 0) && (fabs(zi) <= tolODz)) {
                xi = p.x + sd * v.x;
                yi = p.y + sd * v.y;
                if (!c.full_phi) {
                  if (phi_ok(c, xi, yi, ri, c.cosHDPhiIT)) {
                    if (sd > (R)kHalfRadTol) {
                      snxt = sd;
                    } else if (inner_normal_ok(c, xi, yi, v)) {
                      snxt = sd;
                    }
                  }
                } else {
                  if (sd > (R)kHalfRadTol) return sd;
                  if (inner_normal_ok(c, xi, yi, v)) return sd;
                }
              }
            }
          }
        } else {
          // within tolerance of the inner cone (:810-898)
          if (fabs(p.z) <= tolODz) {
            if (nt2 > 0) {
              if (!c.full_phi) {
                if (phi_ok(c, p.x, p.y, sqrt(t3), c.cosHDPhiIT)) return (R)0.0;
              } else {
                return (R)0.0;
              }
            } else {
              b = nt2 / nt1;
              cc = nt3 / nt1;
              d = b * b - cc;
              if (d >= 0) {
                if (b > 0)
                  sd = -b - sqrt(d);
                else
                  sd = cc / (-b + sqrt(d));
                zi = p.z + sd * v.z;
                ri = rMinAv + zi * (R)c.tanRMin;
                if (ri > 0) {
                  if (b > 0)
                    sd = cc / (-b - sqrt(d));
                  else
                    sd = -b + sqrt(d);
                  zi = p.z + sd * v.z;
                  if ((sd >= 0) && (fabs(zi) <= tolODz)) {
                    if (!c.full_phi) {
                      xi = p.x + sd * v.x;
                      yi = p.y + sd * v.y;
                      ri = rMinAv + zi * (R)c.tanRMin;
                      if (phi_ok(c, xi, yi, ri, c.cosHDPhiIT)) snxt = sd;
                    } else {
                      return sd;
                    }
                  }
                } else {
                  return inf;
                }
              }
            }
          } else {
            b = nt2 / nt1;
            cc = nt3 / nt1;
            d = b * b - cc;
            if (d > 0) {
              if (b > 0)
                sd = cc / (-b - sqrt(d));
              else
                sd = -b + sqrt(d);
              zi = p.z + sd * v.z;
              if ((sd >= 0) && (fabs(zi) <= tolODz)) {
                if (!c.full_phi) {
                  xi = p.x + sd * v.x;
                  yi = p.y + sd * v.y;
                  ri = rMinAv + zi * (R)c.tanRMin;
                  if (phi_ok(c, xi, yi, ri, c.cosHDPhiIT)) snxt = sd;
                } else {
                  return sd;
                }
              }
            }
          }
        }
      }
    }

    // phi planes (:904-1052)
    if (!c.full_phi) {
      R comp = v.x * (R)c.sinSPhi - v.y * (R)c.cosSPhi;
      if (comp < 0) {
        const R dist = (p.y * (R)c.cosSPhi - p.x * (R)c.sinSPhi);
        if (dist < (R)kHalfCarTol) {
          sd = dist / comp;
          if (sd < snxt) {
            if (sd < 0) sd = (R)0.0;
            zi = p.z + sd * v.z;
            if (fabs(zi) <= tolODz) {
              xi = p.x + sd * v.x;
              yi = p.y + sd * v.y;
              rhoi2 = xi * xi + yi * yi;
              const R lo = (rMinOAv + zi * (R)c.tanRMin) * (rMinOAv + zi * (R)c.tanRMin);
              const R hi = (rMaxOAv + zi * (R)c.tanRMax) * (rMaxOAv + zi * (R)c.tanRMax);
              if ((rhoi2 >= lo) && (rhoi2 <= hi)) {
                if ((yi * (R)c.cosCPhi - xi * (R)c.sinCPhi) <= 0) snxt = sd;
              }
            }
          }
        }
      }
      comp = -(v.x * (R)c.sinEPhi - v.y * (R)c.cosEPhi);
      if (comp < 0) {
        const R dist = -(p.y * (R)c.cosEPhi - p.x * (R)c.sinEPhi);
        if (dist < (R)kHalfCarTol) {
          sd = dist / comp;
          if (sd < snxt) {
            if (sd < 0) sd = (R)0.0;
            zi = p.z + sd * v.z;
            if (fabs(zi) <= tolODz) {
              xi = p.x + sd * v.x;
              yi = p.y + sd * v.y;
              rhoi2 = xi * xi + yi * yi;
              const R lo = (rMinOAv + zi * (R)c.tanRMin) * (rMinOAv + zi * (R)c.tanRMin);
              const R hi = (rMaxOAv + zi * (R)c.tanRMax) * (rMaxOAv + zi * (R)c.tanRMax);
              if ((rhoi2 >= lo) && (rhoi2 <= hi)) {
                if ((yi * (R)c.cosCPhi - xi * (R)c.sinCPhi) >= (R)0.0) snxt = sd;
              }
            }
          }
        }
      }
    }
    if (snxt < (R)kHalfCarTol) snxt = (R)0.;
    return snxt;
  }

  // :1221-1794 DistanceToOutUSOLIDS
  static VGB_HD R distance_to_out(const ConeP &c, const V3<R> &p, const V3<R> &v, R /*smax*/) {
    const R inf = Lim<R>::inf();
    R snxt, srd, sphi, pdist, b, cc, d, sr2, sr3, zi, ri, deltaRoi2, xi, yi;

    // z planes (:1251-1284)
    if (v.z > (R)0.0) {
      pdist = (R)c.dz - p.z;
      if (pdist > (R)kHalfCarTol)
        snxt = pdist / v.z;
      else
        return (R)0.0;
    } else if (v.z < (R)0.0) {
      pdist = (R)c.dz + p.z;
      if (pdist > (R)kHalfCarTol)
        snxt = -pdist / v.z;
      else
        return (R)0.0;
    } else {
      snxt = inf;
    }

    // outer cone (:1301-1425)
    const R rMaxAv = ((R)c.rmax1 + (R)c.rmax2) * (R)0.5;
    const R t1 = (R)1.0 - v.z * v.z;
    const R t2 = p.x * v.x + p.y * v.y;
    const R t3 = p.x * p.x + p.y * p.y;
    const R rout = (R)c.tanRMax * p.z + rMaxAv;
    R nt1 = t1 - ((R)c.tanRMax * v.z) * ((R)c.tanRMax * v.z);
    R nt2 = t2 - (R)c.tanRMax * v.z * rout;
    R nt3 = t3 - rout * rout;
    if (v.z > (R)0.0)
      deltaRoi2 = snxt * snxt * t1 + (R)2 * snxt * t2 + t3 -
                  (R)c.rmax2 * ((R)c.rmax2 + (R)kRadTolerance * (R)c.secRMax);
    else if (v.z < (R)0.0)
      deltaRoi2 = snxt * snxt * t1 + (R)2 * snxt * t2 + t3 -
                  (R)c.rmax1 * ((R)c.rmax1 + (R)kRadTolerance * (R)c.secRMax);
    else
      deltaRoi2 = (R)1.0;

    if (nt1 != 0 && (deltaRoi2 > (R)0.0)) {
      b = nt2 / nt1;
      cc = nt3 / nt1;
      d = b * b - cc;
      if (d >= 0) {
        if (nt3 > -(R)kHalfRadTol && nt2 >= 0) return (R)0;
        const Roots r = roots(b, cc, d);
        srd = r.lo;
        zi = p.z + srd * v.z;
        ri = (R)c.tanRMax * zi + rMaxAv;
        if ((ri < 0) || (srd < (R)kHalfRadTol)) {
          sr2 = r.hi;
          zi = p.z + sr2 * v.z;
          ri = (R)c.tanRMax * zi + rMaxAv;
          if ((ri >= 0) && (sr2 > (R)kHalfRadTol))
            srd = sr2;
          else
            srd = inf;
        }
      } else {
        return (R)0.0;
      }
    } else if (nt2 != 0 && (deltaRoi2 > (R)0.0)) {
      return (R)0.0;
    } else {
      srd = inf;
    }

    // inner cone (:1465-1560)
    if (c.rmin1 != 0 || c.rmin2 != 0) {
      nt1 = t1 - ((R)c.tanRMin * v.z) * ((R)c.tanRMin * v.z);
      if (nt1 != 0) {
        const R rMinAv = ((R)c.rmin1 + (R)c.rmin2) * (R)0.5;
        const R rin = (R)c.tanRMin * p.z + rMinAv;
        nt2 = t2 - (R)c.tanRMin * v.z * rin;
        nt3 = t3 - rin * rin;
        b = nt2 / nt1;
        cc = nt3 / nt1;
        d = b * b - cc;
        if (d >= (R)0.0) {
          if (nt3 < (R)kRadTolerance * (rin + (R)kRadTolerance * (R)0.25)) {
            if (nt2 < (R)0.0) return (R)0.0;
          } else {
            const Roots r = roots(b, cc, d);
            sr2 = r.lo;
            zi = p.z + sr2 * v.z;
            ri = (R)c.tanRMin * zi + rMinAv;
            if ((ri < 0) || (sr2 < (R)kHalfRadTol)) {
              sr3 = r.hi;
              if (sr3 > (R)kHalfRadTol) {
                if (sr3 < srd) {
                  zi = p.z + sr3 * v.z;
                  ri = (R)c.tanRMin * zi + rMinAv;
                  if (ri >= (R)0.0) srd = sr3;
                }
              }
            } else if ((sr2 < srd) && (sr2 > (R)kHalfCarTol)) {
              srd = sr2;
            }
          }
        }
      }
    }

    // phi planes (:1592-1740)
    if (!c.full_phi) {
      R vphi = atan2(v.y, v.x);
      if (vphi < (R)c.sphi - (R)kHalfAngTol)
        vphi += (R)2 * (R)kPi;
      else if (vphi > (R)c.sphi + (R)c.dphi + (R)kHalfAngTol)
        vphi -= (R)2 * (R)kPi;
      const bool vphi_in = ((R)c.sphi - (R)kHalfAngTol <= vphi) &&
                           ((R)c.sphi + (R)c.dphi + (R)kHalfAngTol >= vphi);
      if (p.x != 0 || p.y != 0) {
        const R pDistS = p.x * (R)c.sinSPhi - p.y * (R)c.cosSPhi;
        const R pDistE = -p.x * (R)c.sinEPhi + p.y * (R)c.cosEPhi;
        const R compS = -(R)c.sinSPhi * v.x + (R)c.cosSPhi * v.y;
        const R compE = (R)c.sinEPhi * v.x - (R)c.cosEPhi * v.y;
        const R hct = (R)kHalfCarTol;
        if (((c.dphi <= kPi) && ((pDistS <= hct) && (pDistE <= hct))) ||
            ((c.dphi > kPi) && !((pDistS > hct) && (pDistE > hct)))) {
          if (compS < 0) {
            sphi = pDistS / compS;
            if (sphi >= -hct) {
              xi = p.x + sphi * v.x;
              yi = p.y + sphi * v.y;
              if ((fabs(xi) <= (R)kTolerance) && (fabs(yi) <= (R)kTolerance)) {
                if (vphi_in) sphi = inf;
              } else if ((yi * (R)c.cosCPhi - xi * (R)c.sinCPhi) >= 0) {
                sphi = inf;
              } else if (pDistS > -hct) {
                sphi = (R)0.0;
              }
            } else {
              sphi = inf;
            }
          } else {
            sphi = inf;
          }
          if (compE < 0) {
            const R sphi2 = pDistE / compE;
            if ((sphi2 > -hct) && (sphi2 < sphi)) {
              xi = p.x + sphi2 * v.x;
              yi = p.y + sphi2 * v.y;
              if ((fabs(xi) <= (R)kTolerance) && (fabs(yi) <= (R)kTolerance)) {
                if (!vphi_in) sphi = (pDistE <= -hct) ? sphi2 : (R)0.0;
              } else if (yi * (R)c.cosCPhi - xi * (R)c.sinCPhi >= 0) {
                sphi = (pDistE <= -hct) ? sphi2 : (R)0.0;
              }
            }
          }
        } else {
          sphi = inf;
        }
      } else {
        sphi = vphi_in ? inf : (R)0.0;
      }
      if (sphi < snxt) snxt = sphi;
    }
    if (srd < snxt) snxt = srd;
    if (snxt < (R)kHalfCarTol) snxt = (R)0.;
    return snxt;
  }

  // :1813-1908 SafetyToInUSOLIDS<ForPolycone>
  template <bool ForPolycone = false>
  static VGB_HD R safety_to_in_impl(const ConeP &c, const V3<R> &p) {
    R safe;
    const R rho = sqrt(p.x * p.x + p.y * p.y);
    const R safeZ = fabs(p.z) - (R)c.dz;
    if (c.rmin1 != 0 || c.rmin2 != 0) {
      const R pRMin = (R)c.tanRMin * p.z + ((R)c.rmin1 + (R)c.rmin2) * (R)0.5;
      const R safeR1 = (pRMin - rho) * (R)c.invSecRMin;
      const R pRMax = (R)c.tanRMax * p.z + ((R)c.rmax1 + (R)c.rmax2) * (R)0.5;
      const R safeR2 = (rho - pRMax) * (R)c.invSecRMax;
      safe = safeR1 > safeR2 ? safeR1 : safeR2;
    } else {
      const R pRMax = (R)c.tanRMax * p.z + ((R)c.rmax1 + (R)c.rmax2) * (R)0.5;
      safe = (rho - pRMax) * (R)c.invSecRMax;
    }
    if (!ForPolycone && safeZ > safe) safe = safeZ;
    if (!c.full_phi && rho != 0) {
      const R cosPsi = (p.x * (R)c.cosCPhi + p.y * (R)c.sinCPhi);
      if (cosPsi < (R)c.cosHDPhi * rho) {
        R safePhi;
        if ((p.y * (R)c.cosCPhi - p.x * (R)c.sinCPhi) <= (R)0.0)
          safePhi = fabs(p.x * (R)c.sinSPhi - p.y * (R)c.cosSPhi);
        else
          safePhi = fabs(p.x * (R)c.sinEPhi - p.y * (R)c.cosEPhi);
        if (safePhi > safe) safe = safePhi;
      }
    }
    if (safe < (R)0.0) safe = (R)0.0;
    return safe;
  }

  static VGB_HD R safety_to_in(const ConeP &c, const V3<R> &p) { return safety_to_in_impl<false>(c, p); }

  // :1922-1989 SafetyToOutUSOLIDS<ForPolycone>
  template <bool ForPolycone = false>
  static VGB_HD R safety_to_out_impl(const ConeP &c, const V3<R> &p) {
    R safe, safeR1;
    const R rho = sqrt(p.x * p.x + p.y * p.y);
    const R safeZ = (R)c.dz - fabs(p.z);
    if (c.rmin1 != 0 || c.rmin2 != 0) {
      const R pRMin = (R)c.tanRMin * p.z + ((R)c.rmin1 + (R)c.rmin2) * (R)0.5;
      safeR1 = (rho - pRMin) * (R)c.invSecRMin;
    } else {
      safeR1 = Lim<R>::inf();
    }
    const R pRMax = (R)c.tanRMax * p.z + ((R)c.rmax1 + (R)c.rmax2) * (R)0.5;
    const R safeR2 = (pRMax - rho) * (R)c.invSecRMax;
    safe = safeR1 < safeR2 ? safeR1 : safeR2;
    if (!ForPolycone && safeZ < safe) safe = safeZ;
    if (!c.full_phi) {
      R safePhi;
      if ((p.y * (R)c.cosCPhi - p.x * (R)c.sinCPhi) <= 0)
        safePhi = -(p.x * (R)c.sinSPhi - p.y * (R)c.cosSPhi);
      else
        safePhi = (p.x * (R)c.sinEPhi - p.y * (R)c.cosEPhi);
      if (safePhi < safe) safe = safePhi;
    }
    if (safe < 0) safe = 0;
    return safe;
  }

  static VGB_HD R safety_to_out(const ConeP &c, const V3<R> &p) { return safety_to_out_impl<false>(c, p); }
};

}  // namespace vgb
