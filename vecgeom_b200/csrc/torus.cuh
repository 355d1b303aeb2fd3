// torus.cuh -- Torus shape arithmetic (device), templated on the arithmetic type.
//
// Follows volumes/kernel/TorusImplementation.h: distances solve the quartic of
// the line against the torus with a Ferrari-style complex solver
// (solveQuartic2, :440-504), keep the smallest valid real root, polish it with
// two Newton steps (:743-761, :852-856) and resolve grazing cases with the
// surface normal; DistanceToIn first clips the ray to a bounding tube
// (:889-1036).  Reference behaviours kept for parity:
//  * DistanceToIn transforms the direction with the *point* transform
//    (Transform instead of TransformDirection, :906); the batch kernel applies
//    that through kDirectionAsPoint;
//  * the Newton polish runs only when the last root tested was valid (:851).
// The complex cube root takes atan2, sin, cos and cbrt correctly rounded
// (crmath.cuh), on the host and on the GPU alike: the reference calls the C
// library's functions there, and the last bits of those move its roots, so
// only correctly rounded values make the result independent of the library.
#pragma once
#include "crmath.cuh"
#include "tube.cuh"

namespace vgb {

// UnplacedTorus with its cached values (volumes/UnplacedTorus.h:40-80).
struct TorusP {
  double rmin, rmax, rtor, sphi, dphi;
  double rmin2, rmax2, rtor2;
  WedgeP wedge;
  TubeP btube;  // bounding tube, run as TubeTypes::HollowTube (rmin on, phi off)
  int32_t has_phi;
  int32_t pad;
};

// Complex<T> of TorusImplementation.h:46-300, same operation order.
template <class R> struct Cx {
  R r, i;
};
template <class R> VGB_HD Cx<R> cmul(Cx<R> x, Cx<R> y) {
  return {x.r * y.r - x.i * y.i, x.r * y.i + x.i * y.r};
}
template <class R> VGB_HD Cx<R> cscale(Cx<R> x, R y) { return {x.r * y, x.i * y}; }
template <class R> VGB_HD Cx<R> cdivr(Cx<R> x, R y) {
  const R invy = (R)1. / y;
  return {x.r * invy, x.i * invy};
}
// T / Complex: (x * conj(y)) / (y * conj(y)).real
template <class R> VGB_HD Cx<R> rdivc(R x, Cx<R> y) {
  const Cx<R> yc = {y.r, -y.i};
  const Cx<R> tmp = cmul(y, yc);
  return cdivr(cscale(yc, x), tmp.r);
}
template <class R> VGB_HD Cx<R> csqrt_(Cx<R> x) {
  const R l = sqrt(x.r * x.r + x.i * x.i);
  return {sqrt((R)0.5 * (l + x.r)), sqrt((R)0.5 * (l - x.r))};
}
template <class R> VGB_HD Cx<R> csqrt_real(R x) {
  const R imcoef = (x >= (R)0.) ? (R)0. : (R)1.;
  const R realcoef = (x >= 0) ? (R)1. : (R)0.;
  const R l = sqrt(fabs(x));
  return {realcoef * l, imcoef * l};
}
// cbrt(Complex) (:283-316)
template <class R> VGB_HD Cx<R> ccbrt(Cx<R> x) {
  R rr, s, c;
  if (x.i != (R)0.0) {
    rr = sqrt(x.r * x.r + x.i * x.i);
    const R angle = cr_atan2(x.i, x.r);
    const R newangle = angle / (R)3.;
    cr_sincos(newangle, &s, &c);
  } else {
    rr = x.r;
    s = 0.;
    c = 1.;
  }
  const R rc = cr_cbrt(rr);
  return {rc * c, rc * s};
}

template <class R> struct TorusOps {
  static constexpr bool kDirectionAsPoint = true;
  using W = WedgeOps<R>;
  using T = TubeOps<R>;

  // GenericKernelForContainsAndInside<ForInside, notForDisk> (:580-634)
  template <bool ForInside, bool NotForDisk>
  static VGB_HD void kernel(const TorusP &t, const V3<R> &p, bool &cin, bool &cout) {
    const R tol = (R)kTolerance;
    const R rxy = sqrt(p.x * p.x + p.y * p.y);
    const R radsq = (rxy - (R)t.rtor) * (rxy - (R)t.rtor) + p.z * p.z;
    cout = radsq > (ForInside ? (R)t.rmax2 + tol * (R)t.rmax : (R)t.rmax2);
    if (ForInside) cin = radsq < (R)t.rmax2 - tol * (R)t.rmax;
    cout |= radsq < (ForInside ? (R)t.rmin2 - tol * (R)t.rmin : (R)t.rmin2);
    if (ForInside) cin &= radsq > (R)t.rmin2 + tol * (R)t.rmin;
    if (t.has_phi && NotForDisk) {
      bool wi, wo;
      W::template contains_inside<ForInside>(t.wedge, p.x, p.y, wi, wo);
      cout |= wo;
      if (ForInside) cin &= wi;
    }
  }

  static VGB_HD bool contains(const TorusP &t, const V3<R> &p) {
    bool ci, co;
    kernel<false, true>(t, p, ci, co);
    return !co;
  }
  static VGB_HD bool contains_disk(const TorusP &t, const V3<R> &p) {
    bool ci, co;
    kernel<false, false>(t, p, ci, co);
    return !co;
  }
  static VGB_HD int inside(const TorusP &t, const V3<R> &p) {
    bool ci, co;
    kernel<true, true>(t, p, ci, co);
    return ci ? kInside : (co ? kOutside : kSurface);
  }

  // solveQuartic2 (:440-504) for x^4 + b x^3 + c x^2 + d x + e (a == 1)
  static VGB_HD void quartic(R b, R c, R d, R e, Cx<R> *roots) {
    const R inv256 = (R)(1. / 256), inv16 = (R)(1. / 16), inv3 = (R)(1. / 3);
    const R inv27 = (R)(1. / 27), inv6 = (R)(1. / 6), inv108 = (R)(1. / 108), inv12 = (R)(1. / 12);
    const R bb = b * b;
    const R bbb = bb * b;
    const R alpha = (R)-3.0 * (R)0.125 * bb + c;
    const R beta = (R)0.125 * bbb - (R)0.5 * b * c + d;
    const R alpha2 = alpha * alpha;
    const R gamma = (R)-3.0 * bbb * b * inv256 + c * bb * inv16 - (R)0.25 * b * d + e;
    const R P = -alpha2 * inv12 - gamma;
    const R Q = -alpha2 * alpha * inv108 + alpha * gamma * inv3 - (R)0.125 * beta * beta;
    const R tmp = (R)0.25 * Q * Q + P * P * P * inv27;
    const Cx<R> sq = csqrt_real(tmp);
    const Cx<R> Rr = {sq.r + Q * (R)0.5, sq.i};
    const Cx<R> U = ccbrt(Rr);
    const R y0 = (R)-5.0 * alpha * inv6;
    Cx<R> y = {y0 - U.r, -U.i};
    const Cx<R> q = rdivc(P, cscale(U, (R)3.));
    y = {y.r + q.r, y.i + q.i};
    const Cx<R> ay = {y.r + alpha, y.i};
    const Cx<R> W = csqrt_(Cx<R>{ay.r + y.r, ay.i + y.i});
    const R firstPart = (R)-0.25 * b;
    const Cx<R> secondPart = {(R)-3.0 * alpha - y.r * (R)2.0, -(y.i * (R)2.0)};
    const Cx<R> thirdPart = rdivc((R)2.0 * beta, W);
    const Cx<R> sp = csqrt_(Cx<R>{secondPart.r + thirdPart.r, secondPart.i + thirdPart.i});
    const Cx<R> sm = csqrt_(Cx<R>{secondPart.r - thirdPart.r, secondPart.i - thirdPart.i});
    Cx<R> t0 = {-W.r - sp.r, -W.i - sp.i};
    roots[0] = {cscale(t0, (R)0.5).r + firstPart, cscale(t0, (R)0.5).i};
    t0 = {-W.r + sp.r, -W.i + sp.i};
    roots[1] = {cscale(t0, (R)0.5).r + firstPart, cscale(t0, (R)0.5).i};
    t0 = {W.r - sm.r, W.i - sm.i};
    roots[2] = {cscale(t0, (R)0.5).r + firstPart, cscale(t0, (R)0.5).i};
    t0 = {W.r + sm.r, W.i + sm.i};
    roots[3] = {cscale(t0, (R)0.5).r + firstPart, cscale(t0, (R)0.5).i};
  }

  // CheckZero / NewtonIter (:743-761)
  static VGB_HD R check_zero(R b, R c, R d, R e, R x) {
    const R x2 = x * x;
    return x2 * x2 + b * x2 * x + c * x2 + d * x + e;
  }
  static VGB_HD R newton(R b, R c, R d, R e, R x, R fold) {
    (void)e;
    const R x2 = x * x;
    const R fprime = (R)4 * x2 * x + (R)3 * b * x2 + (R)2 * c * x + d;
    return x - fold / fprime;
  }

  // ToBoundary<ForRmin> (:764-887)
  template <bool ForRmin>
  static VGB_HD R to_boundary(const TorusP &t, const V3<R> &p, const V3<R> &v, R radius, bool out) {
    const R inf = Lim<R>::inf();
    const R rtor2 = (R)t.rtor2;
    const R r0sq = p.x * p.x + p.y * p.y + p.z * p.z;
    const R rdotn = p.x * v.x + p.y * v.y + p.z * v.z;
    const R rsumsq = rtor2 + radius * radius;
    const R a = (R)4. * rdotn;
    const R b = (R)2. * (r0sq + (R)2. * rdotn * rdotn - rsumsq + (R)2. * rtor2 * v.z * v.z);
    const R c = (R)4. * (r0sq * rdotn - rsumsq * rdotn + (R)2. * rtor2 * p.z * v.z);
    const R d = r0sq * r0sq - (R)2. * r0sq * rsumsq + (R)4. * rtor2 * p.z * p.z +
                (rtor2 - radius * radius) * (rtor2 - radius * radius);
    Cx<R> roots[4];
    quartic(a, b, c, d, roots);
    R valid = inf, second = inf;
    bool ok = false;
    for (int k = 0; k < 4; ++k) {
      ok = fabs(roots[k].i) < (R)1E-9 && roots[k].r > (R)-1E-9;
      if (t.has_phi && ok) {
        const R rr = roots[k].r;
        ok &= W::contains_with_boundary(t.wedge, p.x + rr * v.x, p.y + rr * v.y);
      }
      if (k == 0) {
        if (ok) valid = roots[0].r;
        if (out && ok) second = valid;
      } else {
        if (ok) valid = vmin(roots[k].r, valid);
        if (out && ok) second = vmax(roots[k].r, valid);
      }
    }
    // the reference polishes only when the last root tested (roots[3]) was
    // valid: havevalidsolution &= (validdistance < kInfinity) (:851)
    if (ok && valid < inf) {
      valid = newton(a, b, c, d, valid, check_zero(a, b, c, d, valid));
      valid = newton(a, b, c, d, valid, check_zero(a, b, c, d, valid));
    }
    if (valid < (R)1E-9) {
      valid = 0.;
      const R rho = sqrt(p.x * p.x + p.y * p.y);
      const R red = (rho - (R)t.rtor) / rho;
      V3<R> n = {p.x * red, p.y * red, p.z};
      if (ForRmin) n = {-n.x, -n.y, -n.z};
      const R dot = v.x * n.x + v.y * n.y + v.z * n.z;
      if (!out && (dot > (R)0.)) valid = second;
      if (out && (dot < (R)0.)) valid = second;
    }
    return valid;
  }

  // Wedge::DistanceToIn (volumes/Wedge.h:292-328)
  static VGB_HD void wedge_dti(const WedgeP &w, const V3<R> &p, const V3<R> &v, R &d1, R &d2) {
    d1 = d2 = Lim<R>::inf();
    const R comp1 = v.x * (R)w.n1x + v.y * (R)w.n1y;
    const R comp2 = v.x * (R)w.n2x + v.y * (R)w.n2y;
    if (comp1 > (R)0.) {
      const R tmp = -(p.x * (R)w.n1x + p.y * (R)w.n1y) / comp1;
      if (tmp > (R)0.) d1 = tmp;
    }
    if (comp2 > (R)0.) {
      const R tmp = -(p.x * (R)w.n2x + p.y * (R)w.n2y) / comp2;
      if (tmp > (R)0.) d2 = tmp;
    }
  }

  // Wedge::DistanceToOut (volumes/Wedge.h:330-366)
  static VGB_HD void wedge_dto(const WedgeP &w, const V3<R> &p, const V3<R> &v, R &d1, R &d2) {
    d1 = d2 = Lim<R>::inf();
    const R comp1 = v.x * (R)w.n1x + v.y * (R)w.n1y;
    const R comp2 = v.x * (R)w.n2x + v.y * (R)w.n2y;
    if (comp1 < (R)0.) {
      const R tmp = -(p.x * (R)w.n1x + p.y * (R)w.n1y) / comp1;
      if (tmp > (R)0.) d1 = tmp;
    }
    if (comp2 < (R)0.) {
      const R tmp = -(p.x * (R)w.n2x + p.y * (R)w.n2y) / comp2;
      if (tmp > (R)0.) d2 = tmp;
    }
  }

  // the phi-plane candidates of DistanceToIn/DistanceToOut (:969-1005, :1066-1100)
  static VGB_HD R phi_candidates(const TorusP &t, const V3<R> &p, const V3<R> &v, R dist, R dphi1,
                                 R dphi2) {
    if (dphi1 < dist) {
      const V3<R> ip = {p.x + v.x * dphi1, p.y + v.y * dphi1, p.z + v.z * dphi1};
      if (contains_disk(t, ip)) {
        const R diri = ip.x * (R)t.wedge.a1x + ip.y * (R)t.wedge.a1y;
        if (diri >= 0) dist = dphi1;
      }
    }
    if (dphi2 < dist) {
      const V3<R> ip = {p.x + v.x * dphi2, p.y + v.y * dphi2, p.z + v.z * dphi2};
      if (contains_disk(t, ip)) {
        const R diri2 = ip.x * (R)t.wedge.a2x + ip.y * (R)t.wedge.a2y;
        if (diri2 >= 0 && dphi2 < dist) dist = dphi2;
      }
    }
    return dist;
  }

  // DistanceToIn (:889-1036); v is the point-transformed direction
  static VGB_HD R distance_to_in(const TorusP &t, const V3<R> &p0, const V3<R> &v, R smax) {
    const R inf = Lim<R>::inf();
    const bool inBounds = T::contains(t.btube, p0);
    const R tubeDistance = T::distance_to_in(t.btube, p0, v, smax);
    const bool done = (!inBounds && tubeDistance == inf);
    if (done) return inf;
    V3<R> p = p0;
    if (!inBounds) p = {p0.x + v.x * tubeDistance, p0.y + v.y * tubeDistance, p0.z + v.z * tubeDistance};
    const R dout = to_boundary<false>(t, p, v, (R)t.rmax, false);
    R din = inf;
    if (t.rmin > 0) din = to_boundary<true>(t, p, v, (R)t.rmin, false);
    R minDist = vmin(dout, din);
    if (t.has_phi) {
      R d1, d2;
      wedge_dti(t.wedge, p, v, d1, d2);
      minDist = phi_candidates(t, p, v, minDist, d1, d2);
    }
    return inBounds ? minDist : minDist + tubeDistance;
  }

  // DistanceToOut (:1038-1110)
  static VGB_HD R distance_to_out(const TorusP &t, const V3<R> &p, const V3<R> &v, R) {
    const R dout = to_boundary<false>(t, p, v, (R)t.rmax, true);
    R din = Lim<R>::inf();
    if (t.rmin > 0) din = to_boundary<true>(t, p, v, (R)t.rmin, true);
    R distance = vmin(dout, din);
    if (t.has_phi) {
      R d1, d2;
      wedge_dto(t.wedge, p, v, d1, d2);
      distance = phi_candidates(t, p, v, distance, d1, d2);
    }
    return distance;
  }

  // SafetyToIn / SafetyToOut (:1112-1170)
  static VGB_HD R safety_to_in(const TorusP &t, const V3<R> &p) {
    const R rxy = sqrt(p.x * p.x + p.y * p.y);
    const R rad = sqrt((rxy - (R)t.rtor) * (rxy - (R)t.rtor) + p.z * p.z);
    R safety = rad - (R)t.rmax;
    if (t.rmin != 0) safety = vmax((R)t.rmin - rad, rad - (R)t.rmax);
    if (t.has_phi && (rxy != (R)0.)) safety = vmax(W::safety_to_in(t.wedge, p.x, p.y), safety);
    return safety;
  }

  static VGB_HD R safety_to_out(const TorusP &t, const V3<R> &p) {
    const R rxy = sqrt(p.x * p.x + p.y * p.y);
    const R rad = sqrt((rxy - (R)t.rtor) * (rxy - (R)t.rtor) + p.z * p.z);
    R safety = (R)t.rmax - rad;
    if (t.rmin != 0) safety = vmin(rad - (R)t.rmin, (R)t.rmax - rad);
    if (t.has_phi) safety = vmin(W::safety_to_out(t.wedge, p.x, p.y), safety);
    return safety;
  }
};

}  // namespace vgb
