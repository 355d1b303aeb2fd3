// boolean.cuh -- Boolean subtraction (left minus right) of two placed components.
//
// UnplacedBooleanVolume{op, VPlacedVolume* left, right} (volumes/UnplacedBooleanVolume.h:46-51)
// answers every query through its components' *placed* virtual calls
// (volumes/kernel/BooleanImplementation.h:41-594).  Here a component is a
// {transform, shape type, record offset} entry in the boolean's own record, and
// each call applies the same frame change as the virtual it stands for:
//   Contains / Inside / DistanceToIn / SafetyToIn   point (and direction) moved
//                                                    by the component transform
//   PlacedDistanceToOut                              point and direction moved
//   DistanceToOut / SafetyToOut                      point used as given (the
//                                                    VPlacedVolume local-frame calls)
// Two component dispatchers exist: FixedComp (shape known at compile time, all
// inline; the launch picks it for the common pairs) and AnyComp (a switch over
// the primitive shapes in non-inlined functions, for every other pair).
// Components are primitive shapes; nested booleans are rejected when the
// boolean is created.
#pragma once
#include "box.cuh"
#include "cone.cuh"
#include "polycone.cuh"
#include "polyhedron.cuh"
#include "sphere.cuh"
#include "torus.cuh"
#include "trd.cuh"
#include "tube.cuh"

namespace vgb {

struct BoolComp {
  DXform xf;        // the component placement's transform (specialised codes)
  int32_t type;     // vgb_shape_type of the component
  int32_t rec_off;  // doubles from the boolean record to the component's record
  int32_t pad[2];
};

struct BooleanP {
  int32_t op;  // VGB_BOOL_SUBTRACTION
  int32_t pad;
  const double *base;  // record address, bound at launch (device) or by host callers
  BoolComp left, right;
  // Transform<kGeneric,kGeneric> of the right placement: SafetyToIn moves the
  // point with GetTransformation()->Transform(p) (BooleanImplementation.h:558)
  DXform right_generic;
};

// Rounds of the DistanceToIn loop before it gives up (the reference loop,
// BooleanImplementation.h:480-520, has no bound).  A ray that needs more
// rounds gets NaN.  Every round moves the ray forward by at least 1e-8.
constexpr int kBoolMaxRounds = 4096;

// (type, ops template, parameter record) of the shapes a boolean may combine
#define VGB_FOR_EACH_PRIMITIVE(X)                             \
  X(VGB_SHAPE_BOX, vgb::BoxOps, vgb::BoxP)                    \
  X(VGB_SHAPE_TUBE, vgb::TubeOps, vgb::TubeP)                 \
  X(VGB_SHAPE_CONE, vgb::ConeOps, vgb::ConeP)                 \
  X(VGB_SHAPE_SPHERE, vgb::SphereOps, vgb::SphereP)           \
  X(VGB_SHAPE_TRD, vgb::TrdOps, vgb::TrdP)                    \
  X(VGB_SHAPE_TORUS, vgb::TorusOps, vgb::TorusP)              \
  X(VGB_SHAPE_POLYCONE, vgb::PolyconeOps, vgb::PolyconeP)    \
  X(VGB_SHAPE_POLYHEDRON, vgb::PolyhedronOps, vgb::PolyhedronP)      \
  X(VGB_SHAPE_ORB, vgb::OrbOps, vgb::OrbP)                            \
  X(VGB_SHAPE_PARALLELEPIPED, vgb::ParaOps, vgb::ParaP)               \
  X(VGB_SHAPE_PARABOLOID, vgb::ParaboloidOps, vgb::ParaboloidP)       \
  X(VGB_SHAPE_TRAPEZOID, vgb::TrapezoidOps, vgb::TrapezoidP)

template <class P> VGB_HD P comp_params(const double *rec) {
  return bind_params(*reinterpret_cast<const P *>(rec), rec);
}

// Component whose shape is known at compile time.
template <class Ops, class P> struct FixedComp {
  using R = double;
  static VGB_HD P prm(const BooleanP &b, const BoolComp &c) {
    return comp_params<P>(b.base + c.rec_off);
  }
  static VGB_HD bool contains(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return Ops::contains(prm(b, c), xf_point(c.xf, p));
  }
  static VGB_HD int inside(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return Ops::inside(prm(b, c), xf_point(c.xf, p));
  }
  static VGB_HD R distance_to_in(const BooleanP &b, const BoolComp &c, const V3<R> &p,
                                 const V3<R> &v, R smax) {
    return Ops::distance_to_in(prm(b, c), xf_point(c.xf, p), dti_dir<Ops>(c.xf, v), smax);
  }
  static VGB_HD R distance_to_out(const BooleanP &b, const BoolComp &c, const V3<R> &p,
                                  const V3<R> &v, R smax) {
    return Ops::distance_to_out(prm(b, c), p, v, smax);
  }
  static VGB_HD R placed_distance_to_out(const BooleanP &b, const BoolComp &c, const V3<R> &p,
                                         const V3<R> &v, R smax) {
    return Ops::distance_to_out(prm(b, c), xf_point(c.xf, p), xf_dir(c.xf, v), smax);
  }
  static VGB_HD R safety_to_in(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return Ops::safety_to_in(prm(b, c), xf_point(c.xf, p));
  }
  static VGB_HD R safety_to_out(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return Ops::safety_to_out(prm(b, c), p);
  }
};

// Component of any primitive shape: the frame change is inline, the shape
// arithmetic sits behind one switch per operation.
namespace anycomp {
using R = double;

template <class Ret, class Fn> VGB_HD Ret visit(int type, const double *rec, Fn fn) {
  switch (type) {
#define VGB_VISIT(T, OPS, P) \
  case T: return fn(OPS<double>{}, comp_params<P>(rec));
    VGB_FOR_EACH_PRIMITIVE(VGB_VISIT)
#undef VGB_VISIT
  default: return Ret{};
  }
}
VGB_HD bool dir_as_point(int type) {
  switch (type) {
#define VGB_DAP(T, OPS, P) \
  case T: return DirAsPoint<OPS<double>>::value;
    VGB_FOR_EACH_PRIMITIVE(VGB_DAP)
#undef VGB_DAP
  default: return false;
  }
}
VGB_HD_NOINLINE bool contains(int type, const double *rec, V3<R> l) {
  return visit<bool>(type, rec, [&](auto o, const auto &p) { return decltype(o)::contains(p, l); });
}
VGB_HD_NOINLINE int inside(int type, const double *rec, V3<R> l) {
  return visit<int>(type, rec, [&](auto o, const auto &p) { return decltype(o)::inside(p, l); });
}
VGB_HD_NOINLINE R distance_to_in(int type, const double *rec, V3<R> l, V3<R> d, R smax) {
  return visit<R>(type, rec, [&](auto o, const auto &p) {
    return decltype(o)::distance_to_in(p, l, d, smax);
  });
}
VGB_HD_NOINLINE R distance_to_out(int type, const double *rec, V3<R> l, V3<R> d, R smax) {
  return visit<R>(type, rec, [&](auto o, const auto &p) {
    return decltype(o)::distance_to_out(p, l, d, smax);
  });
}
VGB_HD_NOINLINE R safety_to_in(int type, const double *rec, V3<R> l) {
  return visit<R>(type, rec, [&](auto o, const auto &p) { return decltype(o)::safety_to_in(p, l); });
}
VGB_HD_NOINLINE R safety_to_out(int type, const double *rec, V3<R> l) {
  return visit<R>(type, rec,
                  [&](auto o, const auto &p) { return decltype(o)::safety_to_out(p, l); });
}
}  // namespace anycomp

struct AnyComp {
  using R = double;
  static VGB_HD const double *rec(const BooleanP &b, const BoolComp &c) { return b.base + c.rec_off; }
  static VGB_HD bool contains(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return anycomp::contains(c.type, rec(b, c), xf_point(c.xf, p));
  }
  static VGB_HD int inside(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return anycomp::inside(c.type, rec(b, c), xf_point(c.xf, p));
  }
  static VGB_HD R distance_to_in(const BooleanP &b, const BoolComp &c, const V3<R> &p,
                                 const V3<R> &v, R smax) {
    const V3<R> d = anycomp::dir_as_point(c.type) ? xf_point(c.xf, v) : xf_dir(c.xf, v);
    return anycomp::distance_to_in(c.type, rec(b, c), xf_point(c.xf, p), d, smax);
  }
  static VGB_HD R distance_to_out(const BooleanP &b, const BoolComp &c, const V3<R> &p,
                                  const V3<R> &v, R smax) {
    return anycomp::distance_to_out(c.type, rec(b, c), p, v, smax);
  }
  static VGB_HD R placed_distance_to_out(const BooleanP &b, const BoolComp &c, const V3<R> &p,
                                         const V3<R> &v, R smax) {
    return anycomp::distance_to_out(c.type, rec(b, c), xf_point(c.xf, p), xf_dir(c.xf, v), smax);
  }
  static VGB_HD R safety_to_in(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return anycomp::safety_to_in(c.type, rec(b, c), xf_point(c.xf, p));
  }
  static VGB_HD R safety_to_out(const BooleanP &b, const BoolComp &c, const V3<R> &p) {
    return anycomp::safety_to_out(c.type, rec(b, c), p);
  }
};

// The three boolean operations: BooleanImplementation<kSubtraction>
// (volumes/kernel/BooleanImplementation.h:41-594), <kUnion>
// (BooleanUnionImplementation.h:240-470) and <kIntersection>
// (BooleanIntersectionImplementation.h:235-420), chosen by the record's op (the
// reference specialises the placed volume on it,
// source/UnplacedBooleanVolume.cpp:36-62).  Double precision only: the
// components are the FP64 shape kernels.  Every loop the reference leaves
// unbounded stops after kBoolMaxRounds rounds and returns NaN.
template <class R, class LC = AnyComp, class RC = AnyComp> struct BoolOps {
  static_assert(std::is_same<R, double>::value, "boolean components run in double");

  // ---- subtraction ----

  // ContainsKernel (:298-314)
  static VGB_HD bool sub_contains(const BooleanP &b, const V3<R> &p) {
    if (!LC::contains(b, b.left, p)) return false;
    return !RC::contains(b, b.right, p);
  }

  // InsideKernel (:319-362)
  static VGB_HD int sub_inside(const BooleanP &b, const V3<R> &p) {
    const int a = LC::inside(b, b.left, p);
    if (a == kOutside) return kOutside;
    const int bb = RC::inside(b, b.right, p);
    if (a == kInside && bb == kOutside) return kInside;
    if ((a == kInside && bb == kSurface) || (bb == kOutside && a == kSurface)) return kSurface;
    return kOutside;
  }

  // DistanceToInKernel (:368-521): hop between the right component's exit and
  // the left component's entry, pushing 1e-8 across each boundary.
  static VGB_HD R sub_distance_to_in(const BooleanP &b, const V3<R> &p, const V3<R> &v, R smax) {
    const R inf = Lim<R>::inf();
    R d1, d2, snxt = 0.;
    V3<R> hit = p;
    bool insideRight = RC::contains(b, b.right, p);
    R epsil = 0.;
    for (int round = 0; round < kBoolMaxRounds; ++round) {
      if (insideRight) {
        d1 = RC::placed_distance_to_out(b, b.right, hit, v, smax);
        const bool fin = d1 > 0. && d1 < inf;
        snxt += fin ? d1 + epsil : (R)0.;
        const R s = fin ? d1 + (R)1E-8 : (R)1E-8;
        hit = {hit.x + s * v.x, hit.y + s * v.y, hit.z + s * v.z};
        epsil = (R)1.E-8;
        if (LC::contains(b, b.left, hit)) return snxt;
      }
      d2 = LC::distance_to_in(b, b.left, hit, v, smax);
      if (d2 == inf) return inf;
      d1 = RC::distance_to_in(b, b.right, hit, v, smax);
      if (d2 < d1 - (R)kTolerance) {
        snxt += d2 + epsil;
        return snxt;
      }
      const bool fin = d1 > 0. && d1 < inf;
      snxt += fin ? d1 + epsil : (R)0.;
      const R s = fin ? d1 + epsil : epsil;
      hit = {hit.x + s * v.x, hit.y + s * v.y, hit.z + s * v.z};
      insideRight = true;
    }
    return Lim<R>::quiet_nan();
  }

  // DistanceToOutKernel (:526-539)
  static VGB_HD R sub_distance_to_out(const BooleanP &b, const V3<R> &p, const V3<R> &v, R smax) {
    const R d = LC::distance_to_out(b, b.left, p, v, smax);
    const R dinright = RC::distance_to_in(b, b.right, p, v, smax);
    return vmin(d, dinright);
  }

  // SafetyToInKernel (:544-576)
  static VGB_HD R sub_safety_to_in(const BooleanP &b, const V3<R> &p) {
    if (LC::contains(b, b.left, p) && RC::contains(b, b.right, p))
      return RC::safety_to_out(b, b.right, xf_point(b.right_generic, p));
    return LC::safety_to_in(b, b.left, p);
  }

  // SafetyToOutKernel (:581-594)
  static VGB_HD R sub_safety_to_out(const BooleanP &b, const V3<R> &p) {
    const R s = LC::safety_to_out(b, b.left, p);
    const R sr = RC::safety_to_in(b, b.right, p);
    return vmin(s, sr);
  }
  // ---- union ----
  // ContainsKernel (BooleanUnionImplementation.h:240-248)
  static VGB_HD bool uni_contains(const BooleanP &b, const V3<R> &p) {
    if (LC::contains(b, b.left, p)) return true;
    return RC::contains(b, b.right, p);
  }
  // InsideKernel (:250-290)
  static VGB_HD int uni_inside(const BooleanP &b, const V3<R> &p) {
    const int a = LC::inside(b, b.left, p);
    if (a == kInside) return kInside;
    const int bb = RC::inside(b, b.right, p);
    if (bb == kInside) return kInside;
    if (bb == kSurface || a == kSurface) return kSurface;
    return kOutside;
  }
  // DistanceToInKernel (:292-305)
  static VGB_HD R uni_distance_to_in(const BooleanP &b, const V3<R> &p, const V3<R> &v, R smax) {
    const R d1 = LC::distance_to_in(b, b.left, p, v, smax);
    const R d2 = RC::distance_to_in(b, b.right, p, v, smax);
    return vmin(d1, d2);
  }
  // DistanceToOutKernel (:307-345): walk out of the component holding the
  // point and through the other wherever it continues, one kTolerance push per
  // round (taken back at the end)
  static VGB_HD R uni_distance_to_out(const BooleanP &b, const V3<R> &p, const V3<R> &v, R) {
    const R inf = Lim<R>::inf();
    R dist = 0., disTmp = 0.;
    int push = 0;
    auto at = [&](R t) { return V3<R>{p.x + t * v.x, p.y + t * v.y, p.z + t * v.z}; };
    if (LC::contains(b, b.left, p)) {
      for (;;) {
        if (push >= kBoolMaxRounds) return Lim<R>::quiet_nan();
        disTmp = LC::distance_to_out(b, b.left, at(dist), v, inf);
        dist += (disTmp >= 0. && disTmp < inf) ? disTmp : (R)0;
        dist += (R)kTolerance;
        ++push;
        if (RC::contains(b, b.right, at(dist))) {
          disTmp = RC::placed_distance_to_out(b, b.right, at(dist), v, inf);
          dist += (disTmp >= 0. && disTmp < inf) ? disTmp : (R)0;
        }
        if (!LC::contains(b, b.left, at(dist))) break;
      }
    } else {
      for (;;) {
        if (push >= kBoolMaxRounds) return Lim<R>::quiet_nan();
        disTmp = RC::placed_distance_to_out(b, b.right, at(dist), v, inf);
        dist += (disTmp >= 0. && disTmp < inf) ? disTmp : (R)0.;
        dist += (R)kTolerance;
        ++push;
        if (LC::contains(b, b.left, at(dist))) {
          disTmp = LC::distance_to_out(b, b.left, at(dist), v, inf);
          dist += disTmp;
        }
        if (!RC::contains(b, b.right, at(dist))) break;
      }
    }
    return dist - push * (R)kTolerance;
  }
  // SafetyToInKernel (:430-441)
  static VGB_HD R uni_safety_to_in(const BooleanP &b, const V3<R> &p) {
    const R distA = LC::safety_to_in(b, b.left, p);
    const R distB = RC::safety_to_in(b, b.right, p);
    const R s = vmin(distA, distB);
    return s < 0 ? (R)0. : s;
  }
  // SafetyToOutKernel (:443-470)
  static VGB_HD R uni_safety_to_out(const BooleanP &b, const V3<R> &p) {
    const bool inA = LC::contains(b, b.left, p);
    const bool inB = RC::contains(b, b.right, p);
    if (inA && inB)
      return vmax(LC::safety_to_out(b, b.left, p),
                  RC::safety_to_out(b, b.right, xf_point(b.right_generic, p)));
    if (inB) return RC::safety_to_out(b, b.right, xf_point(b.right_generic, p));
    return LC::safety_to_out(b, b.left, p);
  }

  // ---- intersection ----
  // ContainsKernel (BooleanIntersectionImplementation.h:235-244)
  static VGB_HD bool int_contains(const BooleanP &b, const V3<R> &p) {
    const bool a = LC::contains(b, b.left, p);
    const bool c = RC::contains(b, b.right, p);
    return a && c;
  }
  // InsideKernel (:246-275)
  static VGB_HD int int_inside(const BooleanP &b, const V3<R> &p) {
    const int a = LC::inside(b, b.left, p);
    if (a == kOutside) return kOutside;
    const int bb = RC::inside(b, b.right, p);
    if (a == kInside && bb == kInside) return kInside;
    if ((a == kInside && bb == kSurface) || (bb == kInside && a == kSurface) ||
        (a == kSurface && bb == kSurface))
      return kSurface;
    return kOutside;
  }
  // DistanceToInKernel (:277-335): advance to the farther of the two entries
  // until the point is in both
  static VGB_HD R int_distance_to_in(const BooleanP &b, const V3<R> &p, const V3<R> &v, R smax) {
    const R inf = Lim<R>::inf();
    V3<R> hit = p;
    bool inleft = LC::contains(b, b.left, hit);
    bool inright = RC::contains(b, b.right, hit);
    R d1 = 0., d2 = 0., snext = 0.;
    if (inleft && inright) {
      d1 = LC::placed_distance_to_out(b, b.left, hit, v, smax);
      d2 = RC::placed_distance_to_out(b, b.right, hit, v, smax);
      if (d1 < 2 * (R)kTolerance) inleft = false;
      if (d2 < 2 * (R)kTolerance) inright = false;
      if (inleft && inright) return (R)0.;
    }
    for (int round = 0; round < kBoolMaxRounds; ++round) {
      d1 = d2 = 0;
      if (!inleft) {
        d1 = LC::distance_to_in(b, b.left, hit, v, inf);
        d1 = vmax(d1, (R)kTolerance);
        if (d1 > (R)1E20) return inf;
      }
      if (!inright) {
        d2 = RC::distance_to_in(b, b.right, hit, v, inf);
        d2 = vmax(d2, (R)kTolerance);
        if (d2 > (R)1E20) return inf;
      }
      if (d1 > d2) {
        snext += d1;
        inleft = true;
        hit = {hit.x + d1 * v.x, hit.y + d1 * v.y, hit.z + d1 * v.z};
        const R t = (R)kTolerance;
        inright = RC::contains(b, b.right, {hit.x + t * v.x, hit.y + t * v.y, hit.z + t * v.z});
        if (inright) return snext;
      } else {
        snext += d2;
        inright = true;
        hit = {hit.x + d2 * v.x, hit.y + d2 * v.y, hit.z + d2 * v.z};
        const R t = (R)kTolerance;
        inleft = LC::contains(b, b.left, {hit.x + t * v.x, hit.y + t * v.y, hit.z + t * v.z});
        if (inleft) return snext;
      }
    }
    return Lim<R>::quiet_nan();
  }
  // DistanceToOutKernel (:337-346)
  static VGB_HD R int_distance_to_out(const BooleanP &b, const V3<R> &p, const V3<R> &v, R) {
    const R inf = Lim<R>::inf();
    return vmin(LC::distance_to_out(b, b.left, p, v, inf),
                RC::placed_distance_to_out(b, b.right, p, v, inf));
  }
  // SafetyToInKernel (:348-372)
  static VGB_HD R int_safety_to_in(const BooleanP &b, const V3<R> &p) {
    const bool inA = LC::contains(b, b.left, p);
    const bool inB = RC::contains(b, b.right, p);
    if (!inA && inB) return LC::safety_to_in(b, b.left, p);
    if (!inB && inA) return RC::safety_to_in(b, b.right, p);
    return vmin(LC::safety_to_in(b, b.left, p), RC::safety_to_in(b, b.right, p));
  }
  // SafetyToOutKernel (:374-386)
  static VGB_HD R int_safety_to_out(const BooleanP &b, const V3<R> &p) {
    const R s = vmin(LC::safety_to_out(b, b.left, p),
                     RC::safety_to_out(b, b.right, xf_point(b.right_generic, p)));
    return s < 0 ? (R)0. : s;
  }

  // ---- the op of the record ----
  static VGB_HD bool contains(const BooleanP &b, const V3<R> &p) {
    if (b.op == VGB_BOOL_UNION) return uni_contains(b, p);
    if (b.op == VGB_BOOL_INTERSECTION) return int_contains(b, p);
    return sub_contains(b, p);
  }
  static VGB_HD int inside(const BooleanP &b, const V3<R> &p) {
    if (b.op == VGB_BOOL_UNION) return uni_inside(b, p);
    if (b.op == VGB_BOOL_INTERSECTION) return int_inside(b, p);
    return sub_inside(b, p);
  }
  static VGB_HD R distance_to_in(const BooleanP &b, const V3<R> &p, const V3<R> &v, R smax) {
    if (b.op == VGB_BOOL_UNION) return uni_distance_to_in(b, p, v, smax);
    if (b.op == VGB_BOOL_INTERSECTION) return int_distance_to_in(b, p, v, smax);
    return sub_distance_to_in(b, p, v, smax);
  }
  static VGB_HD R distance_to_out(const BooleanP &b, const V3<R> &p, const V3<R> &v, R smax) {
    if (b.op == VGB_BOOL_UNION) return uni_distance_to_out(b, p, v, smax);
    if (b.op == VGB_BOOL_INTERSECTION) return int_distance_to_out(b, p, v, smax);
    return sub_distance_to_out(b, p, v, smax);
  }
  static VGB_HD R safety_to_in(const BooleanP &b, const V3<R> &p) {
    if (b.op == VGB_BOOL_UNION) return uni_safety_to_in(b, p);
    if (b.op == VGB_BOOL_INTERSECTION) return int_safety_to_in(b, p);
    return sub_safety_to_in(b, p);
  }
  static VGB_HD R safety_to_out(const BooleanP &b, const V3<R> &p) {
    if (b.op == VGB_BOOL_UNION) return uni_safety_to_out(b, p);
    if (b.op == VGB_BOOL_INTERSECTION) return int_safety_to_out(b, p);
    return sub_safety_to_out(b, p);
  }
};

// the pairs the launch specialises
template <class R>
using BoolBoxTube = BoolOps<R, FixedComp<BoxOps<double>, BoxP>, FixedComp<TubeOps<double>, TubeP>>;
template <class R>
using BoolBoxBox = BoolOps<R, FixedComp<BoxOps<double>, BoxP>, FixedComp<BoxOps<double>, BoxP>>;

}  // namespace vgb
