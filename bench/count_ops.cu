// count_ops.cu -- measurement infrastructure, NOT product code: the algorithmic
// flops of every shape operation, counted by running the shape arithmetic of
// libvgb (vecgeom_b200/csrc/*.cuh, templated on the arithmetic type and written
// in the reference's operation order) on the host with an op-counting number
// type.  make_op_costs.py averages the counts over the benchmark inputs and
// writes op_costs.json, which bench.py reads to place each kernel on its
// FP64 roofline.
//
// Counting rules: + - * / and sqrt count 1 each; a transcendental (atan2, sin,
// cos, tan, asin, cbrt, fmod, floor, correctly rounded or not) counts 1; comparisons, fabs, negation and
// selects count 0.  The kernels are compiled without contraction, so there is
// no FMA to count as 2.
#include <cmath>
#include <cstdint>
#include <type_traits>

namespace vgbcount {

struct Counts {
  int64_t add, mul, div, sqrt, trans;
};
Counts g_counts = {0, 0, 0, 0, 0};

struct CD {
  double v;
  CD() : v(0) {}
  CD(double x) : v(x) {}  // NOLINT: converts like a double
  CD(int x) : v(x) {}     // NOLINT
  explicit operator double() const { return v; }
  explicit operator float() const { return (float)v; }
  CD &operator+=(CD o) { ++g_counts.add; v += o.v; return *this; }
  CD &operator-=(CD o) { ++g_counts.add; v -= o.v; return *this; }
  CD &operator*=(CD o) { ++g_counts.mul; v *= o.v; return *this; }
  CD &operator/=(CD o) { ++g_counts.div; v /= o.v; return *this; }
};
inline CD operator+(CD a, CD b) { ++g_counts.add; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { ++g_counts.add; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { ++g_counts.mul; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { ++g_counts.div; return CD(a.v / b.v); }
inline CD operator-(CD a) { return CD(-a.v); }
inline CD operator+(CD a) { return a; }
#define VGBCOUNT_CMP(op)                                                   \
  inline bool operator op(CD a, CD b) { return a.v op b.v; }               \
  inline bool operator op(CD a, double b) { return a.v op b; }             \
  inline bool operator op(double a, CD b) { return a op b.v; }             \
  inline bool operator op(CD a, int b) { return a.v op b; }                \
  inline bool operator op(int a, CD b) { return a op b.v; }
VGBCOUNT_CMP(<)
VGBCOUNT_CMP(>)
VGBCOUNT_CMP(<=)
VGBCOUNT_CMP(>=)
VGBCOUNT_CMP(==)
VGBCOUNT_CMP(!=)
#undef VGBCOUNT_CMP
inline CD operator+(CD a, double b) { return a + CD(b); }
inline CD operator+(double a, CD b) { return CD(a) + b; }
inline CD operator-(CD a, double b) { return a - CD(b); }
inline CD operator-(double a, CD b) { return CD(a) - b; }
inline CD operator*(CD a, double b) { return a * CD(b); }
inline CD operator*(double a, CD b) { return CD(a) * b; }
inline CD operator/(CD a, double b) { return a / CD(b); }
inline CD operator/(double a, CD b) { return CD(a) / b; }
inline CD operator+(CD a, int b) { return a + CD(b); }
inline CD operator-(CD a, int b) { return a - CD(b); }
inline CD operator*(CD a, int b) { return a * CD(b); }
inline CD operator*(int a, CD b) { return CD(a) * b; }
inline CD operator/(CD a, int b) { return a / CD(b); }

inline CD sqrt(CD a) { ++g_counts.sqrt; return CD(std::sqrt(a.v)); }
inline CD fabs(CD a) { return CD(std::fabs(a.v)); }
inline CD atan2(CD a, CD b) { ++g_counts.trans; return CD(std::atan2(a.v, b.v)); }
inline CD sin(CD a) { ++g_counts.trans; return CD(std::sin(a.v)); }
inline CD cos(CD a) { ++g_counts.trans; return CD(std::cos(a.v)); }
inline CD tan(CD a) { ++g_counts.trans; return CD(std::tan(a.v)); }
inline CD asin(CD a) { ++g_counts.trans; return CD(std::asin(a.v)); }
inline CD cbrt(CD a) { ++g_counts.trans; return CD(std::cbrt(a.v)); }
inline CD fmod(CD a, CD b) { ++g_counts.trans; return CD(std::fmod(a.v, b.v)); }
inline CD floor(CD a) { ++g_counts.trans; return CD(std::floor(a.v)); }
inline CD cr_atan2(CD a, CD b) { ++g_counts.trans; return CD(std::atan2(a.v, b.v)); }
inline void cr_sincos(CD a, CD *s, CD *c) {
  g_counts.trans += 2;
  *s = CD(std::sin(a.v));
  *c = CD(std::cos(a.v));
}
inline CD cr_cbrt(CD a) { ++g_counts.trans; return CD(std::cbrt(a.v)); }
inline bool isinf(CD a) { return std::isinf(a.v); }
inline bool isnan(CD a) { return std::isnan(a.v); }
inline bool signbit(CD a) { return std::signbit(a.v); }
inline CD copysign(CD a, CD b) { return CD(std::copysign(a.v, b.v)); }

}  // namespace vgbcount

#include "../vecgeom_b200/csrc/vgb_core.cuh"

namespace vgb {
template <> struct Lim<vgbcount::CD> {
  static vgbcount::CD inf() { return vgbcount::CD(HUGE_VAL); }
  static vgbcount::CD minimum() { return vgbcount::CD(DBL_MIN); }
  static vgbcount::CD quiet_nan() { return vgbcount::CD((double)NAN); }
};
}  // namespace vgb

#include "../vecgeom_b200/csrc/batch.cuh"
#include "../vecgeom_b200/csrc/geometry.h"

using namespace vgb;
using vgbcount::CD;

namespace {

template <class Ops, class P>
int count(const P &prm, const DXform &X, int op, int64_t n, const double *x, const double *y,
          const double *z, const double *dx, const double *dy, const double *dz,
          const double *st) {
  for (int64_t i = 0; i < n; ++i) {
    const V3<CD> m = {CD(x[i]), CD(y[i]), CD(z[i])};
    V3<CD> d = {CD(0.), CD(0.), CD(0.)};
    if (dx) d = {CD(dx[i]), CD(dy[i]), CD(dz[i])};
    switch (op) {
    case VGB_OP_CONTAINS: (void)Ops::contains(prm, xf_point(X, m)); break;
    case VGB_OP_INSIDE: (void)Ops::inside(prm, xf_point(X, m)); break;
    case VGB_OP_DISTANCE_TO_IN:
      (void)Ops::distance_to_in(prm, xf_point(X, m), dti_dir<Ops>(X, d), CD(st[i]));
      break;
    case VGB_OP_DISTANCE_TO_OUT: (void)Ops::distance_to_out(prm, m, d, CD(st[i])); break;
    case VGB_OP_SAFETY_TO_IN: (void)Ops::safety_to_in(prm, xf_point(X, m)); break;
    case VGB_OP_SAFETY_TO_OUT: (void)Ops::safety_to_out(prm, m); break;
    default: return -1;
    }
  }
  return 0;
}

// The boolean shapes run their components in double only (the component
// kernels are FP64 functions), so they are not counted.
template <template <class...> class OPS> struct IsBoolean : std::false_type {};
template <> struct IsBoolean<BoolOps> : std::true_type {};

template <template <class...> class OPS, class P>
int count_shape(const P &prm, const DXform &X, int op, int64_t n, const double *x,
                const double *y, const double *z, const double *dx, const double *dy,
                const double *dz, const double *st) {
  if constexpr (IsBoolean<OPS>::value)
    return -3;
  else
    return count<OPS<CD>>(prm, X, op, n, x, y, z, dx, dy, dz, st);
}

}  // namespace

// Counts the operations of `op` on n points of placed volume `placed`:
// counts[0..4] = additions/subtractions, multiplications, divisions, square
// roots, transcendentals, summed over the points.
extern "C" int oc_count(const vgb_geometry *g, int32_t placed, int32_t op, int64_t n,
                        const double *x, const double *y, const double *z, const double *dx,
                        const double *dy, const double *dz, const double *st, int64_t *counts) {
  vgbcount::g_counts = {0, 0, 0, 0, 0};
  const PlacedRec &pr = g->placed[placed];
  const DXform &X = g->xforms[pr.xform];
  const int type = g->unplaced[pr.unplaced].type;
  const void *prm = shape_params(g, pr.unplaced);
  int rc = -2;
  switch (type) {
#define VGB_SHAPE_CASE(TYPE, OPS, P)                                                   \
  case TYPE:                                                                           \
    rc = count_shape<OPS>(bind_params(*static_cast<const P *>(prm),                    \
                                      static_cast<const double *>(prm)),               \
                          X, op, n, x, y, z, dx, dy, dz, st);                          \
    break;
    VGB_FOR_EACH_SHAPE(VGB_SHAPE_CASE)
#undef VGB_SHAPE_CASE
  default:
    break;
  }
  counts[0] = vgbcount::g_counts.add;
  counts[1] = vgbcount::g_counts.mul;
  counts[2] = vgbcount::g_counts.div;
  counts[3] = vgbcount::g_counts.sqrt;
  counts[4] = vgbcount::g_counts.trans;
  return rc;
}
