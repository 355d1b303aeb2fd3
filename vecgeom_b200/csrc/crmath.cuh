// crmath.cuh -- correctly rounded atan2, sin, cos and cbrt (host and device).
//
// The torus solver (torus.cuh) builds complex cube roots from atan2, sin, cos
// and cbrt, and its distances depend on the last bit of each.  The C library
// the reference runs with and CUDA's math library round these functions
// differently (both are only faithful: within an ulp or two), so the GPU uses
// the correctly rounded value of each, which every correctly rounding C
// library returns as well.
//
// Method (no table or polynomial of any math library is reproduced):
//  * double-double arithmetic from error-free transformations: TwoSum
//    (Knuth), FastTwoSum (Dekker) and TwoProd through a fused multiply-add;
//  * sin/cos: reduction by the nearest multiple of pi/2 (pi/2 split into three
//    doubles, the first product computed exactly), then the Taylor series of
//    sin and cos in double-double on |r| <= pi/4 (terms to r^27: truncation
//    below 2^-100 relative);
//  * atan2: the library value t0 (within a few ulp), refined by one Newton
//    step on the angle: t = t0 + atan(N / D) with N = y cos t0 - x sin t0 and
//    D = x cos t0 + y sin t0, N in double-double;
//  * cbrt: the library value y, refined by one Newton step y - (y^3 - x) /
//    (3 y^2) with y^3 - x computed exactly to about 2^-106.
// Each result is the double nearest to a value within ~2^-100 (relative) of
// the exact one, so it is the correctly rounded result except when the exact
// value lies within that distance of a rounding midpoint.
//
// The sums below rely on every operation rounding once: the FP64 kernels are
// compiled with -fmad=false and host code with -ffp-contract=off.
#pragma once
#include <cmath>

#include "vgb_core.cuh"

namespace vgb {
namespace crm {

struct DD {
  double hi, lo;
};

VGB_HD DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
VGB_HD DD fast_two_sum(double a, double b) {  // |a| >= |b| or a == 0
  const double s = a + b;
  return {s, b - (s - a)};
}
VGB_HD DD two_prod(double a, double b) {
  const double p = a * b;
  return {p, fma(a, b, -p)};
}
VGB_HD DD dd_add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo = s.lo + t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo = s.lo + t.lo;
  return fast_two_sum(s.hi, s.lo);
}
VGB_HD DD dd_neg(DD a) { return {-a.hi, -a.lo}; }
VGB_HD DD dd_mul(DD a, DD b) {
  DD p = two_prod(a.hi, b.hi);
  p.lo = p.lo + (a.hi * b.lo + a.lo * b.hi);
  return fast_two_sum(p.hi, p.lo);
}
VGB_HD DD dd_mul_d(DD a, double b) {
  DD p = two_prod(a.hi, b);
  p.lo = p.lo + a.lo * b;
  return fast_two_sum(p.hi, p.lo);
}

// 1/n!, n = 0..27, double-double (hi, lo), rounded from 300-bit values.  The
// series below reads them in a loop that is not unrolled (one index for the
// whole warp, so a broadcast read): the code of one evaluation stays small.
#ifdef __CUDACC__
static __constant__ double kCrmInvFactDev[28][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76},
    {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {0x1.93974a8c07c9dp-37, 0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-41, 0x1.1d8656b0ee8cbp-97},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {0x1.6827863b97d97p-53, 0x1.eec01221a8b0bp-107},
    {0x1.2f49b46814157p-57, 0x1.2650f61dbdcb4p-112},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {0x1.0ce396db7f853p-70, -0x1.aebcdbd20331cp-124},
    {0x1.761b41316381ap-75, -0x1.3423c7d91404fp-130},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {0x1.88e85fc6a4e5ap-89, -0x1.71c37ebd16540p-143},
    {0x1.d1ab1c2dccea3p-94, 0x1.054d0c78aea14p-149}};
#endif
static const double kCrmInvFactHost[28][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76},
    {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {0x1.93974a8c07c9dp-37, 0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-41, 0x1.1d8656b0ee8cbp-97},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {0x1.6827863b97d97p-53, 0x1.eec01221a8b0bp-107},
    {0x1.2f49b46814157p-57, 0x1.2650f61dbdcb4p-112},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {0x1.0ce396db7f853p-70, -0x1.aebcdbd20331cp-124},
    {0x1.761b41316381ap-75, -0x1.3423c7d91404fp-130},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {0x1.88e85fc6a4e5ap-89, -0x1.71c37ebd16540p-143},
    {0x1.d1ab1c2dccea3p-94, 0x1.054d0c78aea14p-149}};
struct InvFact {
  double hi, lo;
};
VGB_HD InvFact inv_fact(int n) {
#ifdef __CUDA_ARCH__
  return {kCrmInvFactDev[n][0], kCrmInvFactDev[n][1]};
#else
  return {kCrmInvFactHost[n][0], kCrmInvFactHost[n][1]};
#endif
}

// sin and cos of r, |r| <= pi/4, in double-double: Horner over r^2.
VGB_HD void sincos_reduced(DD r, DD &s, DD &c) {
  const DD r2 = dd_mul(r, r);
  InvFact f = inv_fact(27);
  DD as = {-f.hi, -f.lo};  // (-1)^13 / 27!
  f = inv_fact(26);
  DD ac = {-f.hi, -f.lo};  // (-1)^13 / 26!
#pragma unroll 1
  for (int j = 12; j >= 0; --j) {
    const double sg = (j & 1) ? -1.0 : 1.0;
    const InvFact fs = inv_fact(2 * j + 1), fc = inv_fact(2 * j);
    as = dd_add(dd_mul(as, r2), DD{sg * fs.hi, sg * fs.lo});
    ac = dd_add(dd_mul(ac, r2), DD{sg * fc.hi, sg * fc.lo});
  }
  s = dd_mul(as, r);
  c = ac;
}

// sin and cos of x (|x| < 2^20), double-double.
VGB_HD void sincos_dd(double x, DD &s, DD &c) {
  const double p1 = 0x1.921fb54442d18p+0, p2 = 0x1.1a62633145c07p-54,
               p3 = -0x1.f1976b7ed8fbcp-110;  // pi/2 = p1 + p2 + p3
  const double k = rint(x * 0x1.45f306dc9c883p-1);  // x * 2/pi
  DD r = {x, 0.0};
  if (k != 0.0) {
    const DD t1 = two_prod(k, p1);
    r = two_sum(x - t1.hi, -t1.lo);  // x - t1.hi is exact (Sterbenz)
    r = dd_add(r, dd_neg(two_prod(k, p2)));
    r = dd_add(r, DD{-k * p3, 0.0});
  }
  DD sr, cr;
  sincos_reduced(r, sr, cr);
  const int q = (int)(k - 4.0 * floor(k * 0.25));  // k mod 4 in 0..3
  switch (q) {
  case 0: s = sr; c = cr; break;
  case 1: s = cr; c = dd_neg(sr); break;
  case 2: s = dd_neg(sr); c = dd_neg(cr); break;
  default: s = dd_neg(cr); c = sr; break;
  }
}

}  // namespace crm

// The functions below are kept out of line: each holds an unrolled
// double-double series, and one copy per kernel (instead of one per call site)
// keeps the instruction footprint of the torus kernels small.

// Correctly rounded sin and cos of one argument (|x| < 2^20; beyond, the
// library's values), from one double-double evaluation.
VGB_HD_NOINLINE void cr_sincos(double x, double *sn, double *cs) {
  if (!(fabs(x) < 0x1p20)) {
    *sn = sin(x);
    *cs = cos(x);
    return;
  }
  crm::DD s, c;
  crm::sincos_dd(x, s, c);
  *sn = s.hi;
  *cs = c.hi;
}
VGB_HD double cr_sin(double x) {
  double s, c;
  cr_sincos(x, &s, &c);
  return s;
}
VGB_HD double cr_cos(double x) {
  double s, c;
  cr_sincos(x, &s, &c);
  return c;
}

// Correctly rounded atan2 (finite, not both zero; otherwise the library's value).
VGB_HD_NOINLINE double cr_atan2(double y, double x) {
  const double t0 = atan2(y, x);
  if (!(fabs(x) < HUGE_VAL) || !(fabs(y) < HUGE_VAL) || (x == 0.0 && y == 0.0)) return t0;
  // scale (x, y) by a power of two so the products below neither overflow nor
  // lose their low parts to underflow; atan2 is unchanged
  const int e = ilogb(fmax(fabs(x), fabs(y)));
  const double xs = ldexp(x, -e), ys = ldexp(y, -e);
  crm::DD s, c;
  crm::sincos_dd(t0, s, c);
  const crm::DD n = crm::dd_add(crm::dd_mul_d(c, ys), crm::dd_neg(crm::dd_mul_d(s, xs)));
  const double d = xs * c.hi + ys * s.hi;
  return t0 + n.hi / d;
}

// Correctly rounded cube root (finite, nonzero; otherwise the library's value).
VGB_HD_NOINLINE double cr_cbrt(double x) {
  const double y = cbrt(x);
  if (!(fabs(y) < HUGE_VAL) || y == 0.0 || !(fabs(x) > 0x1p-900) || !(fabs(x) < 0x1p900))
    return y;
  const crm::DD y2 = crm::two_prod(y, y);      // y^2 exactly
  const crm::DD y3 = crm::two_prod(y2.hi, y);  // y2.hi * y exactly
  const double tail = y3.lo + y2.lo * y;       // y^3 = y3.hi + tail (to ~2^-106)
  const double r = (y3.hi - x) + tail;         // y3.hi - x is exact (Sterbenz)
  return y - r / (3.0 * y2.hi);
}

}  // namespace vgb
