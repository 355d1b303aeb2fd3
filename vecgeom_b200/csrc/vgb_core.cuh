// vgb_core.cuh -- constants, small vector type and placement transforms shared by
// every kernel of libvgb.
//
// The FP64 kernels are compiled with -fmad=false: every a*b+c rounds twice, as
// in the reference Scalar build compiled with -ffp-contract=off, so Inside/
// Contains and the navigator's next volume come out bit-identical.
#pragma once

#include <cstdint>
#include <cfloat>
#include <cmath>

#ifdef __CUDACC__
#define VGB_HD __host__ __device__ __forceinline__
#define VGB_D __device__ __forceinline__
#define VGB_HD_NOINLINE inline __host__ __device__ __noinline__
#else
#define VGB_HD inline
#define VGB_D inline
#define VGB_HD_NOINLINE inline __attribute__((noinline))
#endif

namespace vgb {

// base/Global.h:267-302
constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2. * kPi;
constexpr double kDegToRad = kPi / 180.;
constexpr double kTolerance = 1e-9;
constexpr double kHalfTolerance = 0.5 * kTolerance;
constexpr double kRadTolerance = 1e-9;
constexpr double kAngTolerance = 1e-9;
constexpr double kMinimum = DBL_MIN;
constexpr double kTiny = 1e-30;

// EnumInside (base/Global.h:196-207)
constexpr int kInside = 0;
constexpr int kSurface = 1;
constexpr int kOutside = 2;

template <class R> struct Lim;
template <> struct Lim<double> {
  static VGB_HD double inf() { return HUGE_VAL; }
  static VGB_HD double minimum() { return DBL_MIN; }
  static VGB_HD double quiet_nan() { return (double)NAN; }
};
template <> struct Lim<float> {
  static VGB_HD float inf() { return HUGE_VALF; }
  static VGB_HD float minimum() { return FLT_MIN; }
  static VGB_HD float quiet_nan() { return NAN; }
};

// Min/Max of the reference Scalar backend (backend/scalar/Backend.h:146-163) are
// std::min/std::max: min(a,b) = b < a ? b : a, max(a,b) = a < b ? b : a.  The
// same selects keep NaN and signed-zero results identical.
template <class R> VGB_HD R vmin(R a, R b) { return b < a ? b : a; }
template <class R> VGB_HD R vmax(R a, R b) { return a < b ? b : a; }

template <class R> struct V3 {
  R x, y, z;
  VGB_HD R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <class R> VGB_HD V3<R> mk3(R x, R y, R z) { return V3<R>{x, y, z}; }

// True when the ray q + t v (t >= 0) stays farther than rb from the z axis
// wherever zlo <= z <= zhi (or never reaches that slab).  Callers widen the slab
// and the radius by margins far above the rounding of this test and of their own
// arithmetic.  False for a NaN or infinite input.
template <class R>
VGB_HD bool ray_beyond_radius(const V3<R> &q, const V3<R> &v, R zlo, R zhi, R rb) {
  if (!(fabs(q.x) + fabs(q.y) + fabs(q.z) + fabs(v.x) + fabs(v.y) + fabs(v.z) < Lim<R>::inf()))
    return false;
  R t0 = 0, t1 = Lim<R>::inf();
  if (v.z != 0) {
    R ta = (zlo - q.z) / v.z, tb = (zhi - q.z) / v.z;
    if (ta > tb) {
      const R t = ta;
      ta = tb;
      tb = t;
    }
    t0 = ta > t0 ? ta : t0;
    t1 = tb;
    if (t0 > t1) return true;  // the slab lies behind the point
  } else if (q.z < zlo || q.z > zhi) {
    return true;  // parallel to the slab, outside it
  }
  // the closest approach to the axis over [t0, t1]
  const R a = v.x * v.x + v.y * v.y;
  R tm = t0;
  if (a > 0) {
    tm = -(q.x * v.x + q.y * v.y) / a;
    tm = tm < t0 ? t0 : (tm > t1 ? t1 : tm);
  }
  const R x = q.x + tm * v.x, y = q.y + tm * v.y;
  return x * x + y * y > rb * rb;
}

// Placement transform as uploaded to the device.  r/t hold the *effective*
// matrix: the entries a specialised rotation code drops
// (base/Transformation3D.h:367-480, management/TransformationSpecializations.icc)
// are zeroed, and t is zero when the translation code is kIdentity.  The generic
// row-order sum over r then reproduces every specialised DoRotation<code>.
enum : int32_t {
  kXfHasTrans = 1,   // translation applied (translation code kGeneric)
  kXfHasRot = 2,     // rotation applied (rotation code != 0x200)
  kXfQuirk16A = 4,   // rotation code 0x16A: third row is m2*R5 + m2*R8 (reference typo,
                     // base/Transformation3D.h:391)
};

struct alignas(16) DXform {
  double r[9];
  double t[3];
  int32_t flags;
  int32_t pad;
};

// base/Transformation3D.h:533-562 Transform<trans_code, rot_code>
template <class R>
VGB_HD V3<R> xf_point(const DXform &X, const V3<R> &m) {
  V3<R> a = m;
  if (X.flags & kXfHasTrans) {
    a.x = m.x - (R)X.t[0];
    a.y = m.y - (R)X.t[1];
    a.z = m.z - (R)X.t[2];
  }
  if (!(X.flags & kXfHasRot)) return a;
  V3<R> l;
  l.x = a.x * (R)X.r[0];
  l.y = a.x * (R)X.r[1];
  l.z = a.x * (R)X.r[2];
  l.x = l.x + a.y * (R)X.r[3];
  l.y = l.y + a.y * (R)X.r[4];
  l.z = l.z + a.y * (R)X.r[5];
  l.x = l.x + a.z * (R)X.r[6];
  l.y = l.y + a.z * (R)X.r[7];
  l.z = l.z + a.z * (R)X.r[8];
  if (X.flags & kXfQuirk16A) l.z = a.z * (R)X.r[5] + a.z * (R)X.r[8];
  return l;
}

// base/Transformation3D.h:751-767 TransformDirection<rot_code>
template <class R>
VGB_HD V3<R> xf_dir(const DXform &X, const V3<R> &m) {
  if (!(X.flags & kXfHasRot)) return m;
  V3<R> l;
  l.x = m.x * (R)X.r[0];
  l.y = m.x * (R)X.r[1];
  l.z = m.x * (R)X.r[2];
  l.x = l.x + m.y * (R)X.r[3];
  l.y = l.y + m.y * (R)X.r[4];
  l.z = l.z + m.y * (R)X.r[5];
  l.x = l.x + m.z * (R)X.r[6];
  l.y = l.y + m.z * (R)X.r[7];
  l.z = l.z + m.z * (R)X.r[8];
  if (X.flags & kXfQuirk16A) l.z = m.z * (R)X.r[5] + m.z * (R)X.r[8];
  return l;
}

// base/Transformation3D.h:598-632 InverseTransform (local -> master), used by the
// navigator to compose paths.
template <class R>
VGB_HD V3<R> xf_inverse_point(const DXform &X, const V3<R> &l) {
  V3<R> m;
  m.x = (R)X.t[0];
  m.x = m.x + l.x * (R)X.r[0];
  m.x = m.x + l.y * (R)X.r[1];
  m.x = m.x + l.z * (R)X.r[2];
  m.y = (R)X.t[1];
  m.y = m.y + l.x * (R)X.r[3];
  m.y = m.y + l.y * (R)X.r[4];
  m.y = m.y + l.z * (R)X.r[5];
  m.z = (R)X.t[2];
  m.z = m.z + l.x * (R)X.r[6];
  m.z = m.z + l.y * (R)X.r[7];
  m.z = m.z + l.z * (R)X.r[8];
  return m;
}

}  // namespace vgb
