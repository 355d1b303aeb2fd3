// ref_usolids.cpp -- test infrastructure, NOT product code.
//
// The reference's sphere DistanceToIn is an empty stub
// (volumes/kernel/SphereImplementation.h:84-93): a call leaves the caller's
// kInfinity in place.  The vendored USolids USphere::DistanceToIn
// (USolids/src/USphere.cc:630) is the in-tree implementation of that
// operation; this shim exposes it so the golden vectors and the parity tests
// pin the sphere's DistanceToIn to it.  Compiled with the USolids headers and
// -DVECGEOM_USOLIDS (its UVector3 is vecgeom::Vector3D<double>).
#include "base/Transformation3D.h"
#include "USphere.hh"

#include <cstdint>

using vecgeom::Transformation3D;
using vecgeom::Vector3D;

namespace {

// A placed volume of the reference is specialised on its transformation's
// rotation code and applies Transform<kGeneric, code> / TransformDirection<code>
// (volumes/ShapeImplementationHelper.h; the codes of base/Transformation3D.h:360-460,
// including 0x16A with its third-row typo).  The sphere's placed DistanceToIn
// would transform its inputs that way, so the shim does too.
template <vecgeom::RotationCode code>
void run(const USphere &s, const Transformation3D &t, int64_t n, const double *x, const double *y,
         const double *z, const double *dx, const double *dy, const double *dz, double *out) {
  for (int64_t i = 0; i < n; ++i) {
    const Vector3D<double> p(x[i], y[i], z[i]), d(dx[i], dy[i], dz[i]);
    const Vector3D<double> lp = t.Transform<vecgeom::translation::kGeneric, code>(p);
    const Vector3D<double> ld = t.TransformDirection<code>(d);
    out[i] = s.DistanceToIn(lp, ld);
  }
}

}  // namespace

extern "C" {

// DistanceToIn of a USphere(rmin, rmax, sphi, dphi, stheta, dtheta) for points
// and directions in the placement's mother frame, transformed as the
// reference's placed volume specialised on the transformation's rotation code
// transforms them.
int vgref_usphere_distance_to_in(double rmin, double rmax, double sphi, double dphi,
                                 double stheta, double dtheta, void *transform, int64_t n,
                                 const double *x, const double *y, const double *z,
                                 const double *dx, const double *dy, const double *dz,
                                 double *out) {
  USphere s("sphere", rmin, rmax, sphi, dphi, stheta, dtheta);
  Transformation3D const *t = static_cast<Transformation3D const *>(transform);
  if (!t) {
    for (int64_t i = 0; i < n; ++i)
      out[i] = s.DistanceToIn(Vector3D<double>(x[i], y[i], z[i]),
                              Vector3D<double>(dx[i], dy[i], dz[i]));
    return 0;
  }
  switch (t->GenerateRotationCode()) {
#define VGREF_CODE(c) \
  case c: run<c>(s, *t, n, x, y, z, dx, dy, dz, out); break;
    VGREF_CODE(0x1B1) VGREF_CODE(0x18E) VGREF_CODE(0x076) VGREF_CODE(0x16A)
    VGREF_CODE(0x155) VGREF_CODE(0x0AD) VGREF_CODE(0x0DC) VGREF_CODE(0x0E3)
    VGREF_CODE(0x11B) VGREF_CODE(0x0A1) VGREF_CODE(0x10A) VGREF_CODE(0x046)
    VGREF_CODE(0x062) VGREF_CODE(0x054) VGREF_CODE(0x111) VGREF_CODE(0x200)
#undef VGREF_CODE
  default: run<vecgeom::rotation::kGeneric>(s, *t, n, x, y, z, dx, dy, dz, out); break;
  }
  return 0;
}

}  // extern "C"
