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

extern "C" {

// DistanceToIn of a USphere(rmin, rmax, sphi, dphi, stheta, dtheta) for points
// and directions in the placement's mother frame; the placement is applied with
// the reference's generic Transformation3D::Transform/TransformDirection.
int vgref_usphere_distance_to_in(double rmin, double rmax, double sphi, double dphi,
                                 double stheta, double dtheta, void *transform, int64_t n,
                                 const double *x, const double *y, const double *z,
                                 const double *dx, const double *dy, const double *dz,
                                 double *out) {
  USphere s("sphere", rmin, rmax, sphi, dphi, stheta, dtheta);
  Transformation3D const *t = static_cast<Transformation3D const *>(transform);
  for (int64_t i = 0; i < n; ++i) {
    Vector3D<double> p(x[i], y[i], z[i]), d(dx[i], dy[i], dz[i]);
    Vector3D<double> lp = t ? t->Transform(p) : p;
    Vector3D<double> ld = t ? t->TransformDirection(d) : d;
    out[i] = s.DistanceToIn(lp, ld);
  }
  return 0;
}

}  // extern "C"
