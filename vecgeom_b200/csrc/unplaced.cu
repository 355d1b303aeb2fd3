// unplaced.cu -- the unplaced-shape constructors of the C ABI.
//
// Each computes the shape's cached values with the reference constructor's
// formulas (host code, -ffp-contract=off, glibc cos/sin as in the reference),
// so the device kernels see bit-identical constants.
#include <cmath>
#include <cstring>

#include "geometry.h"
#include "shapes.cuh"

using namespace vgb;

namespace vgb {

// Wedge::Wedge(angle, zeroangle) (source/Wedge.cpp:14-45)
WedgeP make_wedge(double dphi, double sphi) {
  WedgeP w;
  std::memset(&w, 0, sizeof(w));
  w.a1x = std::cos(sphi);
  w.a1y = std::sin(sphi);
  w.a2x = std::cos(sphi + dphi);
  w.a2y = std::sin(sphi + dphi);
  w.n1x = -std::sin(sphi);
  w.n1y = std::cos(sphi);
  w.n2x = std::sin(sphi + dphi);
  w.n2y = -std::cos(sphi + dphi);
  w.dphi = dphi;
  w.lt_pi = dphi < kPi;
  return w;
}

// UnplacedTube::calculateCached (volumes/UnplacedTube.h:38-60)
TubeP make_tube(double rmin, double rmax, double z, double sphi, double dphi) {
  TubeP t;
  std::memset(&t, 0, sizeof(t));
  t.rmin = rmin;
  t.rmax = rmax;
  t.z = z;
  t.sphi = sphi;
  t.dphi = dphi;
  t.tolIz = z - kTolerance;
  t.tolOz = z + kTolerance;
  t.rmin2 = rmin * rmin;
  t.rmax2 = rmax * rmax;
  const double tolOrmin = rmin - kTolerance, tolIrmin = rmin + kTolerance;
  t.tolOrmin2 = tolOrmin * tolOrmin;
  t.tolIrmin2 = tolIrmin * tolIrmin;
  const double tolOrmax = rmax + kTolerance, tolIrmax = rmax - kTolerance;
  t.tolOrmax2 = tolOrmax * tolOrmax;
  t.tolIrmax2 = tolIrmax * tolIrmax;
  t.a1x = std::cos(sphi);
  t.a1y = std::sin(sphi);
  t.a2x = std::cos(sphi + dphi);
  t.a2y = std::sin(sphi + dphi);
  t.wedge = make_wedge(dphi, sphi);
  // volumes/kernel/shapetypes/TubeTypes.h:104-158 (UniversalTube: run-time checks)
  t.has_rmin = rmin > 0;
  t.has_phi = dphi < 2 * M_PI;
  t.le_pi = dphi <= M_PI;
  return t;
}

// UnplacedCone constructor (volumes/UnplacedCone.h:108-170)
ConeP make_cone(double rmin1, double rmax1, double rmin2, double rmax2, double dz, double sphi,
                double dphi) {
  ConeP c;
  std::memset(&c, 0, sizeof(c));
  c.rmin1 = rmin1;
  c.rmax1 = rmax1;
  c.rmin2 = rmin2;
  c.rmax2 = rmax2;
  c.dz = dz;
  c.sphi = sphi;
  c.dphi = dphi;
  const double hDPhi = 0.5 * dphi;
  const double cPhi = sphi + hDPhi;
  const double ePhi = sphi + dphi;
  c.sinCPhi = std::sin(cPhi);
  c.cosCPhi = std::cos(cPhi);
  c.cosHDPhi = std::cos(hDPhi);
  c.cosHDPhiIT = std::cos(hDPhi - 0.5 * kAngTolerance);
  c.cosHDPhiOT = std::cos(hDPhi + 0.5 * kAngTolerance);
  c.sinSPhi = std::sin(sphi);
  c.cosSPhi = std::cos(sphi);
  c.sinEPhi = std::sin(ePhi);
  c.cosEPhi = std::cos(ePhi);
  c.tanRMin = (rmin2 - rmin1) * 0.5 / dz;
  c.secRMin = std::sqrt(1.0 + c.tanRMin * c.tanRMin);
  c.invSecRMin = 1. / c.secRMin;
  c.tanRMax = (rmax2 - rmax1) * 0.5 / dz;
  c.secRMax = std::sqrt(1.0 + c.tanRMax * c.tanRMax);
  c.invSecRMax = 1. / c.secRMax;
  c.innerSlope = -(rmin1 - rmin2) / (2. * dz);
  c.outerSlope = -(rmax1 - rmax2) / (2. * dz);
  c.innerOffset = rmin2 - c.innerSlope * dz;
  c.outerOffset = rmax2 - c.outerSlope * dz;
  c.wedge = make_wedge(dphi, sphi);
  c.full_phi = dphi == kTwoPi;
  // volumes/kernel/shapetypes/ConeTypes.h:107-162 (UniversalCone: run-time checks)
  c.has_rmin = rmin1 > 0 || rmin2 > 0;
  c.has_phi = dphi < 2. * M_PI;
  return c;
}

}  // namespace vgb

extern "C" {

vgb_status vgb_unplaced_cone(vgb_geometry *g, double rmin1, double rmax1, double rmin2,
                             double rmax2, double dz, double sphi, double dphi, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(dz > 0 && rmin1 >= 0 && rmin2 >= 0 && rmax1 >= rmin1 && rmax2 >= rmin2 && dphi > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_cone: invalid radii, dz or dphi");
  ConeP c = make_cone(rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi);
  return add_unplaced(g, VGB_SHAPE_CONE, &c, sizeof(c), 0, id);
}

vgb_status vgb_unplaced_box(vgb_geometry *g, double dx, double dy, double dz, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(dx > 0 && dy > 0 && dz > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_box: half-lengths must be > 0");
  BoxP b;
  b.d[0] = dx;
  b.d[1] = dy;
  b.d[2] = dz;
  return add_unplaced(g, VGB_SHAPE_BOX, &b, sizeof(b), 0, id);
}

vgb_status vgb_unplaced_tube(vgb_geometry *g, double rmin, double rmax, double dz, double sphi,
                             double dphi, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(rmin >= 0 && rmax > rmin && dz > 0 && dphi > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_tube: need 0 <= rmin < rmax, dz > 0, dphi > 0");
  TubeP t = make_tube(rmin, rmax, dz, sphi, dphi);
  return add_unplaced(g, VGB_SHAPE_TUBE, &t, sizeof(t), 0, id);
}

// ---------------------------------------------------------------------------
// shapes not yet uploaded by this build report VGB_ENOTSUP
// ---------------------------------------------------------------------------
#define VGB_NOTYET(name) return set_error(VGB_ENOTSUP, name ": shape not available yet")
vgb_status vgb_unplaced_sphere(vgb_geometry *, double, double, double, double, double, double,
                               int32_t *) {
  VGB_NOTYET("vgb_unplaced_sphere");
}
vgb_status vgb_unplaced_torus(vgb_geometry *, double, double, double, double, double, int32_t *) {
  VGB_NOTYET("vgb_unplaced_torus");
}
vgb_status vgb_unplaced_polycone(vgb_geometry *, double, double, int32_t, const double *,
                                 const double *, const double *, int32_t *) {
  VGB_NOTYET("vgb_unplaced_polycone");
}
vgb_status vgb_unplaced_polyhedron(vgb_geometry *, double, double, int32_t, int32_t,
                                   const double *, const double *, const double *, int32_t *) {
  VGB_NOTYET("vgb_unplaced_polyhedron");
}
vgb_status vgb_unplaced_trd(vgb_geometry *, double, double, double, double, double, int32_t *) {
  VGB_NOTYET("vgb_unplaced_trd");
}
vgb_status vgb_unplaced_boolean(vgb_geometry *, int32_t, int32_t, int32_t, int32_t *) {
  VGB_NOTYET("vgb_unplaced_boolean");
}
#undef VGB_NOTYET

}  // extern "C"
