// vecgeom_b200.hpp -- header-only C++ facade over libvgb's C ABI (vgb.h) with the
// reference's batch signatures, so that call sites written against VecGeom's
// VPlacedVolume SOA3D virtuals (volumes/PlacedVolume.h:145-250) and SOA3D
// (base/SOA3D.h:32-39) compile against this library with a namespace change.
//
//   vecgeom_b200::Geometry geo;                        // GeoManager + CudaManager
//   auto box = geo.UnplacedBox(10, 20, 30);
//   auto lv  = geo.LogicalVolume("box", box);
//   auto pv  = geo.Place(lv, geo.Transformation3D());  // LogicalVolume::Place
//   geo.SetWorld(pv); geo.CloseGeometry();
//   vecgeom_b200::SOA3D<double> pts(x, y, z, n);       // wraps caller buffers
//   pv.Inside(pts, inside);                            // same call as the reference
//
// Differences from the reference, all at the boundary:
//   * errors throw vecgeom_b200::Error (a std::runtime_error carrying the
//     vgb_status) instead of asserting;
//   * buffers may be host memory (staged through the device by the library) or
//     device memory on the geometry's GPU;
//   * the batch calls take an optional CUDA stream and are synchronous for host
//     buffers, asynchronous for device buffers.
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>

#include "vgb.h"

namespace vecgeom_b200 {

using Precision = double;
using Inside_t = int;
enum EInside { kInside = VGB_kInside, kSurface = VGB_kSurface, kOutside = VGB_kOutside };
constexpr Precision kTolerance = 1e-9;

class Error : public std::runtime_error {
 public:
  Error(vgb_status s, const std::string &what) : std::runtime_error(what), status(s) {}
  vgb_status status;
};

inline void check(vgb_status s) {
  if (s != VGB_OK) throw Error(s, vgb_last_error());
}

// SOA3D<T> with the reference's member order (fAllocated, fSize, fCapacity, fX,
// fY, fZ); this facade only wraps caller-owned buffers (fAllocated == false).
template <typename T> class SOA3D {
  bool fAllocated;
  size_t fSize, fCapacity;
  T *fX, *fY, *fZ;

 public:
  typedef T value_type;
  SOA3D(T *x, T *y, T *z, size_t size)
      : fAllocated(false), fSize(size), fCapacity(size), fX(x), fY(y), fZ(z) {}
  size_t size() const { return fSize; }
  size_t capacity() const { return fCapacity; }
  T *x() { return fX; }
  T *y() { return fY; }
  T *z() { return fZ; }
  T const *x() const { return fX; }
  T const *y() const { return fY; }
  T const *z() const { return fZ; }
};

class Geometry;

// A placed volume: the VPlacedVolume SOA3D batch virtuals.
class VPlacedVolume {
 public:
  VPlacedVolume() = default;
  VPlacedVolume(vgb_geometry *g, int32_t id) : g_(g), id_(id) {}
  int id() const { return id_; }

  void Contains(SOA3D<Precision> const &p, bool *const output, void *stream = nullptr) const {
    static_assert(sizeof(bool) == 1, "Contains writes one byte (0 or 1) per point");
    check(vgb_Contains(g_, id_, (int64_t)p.size(), p.x(), p.y(), p.z(),
                       reinterpret_cast<uint8_t *>(output), stream));
  }
  void Inside(SOA3D<Precision> const &p, Inside_t *const output, void *stream = nullptr) const {
    check(vgb_Inside(g_, id_, (int64_t)p.size(), p.x(), p.y(), p.z(), output, stream));
  }
  void DistanceToIn(SOA3D<Precision> const &p, SOA3D<Precision> const &d,
                    Precision const *const step_max, Precision *const output,
                    void *stream = nullptr) const {
    check(vgb_DistanceToIn(g_, id_, (int64_t)p.size(), p.x(), p.y(), p.z(), d.x(), d.y(), d.z(),
                           step_max, output, stream));
  }
  void DistanceToInMinimize(SOA3D<Precision> const &p, SOA3D<Precision> const &d,
                            int daughterindex, Precision *const output, int *const nextnodeids,
                            void *stream = nullptr) const {
    batch(VGB_OP_DISTANCE_TO_IN_MINIMIZE, p, &d, nullptr, output, nextnodeids, daughterindex,
          stream);
  }
  void DistanceToOut(SOA3D<Precision> const &p, SOA3D<Precision> const &d,
                     Precision const *const step_max, Precision *const output,
                     void *stream = nullptr) const {
    check(vgb_DistanceToOut(g_, id_, (int64_t)p.size(), p.x(), p.y(), p.z(), d.x(), d.y(),
                            d.z(), step_max, output, stream));
  }
  void DistanceToOut(SOA3D<Precision> const &p, SOA3D<Precision> const &d,
                     Precision const *const step_max, Precision *const output,
                     int *const nextnodeindex, void *stream = nullptr) const {
    batch(VGB_OP_DISTANCE_TO_OUT_NODE, p, &d, step_max, output, nextnodeindex, 0, stream);
  }
  void PlacedDistanceToOut(SOA3D<Precision> const &p, SOA3D<Precision> const &d,
                           Precision const *const step_max, Precision *const output,
                           void *stream = nullptr) const {
    batch(VGB_OP_PLACED_DISTANCE_TO_OUT, p, &d, step_max, output, nullptr, 0, stream);
  }
  void SafetyToIn(SOA3D<Precision> const &p, Precision *const safeties,
                  void *stream = nullptr) const {
    check(vgb_SafetyToIn(g_, id_, (int64_t)p.size(), p.x(), p.y(), p.z(), safeties, stream));
  }
  void SafetyToInMinimize(SOA3D<Precision> const &p, Precision *const safeties,
                          void *stream = nullptr) const {
    batch(VGB_OP_SAFETY_TO_IN_MINIMIZE, p, nullptr, nullptr, safeties, nullptr, 0, stream);
  }
  void SafetyToOut(SOA3D<Precision> const &p, Precision *const safeties,
                   void *stream = nullptr) const {
    check(vgb_SafetyToOut(g_, id_, (int64_t)p.size(), p.x(), p.y(), p.z(), safeties, stream));
  }
  void SafetyToOutMinimize(SOA3D<Precision> const &p, Precision *const safeties,
                           void *stream = nullptr) const {
    batch(VGB_OP_SAFETY_TO_OUT_MINIMIZE, p, nullptr, nullptr, safeties, nullptr, 0, stream);
  }

 private:
  void batch(vgb_op op, SOA3D<Precision> const &p, SOA3D<Precision> const *d,
             Precision const *step_max, void *out, int *aux, int daughter, void *stream) const {
    check(vgb_batch(g_, id_, op, (int64_t)p.size(), p.x(), p.y(), p.z(), d ? d->x() : nullptr,
                    d ? d->y() : nullptr, d ? d->z() : nullptr, step_max, out, aux, daughter,
                    VGB_PREC_FP64, stream));
  }
  vgb_geometry *g_ = nullptr;
  int32_t id_ = -1;
};

// Geometry construction (Unplaced*, Transformation3D, LogicalVolume,
// GeoManager::SetWorld/CloseGeometry) and its upload.
class Geometry {
 public:
  Geometry() { check(vgb_geometry_create(&g_)); }
  ~Geometry() { vgb_geometry_destroy(g_); }
  Geometry(const Geometry &) = delete;
  Geometry &operator=(const Geometry &) = delete;
  vgb_geometry *handle() const { return g_; }

  int UnplacedBox(double dx, double dy, double dz) {
    int32_t id;
    check(vgb_unplaced_box(g_, dx, dy, dz, &id));
    return id;
  }
  int UnplacedTube(double rmin, double rmax, double dz, double sphi, double dphi) {
    int32_t id;
    check(vgb_unplaced_tube(g_, rmin, rmax, dz, sphi, dphi, &id));
    return id;
  }
  int UnplacedCone(double rmin1, double rmax1, double rmin2, double rmax2, double dz, double sphi,
                   double dphi) {
    int32_t id;
    check(vgb_unplaced_cone(g_, rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi, &id));
    return id;
  }
  int UnplacedSphere(double rmin, double rmax, double sphi, double dphi, double stheta,
                     double dtheta) {
    int32_t id;
    check(vgb_unplaced_sphere(g_, rmin, rmax, sphi, dphi, stheta, dtheta, &id));
    return id;
  }
  int UnplacedTorus(double rmin, double rmax, double rtor, double sphi, double dphi) {
    int32_t id;
    check(vgb_unplaced_torus(g_, rmin, rmax, rtor, sphi, dphi, &id));
    return id;
  }
  int UnplacedTrd(double dx1, double dx2, double dy1, double dy2, double dz) {
    int32_t id;
    check(vgb_unplaced_trd(g_, dx1, dx2, dy1, dy2, dz, &id));
    return id;
  }
  int UnplacedPolycone(double sphi, double dphi, int nz, const double *rmin, const double *rmax,
                       const double *z) {
    int32_t id;
    check(vgb_unplaced_polycone(g_, sphi, dphi, nz, rmin, rmax, z, &id));
    return id;
  }
  int UnplacedPolyhedron(double phi_start_deg, double phi_delta_deg, int sides, int nz,
                         const double *z, const double *rmin, const double *rmax) {
    int32_t id;
    check(vgb_unplaced_polyhedron(g_, phi_start_deg, phi_delta_deg, sides, nz, z, rmin, rmax,
                                  &id));
    return id;
  }
  int UnplacedOrb(double r) {
    int32_t id;
    check(vgb_unplaced_orb(g_, r, &id));
    return id;
  }
  // alpha, theta, phi in degrees (volumes/UnplacedParallelepiped.h:34)
  int UnplacedParallelepiped(double x, double y, double z, double alpha, double theta,
                             double phi) {
    int32_t id;
    check(vgb_unplaced_parallelepiped(g_, x, y, z, alpha, theta, phi, &id));
    return id;
  }
  int UnplacedParaboloid(double rlo, double rhi, double dz) {
    int32_t id;
    check(vgb_unplaced_paraboloid(g_, rlo, rhi, dz, &id));
    return id;
  }
  // theta, phi in radians (volumes/UnplacedTrapezoid.h:93-95)
  int UnplacedTrapezoid(double dz, double theta, double phi, double dy1, double dx1, double dx2,
                        double tan_alpha1, double dy2, double dx3, double dx4,
                        double tan_alpha2) {
    int32_t id;
    check(vgb_unplaced_trapezoid(g_, dz, theta, phi, dy1, dx1, dx2, tan_alpha1, dy2, dx3, dx4,
                                 tan_alpha2, &id));
    return id;
  }
  // corners[24]: 8 corners (x, y, z), 0-3 at z = -dz, 4-7 at z = +dz
  // (volumes/UnplacedTrapezoid.h:103)
  int UnplacedTrapezoid(const double *corners) {
    int32_t id;
    check(vgb_unplaced_trapezoid_corners(g_, corners, &id));
    return id;
  }
  int UnplacedBooleanVolume(int op, const VPlacedVolume &left, const VPlacedVolume &right) {
    int32_t id;
    check(vgb_unplaced_boolean(g_, op, left.id(), right.id(), &id));
    return id;
  }
  int Transformation3D(double tx = 0, double ty = 0, double tz = 0, double phi = 0,
                       double theta = 0, double psi = 0) {
    int32_t id;
    check(vgb_transformation(g_, tx, ty, tz, phi, theta, psi, &id));
    return id;
  }
  int LogicalVolume(const char *label, int unplaced) {
    int32_t id;
    check(vgb_logical_volume(g_, label, unplaced, &id));
    return id;
  }
  VPlacedVolume Place(int logical, int transformation) {
    int32_t id;
    check(vgb_place(g_, logical, transformation, &id));
    return VPlacedVolume(g_, id);
  }
  VPlacedVolume PlaceDaughter(int mother, int daughter, int transformation) {
    int32_t id;
    check(vgb_place_daughter(g_, mother, daughter, transformation, &id));
    return VPlacedVolume(g_, id);
  }
  void SetWorld(const VPlacedVolume &w) { check(vgb_set_world(g_, w.id())); }
  void CloseGeometry() { check(vgb_geometry_close(g_)); }
  int getMaxDepth() const {
    int32_t d;
    check(vgb_geometry_max_depth(g_, &d));
    return d;
  }

 private:
  vgb_geometry *g_ = nullptr;
};

}  // namespace vecgeom_b200
