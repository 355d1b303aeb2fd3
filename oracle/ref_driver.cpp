// ref_driver.cpp -- test infrastructure, NOT product code.
//
// A thin C-ABI over the reference VecGeom Scalar backend (compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/).  It is used
// only by tests/ (to pin the C restatement in oracle/vgb_oracle.c and to write
// the golden fixtures in tests/golden/) and by bench.py's CPU-baseline leg.
//
// Every entry point builds or calls the reference's own objects:
//   - shapes: Unplaced{Box,Tube,Cone,Sphere,Torus,Polycone,Polyhedron,Trd,Orb,
//     Parallelepiped,Paraboloid,Trapezoid,BooleanVolume} constructors
//     (volumes/Unplaced*.h),
//   - placement: LogicalVolume::Place / PlaceDaughter (source/LogicalVolume.cpp:60-102),
//   - batch ops: the VPlacedVolume SOA3D virtuals (volumes/PlacedVolume.h:145-250),
//   - navigation: SimpleNavigator (navigation/SimpleNavigator.h:204-743).
#include "base/Global.h"
#include "base/SOA3D.h"
#include "base/Transformation3D.h"
#include "volumes/LogicalVolume.h"
#include "volumes/PlacedVolume.h"
#include "volumes/Box.h"
#include "volumes/Tube.h"
#include "volumes/Cone.h"
#include "volumes/Sphere.h"
#include "volumes/Torus.h"
#include "volumes/Polycone.h"
#include "volumes/Polyhedron.h"
#include "volumes/Trd.h"
#include "volumes/Orb.h"
#include "volumes/Parallelepiped.h"
#include "volumes/Paraboloid.h"
#include "volumes/Trapezoid.h"
#include "volumes/BooleanVolume.h"
#include "management/GeoManager.h"
#include "navigation/NavigationState.h"
#include "navigation/SimpleNavigator.h"
#include "navigation/ABBoxNavigator.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <thread>
#include <vector>

using namespace vecgeom;

namespace {

enum RefOp {
  kOpContains = 0,
  kOpInside = 1,
  kOpDistanceToIn = 2,
  kOpDistanceToOut = 3,
  kOpSafetyToIn = 4,
  kOpSafetyToOut = 5,
  kOpDistanceToInMinimize = 6,
  kOpSafetyToInMinimize = 7,
  kOpSafetyToOutMinimize = 8,
  kOpDistanceToOutNode = 9,
  kOpPlacedDistanceToOut = 10,
};

// One chunk of a batch call on the reference's SOA3D virtuals.
void RunChunk(VPlacedVolume const *v, int op, size_t n, double *x, double *y,
              double *z, double *dx, double *dy, double *dz, double *step,
              void *out, int *aux, int daughter) {
  SOA3D<Precision> p(x, y, z, n);
  SOA3D<Precision> d(dx, dy, dz, n);
  switch (op) {
  case kOpContains:
    v->Contains(p, static_cast<bool *>(out));
    break;
  case kOpInside:
    v->Inside(p, static_cast<Inside_t *>(out));
    break;
  case kOpDistanceToIn: {
    // The Scalar SOA loop (volumes/ShapeImplementationHelper.h:619-634) leaves the
    // output untouched on a miss; the Vc loop (:365-392) and the scalar
    // single-point call (:199-220) start from kInfinity.  Pre-fill kInfinity so
    // the batch result is the single-point result.
    double *o = static_cast<double *>(out);
    for (size_t i = 0; i < n; ++i) o[i] = kInfinity;
    v->DistanceToIn(p, d, step, o);
    break;
  }
  case kOpDistanceToOut: {
    double *o = static_cast<double *>(out);
    for (size_t i = 0; i < n; ++i) o[i] = kInfinity;
    v->DistanceToOut(p, d, step, o);
    break;
  }
  case kOpDistanceToOutNode: {
    double *o = static_cast<double *>(out);
    for (size_t i = 0; i < n; ++i) o[i] = kInfinity;
    v->DistanceToOut(p, d, step, o, aux);
    break;
  }
  case kOpSafetyToIn:
    v->SafetyToIn(p, static_cast<double *>(out));
    break;
  case kOpSafetyToOut:
    v->SafetyToOut(p, static_cast<double *>(out));
    break;
  case kOpDistanceToInMinimize:
    v->DistanceToInMinimize(p, d, daughter, static_cast<double *>(out), aux);
    break;
  case kOpSafetyToInMinimize:
    v->SafetyToInMinimize(p, static_cast<double *>(out));
    break;
  case kOpSafetyToOutMinimize:
    v->SafetyToOutMinimize(p, static_cast<double *>(out));
    break;
  case kOpPlacedDistanceToOut: {
    double *o = static_cast<double *>(out);
    for (size_t i = 0; i < n; ++i)
      o[i] = v->PlacedDistanceToOut(Vector3D<Precision>(x[i], y[i], z[i]),
                                    Vector3D<Precision>(dx[i], dy[i], dz[i]), step[i]);
    break;
  }
  }
}

size_t OutSize(int op) {
  if (op == kOpContains) return sizeof(bool);
  if (op == kOpInside) return sizeof(Inside_t);
  return sizeof(double);
}

} // namespace

extern "C" {

// ---- shapes (parameters exactly as the reference constructors take them) ----
void *vgref_box(double dx, double dy, double dz) { return new UnplacedBox(dx, dy, dz); }
void *vgref_tube(double rmin, double rmax, double dz, double sphi, double dphi) {
  return new UnplacedTube(rmin, rmax, dz, sphi, dphi);
}
void *vgref_cone(double rmin1, double rmax1, double rmin2, double rmax2, double dz,
                 double sphi, double dphi) {
  return new UnplacedCone(rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi);
}
void *vgref_sphere(double rmin, double rmax, double sphi, double dphi, double stheta,
                   double dtheta) {
  return new UnplacedSphere(rmin, rmax, sphi, dphi, stheta, dtheta);
}
void *vgref_torus(double rmin, double rmax, double rtor, double sphi, double dphi) {
  return new UnplacedTorus(rmin, rmax, rtor, sphi, dphi);
}
void *vgref_polycone(double sphi, double dphi, int nz, const double *z, const double *rmin,
                     const double *rmax) {
  std::vector<double> zz(z, z + nz), r0(rmin, rmin + nz), r1(rmax, rmax + nz);
  return new UnplacedPolycone(sphi, dphi, nz, r0.data(), r1.data(), zz.data());
}
void *vgref_polyhedron(double phistart_deg, double phidelta_deg, int nsides, int nz,
                       const double *z, const double *rmin, const double *rmax) {
  std::vector<double> zz(z, z + nz);
  return new UnplacedPolyhedron(phistart_deg, phidelta_deg, nsides, nz, zz.data(), rmin, rmax);
}
// UnplacedOrb(r) computes its tolerance from a member not yet initialised
// (volumes/UnplacedOrb.h:27-35, source/UnplacedOrb.cpp:33-44); SetRadius, the
// reference's own setter, recomputes the cached values with it initialised.
void *vgref_orb(double r) {
  UnplacedOrb *o = new UnplacedOrb(r);
  o->SetRadius(r);
  return o;
}
void *vgref_parallelepiped(double x, double y, double z, double alpha, double theta, double phi) {
  return new UnplacedParallelepiped(x, y, z, alpha, theta, phi);
}
void *vgref_paraboloid(double rlo, double rhi, double dz) {
  return new UnplacedParaboloid(rlo, rhi, dz);
}
void *vgref_trapezoid(double dz, double theta, double phi, double dy1, double dx1, double dx2,
                      double ta1, double dy2, double dx3, double dx4, double ta2) {
  return new UnplacedTrapezoid(dz, theta, phi, dy1, dx1, dx2, ta1, dy2, dx3, dx4, ta2);
}
void *vgref_trapezoid_corners(const double *c) {
  TrapCorners_t pt;
  for (int k = 0; k < 8; ++k) pt[k] = Vector3D<Precision>(c[3 * k], c[3 * k + 1], c[3 * k + 2]);
  return new UnplacedTrapezoid(pt);
}
void *vgref_trd(double x1, double x2, double y1, double y2, double z) {
  return new UnplacedTrd(x1, x2, y1, y2, z);
}
void *vgref_boolean(int op, void *left_placed, void *right_placed) {
  return new UnplacedBooleanVolume(static_cast<BooleanOperation>(op),
                                   static_cast<VPlacedVolume const *>(left_placed),
                                   static_cast<VPlacedVolume const *>(right_placed));
}

// ---- placement ----
void *vgref_transform_euler(double tx, double ty, double tz, double phi, double theta,
                            double psi) {
  return new Transformation3D(tx, ty, tz, phi, theta, psi);
}
void *vgref_transform_matrix(double tx, double ty, double tz, const double *r) {
  return new Transformation3D(tx, ty, tz, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7],
                              r[8]);
}
void *vgref_transform_translation(double tx, double ty, double tz) {
  return new Transformation3D(tx, ty, tz);
}
void vgref_transform_get(void *t, double *out12, int *codes) {
  Transformation3D const *tr = static_cast<Transformation3D const *>(t);
  for (int i = 0; i < 3; ++i) out12[i] = tr->Translation(i);
  for (int i = 0; i < 9; ++i) out12[3 + i] = tr->Rotation(i);
  codes[0] = tr->GenerateTranslationCode();
  codes[1] = tr->GenerateRotationCode();
}
void *vgref_logical(const char *label, void *unplaced) {
  return new LogicalVolume(label, static_cast<VUnplacedVolume const *>(unplaced));
}
void *vgref_place(void *logical, void *transform) {
  return static_cast<LogicalVolume *>(logical)->Place(
      static_cast<Transformation3D const *>(transform));
}
void *vgref_place_daughter(void *mother_logical, void *daughter_logical, void *transform) {
  return const_cast<VPlacedVolume *>(static_cast<LogicalVolume *>(mother_logical)->PlaceDaughter(
      static_cast<LogicalVolume const *>(daughter_logical),
      static_cast<Transformation3D const *>(transform)));
}

// ---- batch ops over the SOA3D virtuals; nthreads > 1 splits the batch into
// contiguous std::thread chunks (the shape calls are const and stateless) ----
int vgref_batch(void *placed, int op, int64_t n, double *x, double *y, double *z, double *dx,
                double *dy, double *dz, double *step, void *out, int *aux, int daughter,
                int nthreads) {
  VPlacedVolume const *v = static_cast<VPlacedVolume const *>(placed);
  if (n <= 0) return 0;
  if (nthreads <= 1 || n < 4096) {
    RunChunk(v, op, (size_t)n, x, y, z, dx, dy, dz, step, out, aux, daughter);
    return 0;
  }
  std::vector<std::thread> pool;
  const int64_t chunk = (n + nthreads - 1) / nthreads;
  const size_t osz = OutSize(op);
  for (int t = 0; t < nthreads; ++t) {
    const int64_t b = t * chunk;
    const int64_t e = std::min<int64_t>(n, b + chunk);
    if (b >= e) break;
    pool.emplace_back([=] {
      RunChunk(v, op, (size_t)(e - b), x + b, y + b, z + b, dx ? dx + b : nullptr,
               dy ? dy + b : nullptr, dz ? dz + b : nullptr, step ? step + b : nullptr,
               static_cast<char *>(out) + b * osz, aux ? aux + b : nullptr, daughter);
    });
  }
  for (auto &th : pool) th.join();
  return 0;
}

// ---- navigation (navigation/SimpleNavigator.h) ----
void vgref_set_world(void *placed) {
  GeoManager::Instance().SetWorld(static_cast<VPlacedVolume const *>(placed));
}
int vgref_close_geometry(void) {
  GeoManager::Instance().CloseGeometry();
  return GeoManager::Instance().getMaxDepth();
}
int vgref_placed_id(void *placed) { return static_cast<VPlacedVolume const *>(placed)->id(); }

// Trace straight-line tracks from their start to the world exit with
// SimpleNavigator::FindNextBoundaryAndStep (navigation/SimpleNavigator.h:340-568)
// and GetSafety (:572-596).  For each step, record the placed-volume id of the
// state's Top() after the step (-1 once outside the world), the step length and
// the safety at the start point.  Returns the number of steps of each track in
// nsteps[i]; the per-track records start at i*max_steps.  nthreads splits tracks.
int vgref_nav_trace(int64_t ntracks, const double *x, const double *y, const double *z,
                    const double *dx, const double *dy, const double *dz, double pstep,
                    int max_steps, int *next_ids, double *steps, double *safeties,
                    int *nsteps, int nthreads) {
  const int depth = GeoManager::Instance().getMaxDepth();
  VPlacedVolume const *world = GeoManager::Instance().GetWorld();
  auto work = [=](int64_t b, int64_t e) {
    SimpleNavigator nav;
    NavigationState *cur = NavigationState::MakeInstance(depth);
    NavigationState *nxt = NavigationState::MakeInstance(depth);
    for (int64_t i = b; i < e; ++i) {
      Vector3D<Precision> p(x[i], y[i], z[i]);
      Vector3D<Precision> d(dx[i], dy[i], dz[i]);
      cur->Clear();
      nav.LocatePoint(world, p, *cur, true);
      int k = 0;
      while (!cur->IsOutside() && k < max_steps) {
        double safety = nav.GetSafety(p, *cur);
        double step = 0;
        nxt->Clear();
        nav.FindNextBoundaryAndStep(p, d, *cur, *nxt, pstep, step);
        next_ids[i * max_steps + k] = nxt->IsOutside() ? -1 : nxt->Top()->id();
        steps[i * max_steps + k] = step;
        safeties[i * max_steps + k] = safety;
        // advance like a client stepping to the boundary (the navigator itself
        // only pushes the point used for the relocation, :460-470)
        p = p + d * step;
        std::swap(cur, nxt);
        ++k;
      }
      nsteps[i] = k;
    }
    NavigationState::ReleaseInstance(cur);
    NavigationState::ReleaseInstance(nxt);
  };
  if (nthreads <= 1) {
    work(0, ntracks);
    return 0;
  }
  std::vector<std::thread> pool;
  const int64_t chunk = (ntracks + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    const int64_t b = t * chunk, e = std::min<int64_t>(ntracks, b + chunk);
    if (b >= e) break;
    pool.emplace_back(work, b, e);
  }
  for (auto &th : pool) th.join();
  return 0;
}

// Basket navigation (navigation/SimpleNavigator.h:599-743).  Every track is
// located from the world and moved by `prior` scalar steps (GetSafety is not
// needed for that; FindNextBoundaryAndStep and p += d * step, as the trace
// does); the tracks that are then inside are grouped into baskets by Top()
// volume, in track order, and each basket takes one basket
// FindNextBoundaryAndStep (SOA3D containers) and one GetSafeties.  Per track:
// distance, safety, next-node workspace entry, the new state's Top() id (-1
// outside) and boundary flag; tracks outside before the basket step get -7 ids
// and NaN values.  The points the basket step starts from are written to
// px/py/pz.
int vgref_nav_basket_step(int64_t n, const double *x, const double *y, const double *z,
                          const double *dx, const double *dy, const double *dz,
                          const double *pstep, int prior, double *px, double *py, double *pz,
                          double *dist, double *safety, int *nextnode, int *newtop,
                          int *boundary) {
  const int depth = GeoManager::Instance().getMaxDepth();
  VPlacedVolume const *world = GeoManager::Instance().GetWorld();
  SimpleNavigator nav;
  std::vector<NavigationState *> cur((size_t)n), nxt((size_t)n);
  NavigationState *tmp = NavigationState::MakeInstance(depth);
  for (int64_t i = 0; i < n; ++i) {
    cur[i] = NavigationState::MakeInstance(depth);
    nxt[i] = NavigationState::MakeInstance(depth);
    Vector3D<Precision> p(x[i], y[i], z[i]);
    Vector3D<Precision> d(dx[i], dy[i], dz[i]);
    nav.LocatePoint(world, p, *cur[i], true);
    for (int k = 0; k < prior && !cur[i]->IsOutside(); ++k) {
      double step = 0;
      tmp->Clear();
      nav.FindNextBoundaryAndStep(p, d, *cur[i], *tmp, 1e30, step);
      p = p + d * step;
      tmp->CopyTo(cur[i]);
    }
    px[i] = p.x();
    py[i] = p.y();
    pz[i] = p.z();
    dist[i] = safety[i] = std::numeric_limits<double>::quiet_NaN();
    nextnode[i] = newtop[i] = boundary[i] = -7;
  }
  std::map<VPlacedVolume const *, std::vector<int64_t>> baskets;
  for (int64_t i = 0; i < n; ++i)
    if (!cur[i]->IsOutside()) baskets[cur[i]->Top()].push_back(i);
  for (auto &kv : baskets) {
    const std::vector<int64_t> &ix = kv.second;
    const size_t m = ix.size();
    SOA3D<Precision> gp(m), gd(m), lp(m), ld(m);
    std::vector<NavigationState *> cs(m), ns(m);
    // the basket step leaves a distance untouched where a shape kernel does not
    // write it; start from kInfinity as the batch calls here do
    std::vector<double> ps(m), ds(m, kInfinity), sf(m);
    std::vector<int> nn(m);
    for (size_t k = 0; k < m; ++k) {
      const int64_t i = ix[k];
      gp.set(k, px[i], py[i], pz[i]);
      gd.set(k, dx[i], dy[i], dz[i]);
      cs[k] = cur[i];
      ns[k] = nxt[i];
      ps[k] = pstep[i];
    }
    nav.FindNextBoundaryAndStep(gp, gd, lp, ld, cs.data(), ns.data(), ps.data(), sf.data(),
                                ds.data(), nn.data());
    SOA3D<Precision> work(m);
    nav.GetSafeties(gp, cs.data(), work, sf.data());
    for (size_t k = 0; k < m; ++k) {
      const int64_t i = ix[k];
      dist[i] = ds[k];
      safety[i] = sf[k];
      nextnode[i] = nn[k];
      newtop[i] = ns[k]->IsOutside() ? -1 : ns[k]->Top()->id();
      boundary[i] = ns[k]->IsOnBoundary() ? 1 : 0;
    }
  }
  for (int64_t i = 0; i < n; ++i) {
    NavigationState::ReleaseInstance(cur[i]);
    NavigationState::ReleaseInstance(nxt[i]);
  }
  NavigationState::ReleaseInstance(tmp);
  return 0;
}

// ---- ABBoxNavigator (navigation/ABBoxNavigator.h, source/ABBoxManager.cpp) ----
// ABBoxManager::ComputeABBox of one placed volume: lower xyz, upper xyz.
void vgref_abbox_compute(void *placed, double *out6) {
  ABBoxManager::ABBox_t lo, hi;
  ABBoxManager::ComputeABBox(static_cast<VPlacedVolume const *>(placed), &lo, &hi);
  for (int k = 0; k < 3; ++k) {
    out6[k] = lo[k];
    out6[3 + k] = hi[k];
  }
}

// ABBoxManager::InitABBoxesForCompleteGeometry, then the trace of
// vgref_nav_trace with ABBoxNavigator::FindNextBoundaryAndStep / GetSafety.
// Single-threaded: the reference's ABBoxManager shares one hit list
// (navigation/ABBoxNavigator.h:79, :128-130).
int vgref_abbox_nav_trace(int64_t ntracks, const double *x, const double *y, const double *z,
                          const double *dx, const double *dy, const double *dz, double pstep,
                          int max_steps, int *next_ids, double *steps, double *safeties,
                          int *nsteps) {
  ABBoxManager::Instance().InitABBoxesForCompleteGeometry();
  const int depth = GeoManager::Instance().getMaxDepth();
  VPlacedVolume const *world = GeoManager::Instance().GetWorld();
  ABBoxNavigator nav;
  SimpleNavigator locator;
  NavigationState *cur = NavigationState::MakeInstance(depth);
  NavigationState *nxt = NavigationState::MakeInstance(depth);
  for (int64_t i = 0; i < ntracks; ++i) {
    Vector3D<Precision> p(x[i], y[i], z[i]);
    Vector3D<Precision> d(dx[i], dy[i], dz[i]);
    cur->Clear();
    locator.LocatePoint(world, p, *cur, true);
    int k = 0;
    while (!cur->IsOutside() && k < max_steps) {
      double safety = nav.GetSafety(p, *cur);
      double step = 0;
      nxt->Clear();
      nav.FindNextBoundaryAndStep(p, d, *cur, *nxt, pstep, step);
      next_ids[i * max_steps + k] = nxt->IsOutside() ? -1 : nxt->Top()->id();
      steps[i * max_steps + k] = step;
      safeties[i * max_steps + k] = safety;
      p = p + d * step;
      std::swap(cur, nxt);
      ++k;
    }
    nsteps[i] = k;
  }
  NavigationState::ReleaseInstance(cur);
  NavigationState::ReleaseInstance(nxt);
  return 0;
}

// Single calls for known-answer checks: LocatePoint from the world, returning
// the id of Top() (-1 when outside) and the level.
int vgref_locate(double x, double y, double z, int *level) {
  const int depth = GeoManager::Instance().getMaxDepth();
  NavigationState *s = NavigationState::MakeInstance(depth);
  SimpleNavigator nav;
  nav.LocatePoint(GeoManager::Instance().GetWorld(), Vector3D<Precision>(x, y, z), *s, true);
  int id = s->IsOutside() ? -1 : s->Top()->id();
  *level = s->GetCurrentLevel();
  NavigationState::ReleaseInstance(s);
  return id;
}

} // extern "C"
