// polyhedron.cuh -- Polyhedron shape arithmetic (device), templated on the arithmetic type.
//
// A polyhedron is a stack of z-segments, each a set of planar quadrilaterals:
// the outer sides, the inner sides (when the segment has an inner radius) and
// the two phi-cutout faces (volumes/UnplacedPolyhedron.h, source/UnplacedPolyhedron.cpp:20-175,
// volumes/Quadrilaterals.h, volumes/Planes.h).  The operations follow
// volumes/kernel/PolyhedronImplementation.h (the scalar kernels the reference
// runs for every backend): bounding-tube rejection, z-segment walks and
// per-quadrilateral plane tests.  Placed polyhedra always take the generic
// transform (source/UnplacedPolyhedron.cpp:321-333).
//
// The record holds a header, then the segment table, the quadrilaterals, the z
// planes and the phi-section vectors; `base` is bound to the record's address
// at launch.
#pragma once
#include "tube.cuh"

namespace vgb {

// One quadrilateral: its plane (unit normal, distance to the origin), the four
// side planes bounding it and its four corners (volumes/Quadrilaterals.h:28-35).
// 33 doubles: the padding double makes consecutive quadrilaterals start 66
// 4-byte words apart, i.e. two shared-memory banks apart, so the lanes of a warp
// reading the quadrilaterals of different phi sides (the safety and distance
// walks do) hit different banks instead of all one (a 256-byte stride is a
// multiple of the 128-byte bank cycle).
struct PhQuad {
  double n[3];
  double d;
  double sn[4][3];
  double sd[4];
  double c[4][3];
  double pad;
};
static_assert(sizeof(PhQuad) == 33 * sizeof(double), "PhQuad stride");

// A z-segment: index ranges into the quadrilateral table.
struct PhSeg {
  int32_t outer_off, outer_n;
  int32_t inner_off, inner_n;
  int32_t phi_off, phi_n;
  int32_t has_inner;
  int32_t pad;
};

struct PolyhedronP {
  int32_t sides;
  int32_t nseg;        // z-segments = z planes - 1
  int32_t seg_off;     // doubles from the record start to the PhSeg table
  int32_t quad_off;    // ... to the PhQuad table
  int32_t zp_off;      // ... to the z planes (nseg + 1)
  int32_t phisec_off;  // ... to the phi-section vectors (3 * (sides + 1))
  int32_t has_inner_radii;
  int32_t has_phi_cutout;
  int32_t large_phi_cutout;
  int32_t pad;
  double btube_offset;
  TubeP btube;  // bounding tube; HollowTube kernels when has_inner_radii else NonHollowTube
  const double *base;
};

template <class R> struct PolyhedronOps {
  using T = TubeOps<R>;

  static VGB_HD const PhSeg &seg(const PolyhedronP &p, int i) {
    return reinterpret_cast<const PhSeg *>(p.base + p.seg_off)[i];
  }
  static VGB_HD const PhQuad &quad(const PolyhedronP &p, int i) {
    return reinterpret_cast<const PhQuad *>(p.base + p.quad_off)[i];
  }
  static VGB_HD R zplane(const PolyhedronP &p, int i) { return (R)p.base[p.zp_off + i]; }

  static VGB_HD R dot_n(const PhQuad &q, const V3<R> &v) {
    return v.x * (R)q.n[0] + v.y * (R)q.n[1] + v.z * (R)q.n[2];
  }

  // Planes::Contains (volumes/Planes.h:150-160) over a range of quadrilaterals
  static VGB_HD bool planes_contain(const PolyhedronP &p, int off, int n, const V3<R> &v) {
    bool result = true;
    for (int i = 0; i < n; ++i) {
      const PhQuad &q = quad(p, off + i);
      result &= dot_n(q, v) + (R)q.d < 0;
    }
    return result;
  }

  // Planes::Inside (volumes/Planes.h:200-218)
  static VGB_HD int planes_inside(const PolyhedronP &p, int off, int n, const V3<R> &v) {
    int result = kInside;
    for (int i = 0; i < n; ++i) {
      const PhQuad &q = quad(p, off + i);
      const R dr = (R)q.n[0] * v.x + (R)q.n[1] * v.y + (R)q.n[2] * v.z + (R)q.d;
      if (dr > (R)kTolerance) result = kOutside;
      if (result == kInside && dr > -(R)kTolerance) result = kSurface;
    }
    return result;
  }

  // Quadrilaterals::DistanceToIn<behindPlanes> (volumes/Quadrilaterals.h:218-257)
  template <bool Behind>
  static VGB_HD R quads_dti(const PolyhedronP &p, int off, int n, const V3<R> &pt, const V3<R> &dir) {
    R best = Lim<R>::inf();
    for (int i = 0; i < n; ++i) {
      const PhQuad &q = quad(p, off + i);
      R distance = dot_n(q, pt) + (R)q.d;
      bool valid = (Behind ? -distance : distance) >= 0;
      if (!valid) continue;
      const R proj = dot_n(q, dir);
      valid &= (Behind ? proj : -proj) >= 0;
      if (!valid) continue;
      distance /= -proj;
      const V3<R> ix = {pt.x + dir.x * distance, pt.y + dir.y * distance, pt.z + dir.z * distance};
      for (int j = 0; j < 4; ++j) {
        valid &= ix.x * (R)q.sn[j][0] + ix.y * (R)q.sn[j][1] + ix.z * (R)q.sn[j][2] + (R)q.sd[j] >= 0;
        if (!valid) break;
      }
      if (valid) best = distance;
      if (best < Lim<R>::inf()) break;
    }
    return best;
  }

  // Quadrilaterals::DistanceToOut(point, dir, zMin, zMax) (:318-352)
  static VGB_HD R quads_dto(const PolyhedronP &p, int off, int n, const V3<R> &pt, const V3<R> &dir,
                            R zMin, R zMax) {
    R best = Lim<R>::inf();
    for (int i = 0; i < n; ++i) {
      const PhQuad &q = quad(p, off + i);
      R dt = dot_n(q, pt) + (R)q.d;
      bool valid = dt < 0;
      if (!valid) continue;
      const R proj = dot_n(q, dir);
      valid &= proj >= 0;
      if (!valid) continue;
      // dt / -proj < best needs -dt < best * proj; a side farther than that by
      // more than the rounding of either side is rejected without the division
      // (best * 0 with best = inf is NaN, which never rejects)
      if (-dt > best * proj * (R)(1 + 1e-12)) continue;
      dt /= -proj;
      valid &= dt < best;
      if (!valid) continue;
      if (zMin == zMax) {
        const V3<R> ix = {pt.x + dt * dir.x, pt.y + dt * dir.y, pt.z + dt * dir.z};
        valid = true;
        for (int j = 0; j < 4; ++j) {  // RayHitsQuadrilateral (:60-68)
          valid &= ix.x * (R)q.sn[j][0] + ix.y * (R)q.sn[j][1] + ix.z * (R)q.sn[j][2] + (R)q.sd[j] >= 0;
          if (!valid) break;
        }
      } else {
        const R zp = pt.z + dt * dir.z;
        valid &= zp >= zMin && zp < zMax;
      }
      if (!valid) continue;
      best = dt;
    }
    return best;
  }

  // GenericKernels DistanceToLineSegmentSquared (volumes/kernel/GenericKernels.h:116-147)
  static VGB_HD R seg_dist2(const double *c0, const double *c1, const V3<R> &pt) {
    const R lx = (R)c1[0] - (R)c0[0], ly = (R)c1[1] - (R)c0[1], lz = (R)c1[2] - (R)c0[2];
    const R px = pt.x - (R)c0[0], py = pt.y - (R)c0[1], pz = pt.z - (R)c0[2];
    const R dot0 = px * lx + py * ly + pz * lz;
    if (dot0 <= 0) return px * px + py * py + pz * pz;
    const R dot1 = lx * lx + ly * ly + lz * lz;
    if (dot1 <= dot0) {
      const R qx = pt.x - (R)c1[0], qy = pt.y - (R)c1[1], qz = pt.z - (R)c1[2];
      const R r = qx * qx + qy * qy + qz * qz;
      if (r < Lim<R>::inf()) return r;
    }
    const R f = dot0 / dot1;
    const R ax = ((R)c0[0] + f * lx) - pt.x, ay = ((R)c0[1] + f * ly) - pt.y,
            az = ((R)c0[2] + f * lz) - pt.z;
    return ax * ax + ay * ay + az * az;
  }

  // Quadrilaterals::ScalarDistanceSquared (:361-395)
  static VGB_HD R quad_dist2(const PhQuad &q, const V3<R> &pt) {
    const R distance = dot_n(q, pt) + (R)q.d;
    const V3<R> ix = {pt.x + distance * (R)q.n[0], pt.y + distance * (R)q.n[1],
                      pt.z + distance * (R)q.n[2]};
    bool wb[4];
    for (int j = 0; j < 4; ++j)
      wb[j] = ix.x * (R)q.sn[j][0] + ix.y * (R)q.sn[j][1] + ix.z * (R)q.sn[j][2] + (R)q.sd[j] >= 0;
    if (wb[0] && wb[1] && wb[2] && wb[3]) return distance * distance;
    int a, b;
    if (!wb[0]) { a = 0; b = 1; }
    else if (!wb[2]) { a = 2; b = 3; }
    else if (!wb[1]) { a = 1; b = 2; }
    else { a = 3; b = 0; }
    return seg_dist2(q.c[a], q.c[b], pt);
  }

  // FindZSegmentKernel (:368-380): number of planes strictly below z, minus one
  static VGB_HD int find_z(const PolyhedronP &p, R z) {
    int index = -1;
    for (int i = 0; i <= p.nseg && z > zplane(p, i); ++i) ++index;
    return index;
  }

  // FindPhiSegment (:405-438)
  static VGB_HD int find_phi(const PolyhedronP &p, const V3<R> &pt) {
    const double *ps = p.base + p.phisec_off;
    int index = -1;
    R first = pt.x * (R)ps[0] + pt.y * (R)ps[1] + pt.z * (R)ps[2];
    for (int i = 1; i < p.sides + 1; ++i) {
      const R second = pt.x * (R)ps[3 * i] + pt.y * (R)ps[3 * i + 1] + pt.z * (R)ps[3 * i + 2];
      if (first >= 0 && second < 0) index = i - 1;
      if (index >= 0) break;
      first = second;
    }
    return index;
  }

  // InPhiCutoutWedge (:692-706)
  static VGB_HD bool in_cutout(const PolyhedronP &p, const PhSeg &s, const V3<R> &pt) {
    const PhQuad &q0 = quad(p, s.phi_off), &q1 = quad(p, s.phi_off + 1);
    const bool first = dot_n(q0, pt) + (R)q0.d >= 0;
    const bool second = dot_n(q1, pt) + (R)q1.d >= 0;
    if (p.large_phi_cutout) return first || second;
    return first && second;
  }

  static VGB_HD bool in_bounds(const PolyhedronP &p, const V3<R> &pt) {
    return T::contains(p.btube, {pt.x, pt.y, pt.z - (R)p.btube_offset});
  }

  // ScalarSegmentContainsKernel (:708-720)
  static VGB_HD bool segment_contains(const PolyhedronP &p, const V3<R> &pt, int zi) {
    const PhSeg &s = seg(p, zi);
    if (!planes_contain(p, s.outer_off, s.outer_n, pt)) return false;
    if (s.has_inner && planes_contain(p, s.inner_off, s.inner_n, pt)) return false;
    if (p.has_phi_cutout) {
      bool wi, wo;
      WedgeOps<R>::template contains_inside<false>(p.btube.wedge, pt.x, pt.y, wi, wo);
      if (wo) return false;
    }
    return true;
  }

  // ScalarContainsKernel (:722-740)
  static VGB_HD bool contains(const PolyhedronP &p, const V3<R> &pt) {
    if (!in_bounds(p, pt)) return false;
    const int zi = find_z(p, pt.z);
    if (!(zi >= 0)) return false;
    const PhSeg &s = seg(p, zi < p.nseg ? zi : p.nseg - 1);
    if (!planes_contain(p, s.outer_off, s.outer_n, pt)) return false;
    if (s.has_inner && planes_contain(p, s.inner_off, s.inner_n, pt)) return false;
    return true;
  }

  // ScalarInsideKernel (:742-773).  The reference indexes the segment without
  // clamping (a point within 1e-9 of the first or last z plane reads outside
  // its segment array); here the index is clamped to the nearest segment.
  static VGB_HD int inside(const PolyhedronP &p, const V3<R> &pt) {
    if (!in_bounds(p, pt)) return kOutside;
    int zi = find_z(p, pt.z);
    zi = zi < 0 ? 0 : (zi >= p.nseg ? p.nseg - 1 : zi);
    const PhSeg &s = seg(p, zi);
    const int io = planes_inside(p, s.outer_off, s.outer_n, pt);
    if (io != kInside) return io;
    if (s.has_inner) {
      const int ii = planes_inside(p, s.inner_off, s.inner_n, pt);
      if (ii == kInside) return kOutside;
      if (ii == kSurface) return kSurface;
    }
    if (p.has_phi_cutout && in_cutout(p, s, pt)) return kOutside;
    return kInside;
  }

  // DistanceToInZSegment (:440-470)
  static VGB_HD R dti_segment(const PolyhedronP &p, int zi, const V3<R> &pt, const V3<R> &dir) {
    const PhSeg &s = seg(p, zi);
    R distance = quads_dti<false>(p, s.outer_off, s.outer_n, pt, dir);
    bool done = distance < Lim<R>::inf();
    if (done) return distance;
    if (p.has_phi_cutout) distance = quads_dti<false>(p, s.phi_off, s.phi_n, pt, dir);
    done |= distance < Lim<R>::inf();
    if (done) return distance;
    if (s.has_inner) distance = quads_dti<true>(p, s.inner_off, s.inner_n, pt, dir);
    return distance;
  }

  // DistanceToOutZSegment (:472-500)
  static VGB_HD R dto_segment(const PolyhedronP &p, int zi, R zMin, R zMax, const V3<R> &pt,
                              const V3<R> &dir) {
    const PhSeg &s = seg(p, zi);
    bool done = false;
    R distance = Lim<R>::inf();
    if (s.has_inner) {
      distance = quads_dti<false>(p, s.inner_off, s.inner_n, pt, dir);
      done = distance < Lim<R>::inf();
      if (done) return distance;
    }
    if (p.has_phi_cutout) {
      const R distphi = quads_dti<true>(p, s.phi_off, s.phi_n, pt, dir);
      if (!done && distance >= (R)0.) distance = distphi;
      done = distance >= (R)0. && distance < Lim<R>::inf();
      if (done) return distance;
    }
    const R distout = quads_dto(p, s.outer_off, s.outer_n, pt, dir, zMin, zMax);
    if (!done) distance = distout;
    return distance;
  }

  // ScalarDistanceToEndcaps<pointInside> (:535-585)
  template <bool PointInside>
  static VGB_HD void to_endcaps(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R &distance) {
    int si, zi;
    if (PointInside) {
      if (dir.z < 0) { si = 0; zi = 0; }
      else { si = p.nseg - 1; zi = p.nseg; }
    } else {
      if (dir.z < 0) { si = p.nseg - 1; zi = p.nseg; }
      else { si = 0; zi = 0; }
    }
    const PhSeg &s = seg(p, si);
    const R dt = (zplane(p, zi) - pt.z) / dir.z;
    if (dt < 0 || dt >= distance) return;
    const V3<R> ix = {pt.x + dt * dir.x, pt.y + dt * dir.y, pt.z + dt * dir.z};
    if (!planes_contain(p, s.outer_off, s.outer_n, ix)) return;
    if (s.has_inner && planes_contain(p, s.inner_off, s.inner_n, ix)) return;
    if (p.has_phi_cutout && in_cutout(p, s, ix)) return;
    distance = dt;
  }

  // ScalarDistanceToInKernel (:775-827) and ScalarDistanceToOutKernel
  // (:851-890) as z-segment walks: *_begin does the set-up (and may settle the
  // point at once), each *_step evaluates one segment and says whether the walk
  // is over, *_end adds the endcaps and the step limit.  The batch kernel runs
  // the steps of many points interleaved (warp-regrouped); distance_to_in/out
  // run them in a loop: the same segments in the same order either way.  The
  // batch kernel applies the generic transform.
  struct Walk {
    int zi;
    bool right;
    R distance;
  };
  static VGB_HD bool dti_begin(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R smax,
                               Walk &w, R &res) {
    const V3<R> bp = {pt.x, pt.y, pt.z - (R)p.btube_offset};
    const bool inBounds = T::contains(p.btube, bp);
    if (!inBounds) {
      const R tubeDistance = T::distance_to_in(p.btube, bp, dir, smax);
      if (tubeDistance == Lim<R>::inf()) {
        res = Lim<R>::inf();
        return true;
      }
    }
    int zi = find_z(p, pt.z);
    const int zMax = p.nseg;
    zi = zi < 0 ? 0 : (zi >= zMax ? zMax - 1 : zi);
    if (inBounds && segment_contains(p, pt, zi)) {
      res = (R)-1.;
      return true;
    }
    w.zi = zi;
    w.right = dir.z >= 0;
    w.distance = Lim<R>::inf();
    return false;
  }
  static VGB_HD bool dti_step(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R,
                              Walk &w) {
    w.distance = dti_segment(p, w.zi, pt, dir);
    if (w.distance >= 0 && w.distance < Lim<R>::inf()) return true;
    if (w.right) return !(++w.zi < p.nseg);
    return !(--w.zi >= 0);
  }
  static VGB_HD R dti_end(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R smax,
                          const Walk &w) {
    R distance = w.distance;
    to_endcaps<false>(p, pt, dir, distance);
    return distance < smax ? distance : smax;
  }
  static VGB_HD R distance_to_in(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R smax) {
    Walk w;
    R r;
    if (dti_begin(p, pt, dir, smax, w, r)) return r;
    while (!dti_step(p, pt, dir, smax, w)) {
    }
    return dti_end(p, pt, dir, smax, w);
  }

  static VGB_HD bool dto_begin(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R,
                               Walk &w, R &) {
    int zi = find_z(p, pt.z);
    const int zMax = p.nseg;
    w.zi = zi < 0 ? 0 : (zi >= zMax ? zMax - 1 : zi);
    w.right = dir.z >= 0;
    w.distance = Lim<R>::inf();
    return false;
  }
  static VGB_HD bool dto_step(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R,
                              Walk &w) {
    const int zi = w.zi;
    w.distance = dto_segment(p, zi, zplane(p, zi), zplane(p, zi + 1), pt, dir);
    if (w.distance >= 0 && w.distance < Lim<R>::inf()) return true;
    if (w.right) {
      if (zplane(p, zi) - pt.z > w.distance) return true;
      return !(++w.zi < p.nseg);
    }
    if (pt.z - zplane(p, zi) > w.distance) return true;
    return !(--w.zi >= 0);
  }
  static VGB_HD R dto_end(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R smax,
                          const Walk &w) {
    R distance = w.distance;
    to_endcaps<true>(p, pt, dir, distance);
    return distance < smax ? distance : smax;
  }
  static VGB_HD R distance_to_out(const PolyhedronP &p, const V3<R> &pt, const V3<R> &dir, R smax) {
    Walk w;
    R r;
    if (dto_begin(p, pt, dir, smax, w, r)) return r;
    while (!dto_step(p, pt, dir, smax, w)) {
    }
    return dto_end(p, pt, dir, smax, w);
  }

  // ScalarSafetyToZSegmentSquared (:502-533)
  static VGB_HD R seg_safety2(const PolyhedronP &p, int zi, int phiIndex, const V3<R> &pt) {
    const PhSeg &s = seg(p, zi);
    if (p.has_phi_cutout && s.phi_n == 2 && in_cutout(p, s, pt))
      return vmin(quad_dist2(quad(p, s.phi_off), pt), quad_dist2(quad(p, s.phi_off + 1), pt));
    if (phiIndex < 0) return Lim<R>::inf();
    R outer = Lim<R>::inf();
    if (s.outer_n > 0) outer = quad_dist2(quad(p, s.outer_off + phiIndex), pt);
    R inner = Lim<R>::inf();
    if (s.has_inner && s.inner_n > 0) inner = quad_dist2(quad(p, s.inner_off + phiIndex), pt);
    return vmin(inner, outer);
  }

  // ScalarSafetyToEndcapsSquared (:587-612)
  static VGB_HD void endcaps_safety2(const PolyhedronP &p, const V3<R> &pt, R &d2) {
    const R firstDistance = zplane(p, 0) - pt.z;
    const R lastDistance = zplane(p, p.nseg) - pt.z;
    const bool isFirst = fabs(firstDistance) < fabs(lastDistance);
    const PhSeg &s = seg(p, isFirst ? 0 : p.nseg - 1);
    const R dt = isFirst ? firstDistance : lastDistance;
    const R dt2 = dt * dt;
    if (dt2 >= d2) return;
    const V3<R> ix = {pt.x, pt.y, pt.z + dt};
    if (!planes_contain(p, s.outer_off, s.outer_n, ix)) return;
    if (s.has_inner && planes_contain(p, s.inner_off, s.inner_n, ix)) return;
    if (p.has_phi_cutout && in_cutout(p, s, ix)) return;
    d2 = dt2;
  }

  // ScalarSafetyKernel (:829-849), used for SafetyToIn and SafetyToOut.  The
  // walk visits the segments the reference visits (its stopping rule compares the
  // z distance with the squared safety, and is kept) and returns the same minimum.
  // Every quadrilateral of segment z lies in the slab zplane(z) <= z <= zplane(z+1)
  // (its corners have those z values, except that a corner within 1e-9 of z = 0 is
  // set to 0) and each value seg_safety2 returns is the squared distance to a point
  // of one, so the squared z distance to the slab, less 2e-9 for those corners,
  // bounds it from below; where that bound exceeds the running minimum (with a
  // margin far above the rounding of either), the segment cannot lower the minimum
  // and is not evaluated.  vmin keeps its first argument against a NaN, so an
  // unevaluated NaN changes nothing either.
  static VGB_HD bool may_lower(R dz, R s) {
    const R lb = dz - (R)2e-9;
    return !(lb > 0 && lb * lb > s + (R)1e-6 * s + (R)1e-12);
  }
  static VGB_HD R safety(const PolyhedronP &p, const V3<R> &pt) {
    R s = Lim<R>::inf();
    const int zMax = p.nseg;
    int zi = find_z(p, pt.z);
    zi = zi < 0 ? 0 : (zi >= zMax ? zMax - 1 : zi);
    const int phiIndex = find_phi(p, pt);
    for (int z = zi; z < zMax;) {
      const R dz = vmax(zplane(p, z) - pt.z, pt.z - zplane(p, z + 1));
      if (may_lower(dz, s)) s = vmin(s, seg_safety2(p, z, phiIndex, pt));
      ++z;
      if (zplane(p, z) - pt.z > s) break;
    }
    for (int z = zi - 1; z >= 0; --z) {
      const R dz = vmax(zplane(p, z) - pt.z, pt.z - zplane(p, z + 1));
      if (may_lower(dz, s)) s = vmin(s, seg_safety2(p, z, phiIndex, pt));
      if (pt.z - zplane(p, z) > s) break;
    }
    endcaps_safety2(p, pt, s);
    return sqrt(s);
  }

  static VGB_HD R safety_to_in(const PolyhedronP &p, const V3<R> &pt) { return safety(p, pt); }
  static VGB_HD R safety_to_out(const PolyhedronP &p, const V3<R> &pt) { return safety(p, pt); }
};

}  // namespace vgb
