// polycone.cuh -- Polycone shape arithmetic (device), templated on the arithmetic type.
//
// A polycone is a z-ordered stack of cone sections (volumes/UnplacedPolycone.h:32-124,
// source/UnplacedPolycone.cpp:22-165); every operation walks the sections as
// volumes/kernel/PolyconeImplementation.h does, calling the cone arithmetic of
// cone.cuh on the point shifted into the section frame.  The section table sits
// in the geometry's parameter pool right after this header; `base` is bound to
// the record's address when the kernel is launched.
#pragma once
#include "cone.cuh"

namespace vgb {

// 41 doubles (82 4-byte words): consecutive sections start 18 words apart, so
// up to 16 sections map to distinct shared-memory banks when the lanes of a
// warp read different sections (a 40-double record put every other section on
// the same bank).
struct PolySec {
  ConeP cone;    // UnplacedCone(prevRmin, prevRmax, rMin, rMax, dz, phiStart, phiTotal)
  double shift;  // fShift: z of the section centre
  double pad[2];
};
static_assert(sizeof(PolySec) == 41 * sizeof(double), "PolySec stride");

struct PolyconeP {
  int32_t nsec;
  int32_t sec_off;  // doubles from the record start to the PolySec array
  int32_t zs_off;   // doubles from the record start to fZs (nsec + 1 values)
  int32_t pad;
  const double *base;  // record address, bound at launch (device) or by host callers
};

template <class R> struct PolyconeOps {
  using C = ConeOps<R>;

  static VGB_HD const PolySec &sec(const PolyconeP &p, int i) {
    return reinterpret_cast<const PolySec *>(p.base + p.sec_off)[i];
  }
  static VGB_HD R zs(const PolyconeP &p, int i) { return (R)p.base[p.zs_off + i]; }

  // UnplacedPolycone::GetSectionIndex (volumes/UnplacedPolycone.h:113-124)
  static VGB_HD int section_index(const PolyconeP &p, R z) {
    if (z < zs(p, 0)) return -1;
    for (int i = 0; i < p.nsec; ++i)
      if (z >= zs(p, i) && z <= zs(p, i + 1)) return i;
    return -2;
  }

  static VGB_HD V3<R> shifted(const V3<R> &q, const PolySec &s) {
    return {q.x - (R)0, q.y - (R)0, q.z - (R)s.shift};
  }

  // ContainsKernel (:52-72)
  static VGB_HD bool contains(const PolyconeP &p, const V3<R> &q) {
    if (q.z < zs(p, 0) || q.z > zs(p, p.nsec)) return false;
    const PolySec &s = sec(p, section_index(p, q.z));
    return C::contains(s.cone, shifted(q, s));
  }

  // InsideKernel (:74-88): kInside or kOutside only
  static VGB_HD int inside(const PolyconeP &p, const V3<R> &q) {
    return contains(p, q) ? kInside : kOutside;
  }

  // DistanceToIn (:125-165) as a section walk: dti_begin picks the first
  // section and the direction, each dti_step evaluates one section and says
  // whether the walk is over (a finite distance, no z motion, or no section
  // left), dti_end returns the distance.  The batch kernel runs the steps of
  // many points interleaved (warp-regrouped), distance_to_in runs them in a
  // loop: the same sections in the same order either way.
  struct Walk {
    int index, increment;
    R distance;
    // DistanceToOut: the distance so far, the steps taken, the point in the
    // current section's frame
    int istep;
    R total;
    V3<R> pn;
  };
  static VGB_HD bool dti_begin(const PolyconeP &p, const V3<R> &q, const V3<R> &v, R,
                               Walk &w, R &) {
    w.increment = (v.z > 0) ? 1 : -1;
    if (fabs(v.z) < (R)kTolerance) w.increment = 0;
    w.index = section_index(p, q.z);
    if (w.index == -1) w.index = 0;
    if (w.index == -2) w.index = p.nsec - 1;
    w.distance = Lim<R>::inf();
    return false;
  }
  // Every finite answer of the cone's DistanceToIn is a point of the section's
  // surface: a z face point within the section's radii, a cone root inside the z
  // slab, or a phi plane point within the radii; so it lies in the slab (widened
  // by the tolerance) within the section's larger outer radius.  A ray that stays
  // farther from the z axis than that radius while it crosses the slab, both
  // widened by margins far above the rounding of either computation, gets
  // kInfinity from the section: the walk skips that evaluation and goes on as
  // after an infinite answer.  (The same test inside the single cone's
  // DistanceToIn, which rejects such rays cheaply on its own, measured slower.)
  static VGB_HD bool out_of_reach(const PolySec &s, const V3<R> &q, const V3<R> &v) {
    // the cone arithmetic takes v as a unit vector (1 - v.z^2 for v.x^2 + v.y^2);
    // for any other v (the reference's 0x16A rotation code hands one over) its
    // answers are not points of the surface along the ray, so it is evaluated
    if (!(fabs(v.x * v.x + v.y * v.y + v.z * v.z - (R)1) < (R)1e-10)) return false;
    const R dz = (R)s.cone.dz, zc = (R)s.shift;
    const R mz = (R)1e-3 + (R)1e-6 * (fabs(zc) + dz);
    const R rmax = vmax((R)s.cone.rmax1, (R)s.cone.rmax2);
    return ray_beyond_radius(q, v, zc - dz - mz, zc + dz + mz, rmax + (R)1e-3 + (R)1e-6 * rmax);
  }

  static VGB_HD bool dti_step(const PolyconeP &p, const V3<R> &q, const V3<R> &v, R smax,
                              Walk &w) {
    const PolySec &s = sec(p, w.index);
    w.distance = out_of_reach(s, q, v) ? Lim<R>::inf()
                                       : C::distance_to_in(s.cone, shifted(q, s), v, smax);
    if (w.distance < Lim<R>::inf() || !w.increment) return true;
    w.index += w.increment;
    return !(w.index >= 0 && w.index < p.nsec);
  }
  static VGB_HD R dti_end(const PolyconeP &, const V3<R> &, const V3<R> &, R, const Walk &w) {
    return w.distance;
  }
  static VGB_HD R distance_to_in(const PolyconeP &p, const V3<R> &q, const V3<R> &v, R smax) {
    Walk w;
    R r;
    if (dti_begin(p, q, v, smax, w, r)) return r;
    while (!dti_step(p, q, v, smax, w)) {
    }
    return dti_end(p, q, v, smax, w);
  }

  // DistanceToOut (:167-292) as a section walk, like DistanceToIn: dto_begin
  // finds the starting section (and settles single-section polycones and points
  // in no section), each dto_step runs one section of the loop body and says
  // whether the walk is over, dto_end returns the accumulated distance.
  static VGB_HD bool dto_begin(const PolyconeP &p, const V3<R> &q, const V3<R> &v, R smax,
                               Walk &w, R &res) {
    if (p.nsec == 1) {
      const PolySec &s = sec(p, 0);
      res = C::distance_to_out(s.cone, shifted(q, s), v, smax);
      return true;
    }
    const int indexLow = section_index(p, q.z - (R)kTolerance);
    const int indexHigh = section_index(p, q.z + (R)kTolerance);
    int index;
    if (indexLow != indexHigh && (indexLow >= 0)) {
      const PolySec &s = sec(p, indexLow);
      index = C::contains(s.cone, shifted(q, s)) ? indexLow : indexHigh;
    } else {
      index = indexLow;
      if (index < 0) index = section_index(p, q.z);
    }
    if (index < 0) {
      res = (R)0.;
      return true;
    }
    w.index = index;
    w.total = 0.;
    w.increment = (v.z > 0) ? 1 : -1;
    if (fabs(v.z) < (R)kTolerance) w.increment = 0;
    w.istep = 0;
    w.pn = q;
    return false;
  }
  static VGB_HD bool dto_step(const PolyconeP &p, const V3<R> &q, const V3<R> &v, R smax,
                              Walk &w) {
    const PolySec &s = sec(p, w.index);
    if ((w.total != 0) || (w.istep < 2)) {
      w.pn = {q.x + w.total * v.x, q.y + w.total * v.y, q.z + w.total * v.z};
      w.pn.z = w.pn.z - (R)s.shift;
      if (C::inside(s.cone, w.pn) == kOutside) return true;
    } else {
      w.pn.z = w.pn.z - (R)s.shift;
    }
    w.istep++;
    const R dist = C::distance_to_out(s.cone, w.pn, v, smax);
    if (fabs(dist) < (R)0.5 * (R)kTolerance) {
      int index1 = w.index;
      if ((w.index > 0) && (w.index < p.nsec - 1)) {
        index1 += w.increment;
      } else {
        if ((w.index == 0) && (w.increment > 0)) index1 += w.increment;
        if ((w.index == p.nsec - 1) && (w.increment < 0)) index1 += w.increment;
      }
      const R td = w.total + dist;
      V3<R> pte = {q.x + td * v.x, q.y + td * v.y, q.z + td * v.z};
      const PolySec &s1 = sec(p, index1);
      pte.z = pte.z - (R)s1.shift;
      if (!C::contains(s1.cone, pte)) return true;
    }
    w.total += dist;
    w.index += w.increment;
    return !(w.increment != 0 && w.index >= 0 && w.index < p.nsec);
  }
  static VGB_HD R dto_end(const PolyconeP &, const V3<R> &, const V3<R> &, R, const Walk &w) {
    return w.total;
  }
  static VGB_HD R distance_to_out(const PolyconeP &p, const V3<R> &q, const V3<R> &v, R smax) {
    Walk w;
    R r;
    if (dto_begin(p, q, v, smax, w, r)) return r;
    while (!dto_step(p, q, v, smax, w)) {
    }
    return dto_end(p, q, v, smax, w);
  }

  static VGB_HD R safety_to_in(const PolyconeP &p, const V3<R> &q) {
    int index = section_index(p, q.z);
    bool needZ = false;
    if (index < 0) {
      needZ = true;
      if (index == -1) index = 0;
      if (index == -2) index = p.nsec - 1;
    }
    const PolySec &s = sec(p, index);
    if (needZ) return C::template safety_to_in_impl<false>(s.cone, shifted(q, s));
    R safety = C::template safety_to_in_impl<true>(s.cone, shifted(q, s));
    if (safety < (R)kTolerance) return safety;
    R minSafety = safety;
    R zbase = zs(p, index + 1);
    for (int i = index + 1; i < p.nsec; ++i) {
      const R dz = zs(p, i) - zbase;
      if (dz >= minSafety) break;
      const PolySec &si = sec(p, i);
      safety = C::template safety_to_in_impl<false>(si.cone, shifted(q, si));
      if (safety < minSafety) minSafety = safety;
    }
    if (index > 0) {  // the reference reads fZs[index-1] unconditionally; unused when index == 0
      zbase = zs(p, index - 1);
      for (int i = index - 1; i >= 0; --i) {
        const R dz = zbase - zs(p, i);
        if (dz >= minSafety) break;
        const PolySec &si = sec(p, i);
        safety = C::template safety_to_in_impl<false>(si.cone, shifted(q, si));
        if (safety < minSafety) minSafety = safety;
      }
    }
    return minSafety;
  }

  // SafetyToOut (:431-476)
  static VGB_HD R safety_to_out(const PolyconeP &p, const V3<R> &q) {
    const int index = section_index(p, q.z);
    if (index < 0) return (R)0;
    const PolySec &s = sec(p, index);
    R safety = C::template safety_to_out_impl<false>(s.cone, shifted(q, s));
    R minSafety = safety;
    if (minSafety == Lim<R>::inf()) return (R)0.;
    if (minSafety < (R)kTolerance) return (R)0.;
    R zbase = zs(p, index + 1);
    for (int i = index + 1; i < p.nsec; ++i) {
      const R dz = zs(p, i) - zbase;
      if (dz >= minSafety) break;
      const PolySec &si = sec(p, i);
      safety = C::template safety_to_in_impl<false>(si.cone, shifted(q, si));
      if (safety < minSafety) minSafety = safety;
    }
    if (index > 0) {
      zbase = zs(p, index - 1);
      for (int i = index - 1; i >= 0; --i) {
        const R dz = zbase - zs(p, i);
        if (dz >= minSafety) break;
        const PolySec &si = sec(p, i);
        safety = C::template safety_to_in_impl<false>(si.cone, shifted(q, si));
        if (safety < minSafety) minSafety = safety;
      }
    }
    return minSafety;
  }
};

}  // namespace vgb
