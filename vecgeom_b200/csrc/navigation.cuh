// navigation.cuh -- SimpleNavigator on the device: LocatePoint, RelocatePointFromPath,
// FindNextBoundaryAndStep and GetSafety over a flat geometry image.
//
// The per-track logic follows navigation/SimpleNavigator.h:204-596 step by
// step, so the next-volume sequence, the steps and the safeties are those of the
// reference.  The daughter loops are written over a group of lanes (the Lanes
// policy): on the GPU one warp serves one track and its 32 lanes share the
// daughters of the current volume; the minimum over the lanes keeps the
// reference's first-index tie rule, and the containment searches keep its
// order (first daughter for LocatePoint, last for LocatePointExclVolume) through
// warp ballots.  The host build runs the same code with a single lane.
//
// A DistanceToIn candidate is evaluated with the mother's step as its step
// limit rather than the running minimum the reference passes
// (SimpleNavigator.h:396-410).  The kernels only use the limit to return
// kInfinity early for rays that cannot beat it (box: safety >= limit), and a
// larger limit only turns such an early kInfinity into a distance that is no
// smaller than the running minimum at that daughter, so the first minimum, and
// with it the chosen daughter and the step, are unchanged.
#pragma once
#include "batch.cuh"
#include "geometry.h"

namespace vgb {

constexpr int kNavMaxLevels = 16;

// Device view of the geometry tables (all indices are placed / logical ids).
struct NavGeom {
  const double *params;         // shape parameter pool
  const UnplacedRec *unplaced;  // type + record offset per unplaced shape
  const PlacedRec *placed;      // unplaced, logical, effective and raw transform ids
  const DXform *xforms;         // effective transform of each placed volume's placed ops
  const NavXform *raw;          // per Transformation3D
  const LogicalRec *logicals;   // daughter range per logical volume
  const int32_t *daughters;     // CSR over logicals
  const float *pl_box;          // per placed: enclosing box in the mother's frame (6 floats)
  const float *ab_box;          // per placed: ABBoxManager's aligned box, float (6 floats)
  const float4 *ab_slot;        // per daughter slot (CSR order): lower, upper as float4
  int32_t world;
  int32_t max_depth;            // levels of the deepest path
};

// NavigationState in the reference's field layout (navigation/NavigationState.h:45-66,
// VecCore/inc/VariableSizeObj.h:25-31): int32 level @0, bool onBoundary @4,
// {selfAlloc:1, N:31} @8, then N path slots of 8 bytes @16.  On the device a
// slot holds the placed-volume index (int64) where the reference holds a pointer.
struct NavStateRef {
  unsigned char *p;
  VGB_HD int32_t &level() const { return *reinterpret_cast<int32_t *>(p); }
  VGB_HD uint8_t &boundary() const { return p[4]; }
  VGB_HD uint32_t &header() const { return *reinterpret_cast<uint32_t *>(p + 8); }
  VGB_HD int64_t &slot(int i) const { return reinterpret_cast<int64_t *>(p + 16)[i]; }
};
VGB_HD int64_t nav_state_stride(int max_depth) { return 16 + 8 * (int64_t)(max_depth + 1); }

// A path held in registers while a track is processed.
struct NavPath {
  int32_t level;
  bool boundary;
  int32_t v[kNavMaxLevels];
  VGB_HD int32_t top() const { return level > 0 ? v[level - 1] : -1; }
  VGB_HD void push(int32_t pv) { v[level++] = pv; }
  VGB_HD void pop() {
    if (level > 0) v[--level] = -1;
  }
};

VGB_HD void nav_load(NavPath &s, const NavStateRef &r) {
  s.level = r.level();
  s.boundary = r.boundary() != 0;
  for (int i = 0; i < kNavMaxLevels; ++i) s.v[i] = (i < s.level) ? (int32_t)r.slot(i) : -1;
}
VGB_HD void nav_store(const NavPath &s, const NavStateRef &r, int max_depth) {
  r.level() = s.level;
  r.boundary() = s.boundary ? 1 : 0;
  r.header() = (uint32_t)(max_depth + 1) << 1;
  for (int i = 0; i <= max_depth; ++i) r.slot(i) = (i < s.level) ? s.v[i] : -1;
}

// ---------------------------------------------------------------------------
// lanes: one warp per track on the GPU, one thread on the host
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
struct WarpLanes {
  static constexpr int N = 32;
  static VGB_D int lane() { return threadIdx.x & 31; }
  static VGB_D uint32_t ballot(bool b) { return __ballot_sync(0xffffffffu, b); }
  static VGB_D double shfl_xor(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
  static VGB_D int shfl_xor(int v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
  static VGB_D float shfl_xor(float v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
  static VGB_D double shfl_up(double v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
  static VGB_D uint32_t lanes_below() { return (1u << lane()) - 1u; }
  static VGB_D void sync() { __syncwarp(); }
};
#endif
struct OneLane {
  static constexpr int N = 1;
  static VGB_HD int lane() { return 0; }
  static VGB_HD uint32_t ballot(bool b) { return b ? 1u : 0u; }
  static VGB_HD double shfl_xor(double v, int) { return v; }
  static VGB_HD int shfl_xor(int v, int) { return v; }
  static VGB_HD float shfl_xor(float v, int) { return v; }
  static VGB_HD double shfl_up(double v, int) { return v; }
  static VGB_HD uint32_t lanes_below() { return 0u; }
  static VGB_HD void sync() {}
};

VGB_HD int nav_lowbit(uint32_t b) {
#ifdef __CUDA_ARCH__
  return __ffs(b) - 1;
#else
  return __builtin_ctz(b);
#endif
}
VGB_HD int nav_highbit(uint32_t b) {
#ifdef __CUDA_ARCH__
  return 31 - __clz(b);
#else
  return 31 - __builtin_clz(b);
#endif
}

VGB_HD int nav_popc(uint32_t b) {
#ifdef __CUDA_ARCH__
  return __popc(b);
#else
  return __builtin_popcount(b);
#endif
}

// (value, index) minimum; equal values keep the lower index, NaN never wins
VGB_HD void nav_min_merge(double &v, int &i, double ov, int oi) {
  if (ov < v || (ov == v && oi < i)) {
    v = ov;
    i = oi;
  }
}
template <class L> VGB_HD void nav_min_reduce(double &v, int &i) {
  for (int m = L::N / 2; m > 0; m >>= 1) {
    const double ov = L::shfl_xor(v, m);
    const int oi = L::shfl_xor(i, m);
    nav_min_merge(v, i, ov, oi);
  }
}

// ---------------------------------------------------------------------------
// shape dispatch over the shape types a geometry holds (kMask bit = type)
// ---------------------------------------------------------------------------
constexpr uint32_t kNavMaskAll = 0x3ffeu;  // types 1..13
constexpr uint32_t kNavMaskBoxTubeTrd =
    (1u << VGB_SHAPE_BOX) | (1u << VGB_SHAPE_TUBE) | (1u << VGB_SHAPE_TRD);

template <uint32_t kMask, class Ret, class Fn>
VGB_HD Ret nav_visit(const NavGeom &G, int32_t unplaced, Fn fn) {
  const int type = G.unplaced[unplaced].type;
  const double *rec = G.params + G.unplaced[unplaced].param_off;
#define VGB_NAV_VISIT(T, OPS, P)                                          \
  if constexpr ((kMask >> T) & 1u) {                                      \
    if (type == T) return fn(OPS<double>{}, bind_params(*reinterpret_cast<const P *>(rec), rec)); \
  }
  VGB_FOR_EACH_SHAPE(VGB_NAV_VISIT)
#undef VGB_NAV_VISIT
  return Ret{};
}

template <uint32_t kMask> struct NavShapes {
  using R = double;
  // VPlacedVolume::Contains(point, localPoint) (volumes/ShapeImplementationHelper.h:163-180)
  static VGB_HD bool contains(const NavGeom &G, int32_t pv, const V3<R> &p, V3<R> &local) {
    local = xf_point(G.xforms[G.placed[pv].xform], p);
    const V3<R> l = local;
    return nav_visit<kMask, bool>(G, G.placed[pv].unplaced,
                                  [&](auto o, const auto &s) { return decltype(o)::contains(s, l); });
  }
  static VGB_HD bool unplaced_contains(const NavGeom &G, int32_t pv, const V3<R> &l) {
    return nav_visit<kMask, bool>(G, G.placed[pv].unplaced,
                                  [&](auto o, const auto &s) { return decltype(o)::contains(s, l); });
  }
  static VGB_HD R distance_to_in(const NavGeom &G, int32_t pv, const V3<R> &p, const V3<R> &v,
                                 R smax) {
    const DXform &X = G.xforms[G.placed[pv].xform];
    return nav_visit<kMask, R>(G, G.placed[pv].unplaced, [&](auto o, const auto &s) {
      using O = decltype(o);
      return O::distance_to_in(s, xf_point(X, p), dti_dir<O>(X, v), smax);
    });
  }
  static VGB_HD R distance_to_out(const NavGeom &G, int32_t pv, const V3<R> &l, const V3<R> &v,
                                  R smax) {
    return nav_visit<kMask, R>(G, G.placed[pv].unplaced, [&](auto o, const auto &s) {
      return decltype(o)::distance_to_out(s, l, v, smax);
    });
  }
  static VGB_HD R safety_to_in(const NavGeom &G, int32_t pv, const V3<R> &p) {
    const DXform &X = G.xforms[G.placed[pv].xform];
    return nav_visit<kMask, R>(G, G.placed[pv].unplaced, [&](auto o, const auto &s) {
      return decltype(o)::safety_to_in(s, xf_point(X, p));
    });
  }
  static VGB_HD R safety_to_out(const NavGeom &G, int32_t pv, const V3<R> &l) {
    return nav_visit<kMask, R>(G, G.placed[pv].unplaced, [&](auto o, const auto &s) {
      return decltype(o)::safety_to_out(s, l);
    });
  }
};

// ---------------------------------------------------------------------------
// transforms
// ---------------------------------------------------------------------------
// Transformation3D::MultiplyFromRight (base/Transformation3D.h:674-743)
VGB_HD void nav_multiply_from_right(double t[3], double r[9], const NavXform &rhs) {
  if (rhs.flags & kNavIdentity) return;
  if (rhs.flags & kNavHasTrans) {
    for (int i = 0; i < 3; ++i) {
      t[i] = t[i] + r[3 * i + 0] * rhs.t[0];
      t[i] = t[i] + r[3 * i + 1] * rhs.t[1];
      t[i] = t[i] + r[3 * i + 2] * rhs.t[2];
    }
  }
  if (rhs.flags & kNavHasRot) {
    for (int i = 0; i < 3; ++i) {
      const double tx = r[3 * i + 0], ty = r[3 * i + 1], tz = r[3 * i + 2];
      r[3 * i + 0] = tx * rhs.r[0];
      r[3 * i + 1] = tx * rhs.r[1];
      r[3 * i + 2] = tx * rhs.r[2];
      r[3 * i + 0] = r[3 * i + 0] + ty * rhs.r[3];
      r[3 * i + 1] = r[3 * i + 1] + ty * rhs.r[4];
      r[3 * i + 2] = r[3 * i + 2] + ty * rhs.r[5];
      r[3 * i + 0] = r[3 * i + 0] + tz * rhs.r[6];
      r[3 * i + 1] = r[3 * i + 1] + tz * rhs.r[7];
      r[3 * i + 2] = r[3 * i + 2] + tz * rhs.r[8];
    }
  }
}

// NavigationState::TopMatrix (navigation/NavigationState.h:401-408): the product
// of the transforms of path[1..level-1], applied with Transform<kGeneric,kGeneric>.
VGB_HD DXform nav_top_matrix(const NavGeom &G, const NavPath &s) {
  DXform m;
  for (int i = 0; i < 3; ++i) m.t[i] = 0.;
  for (int i = 0; i < 9; ++i) m.r[i] = (i % 4 == 0) ? 1. : 0.;
  for (int i = 1; i < s.level; ++i) nav_multiply_from_right(m.t, m.r, G.raw[G.placed[s.v[i]].raw_xform]);
  m.flags = kXfHasTrans | kXfHasRot;
  m.pad = 0;
  return m;
}

// Transform<kGeneric,kGeneric> of a raw transformation
VGB_HD V3<double> nav_generic_point(const NavXform &X, const V3<double> &p) {
  DXform d;
  for (int i = 0; i < 3; ++i) d.t[i] = X.t[i];
  for (int i = 0; i < 9; ++i) d.r[i] = X.r[i];
  d.flags = kXfHasTrans | kXfHasRot;
  d.pad = 0;
  return xf_point(d, p);
}

// InverseTransform (base/Transformation3D.h:598-632)
VGB_HD V3<double> nav_inverse_point(const NavXform &X, const V3<double> &l) {
  V3<double> m;
  m.x = X.t[0];
  m.x = m.x + l.x * X.r[0];
  m.x = m.x + l.y * X.r[1];
  m.x = m.x + l.z * X.r[2];
  m.y = X.t[1];
  m.y = m.y + l.x * X.r[3];
  m.y = m.y + l.y * X.r[4];
  m.y = m.y + l.z * X.r[5];
  m.z = X.t[2];
  m.z = m.z + l.x * X.r[6];
  m.z = m.z + l.y * X.r[7];
  m.z = m.z + l.z * X.r[8];
  return m;
}

// ---------------------------------------------------------------------------
// float screen of the FP32+refine form (ABBoxNavigator's idea, kept exact)
// ---------------------------------------------------------------------------
// A daughter's DistanceToIn is only needed when it can beat the running best:
// a ray that misses the daughter's widened box in the mother's frame, or enters
// it beyond best, cannot (the box encloses the shape; the widening, 1e-3 mm +
// 1e-5 of the coordinates, and the relative margin below cover float rounding),
// so the FP64 call is skipped and the result is unchanged.
struct RayF {
  float p[3], inv[3];
  bool flat[3];
};
VGB_HD RayF ray_f(const V3<double> &p, const V3<double> &d) {
  RayF r;
  const double pp[3] = {p.x, p.y, p.z}, dd[3] = {d.x, d.y, d.z};
  for (int k = 0; k < 3; ++k) {
    r.p[k] = (float)pp[k];
    r.flat[k] = fabs(dd[k]) < 1e-30;
    r.inv[k] = r.flat[k] ? 0.f : (float)(1.0 / dd[k]);
  }
  return r;
}
// true when the box cannot hold a hit closer than `best`
VGB_HD bool box_skips(const float *b, const RayF &r, double best) {
  float tn = 0.f, tf = 3.0e38f;
  for (int k = 0; k < 3; ++k) {
    if (r.flat[k]) {
      if (r.p[k] < b[k] || r.p[k] > b[3 + k]) return true;
      continue;
    }
    float t1 = (b[k] - r.p[k]) * r.inv[k], t2 = (b[3 + k] - r.p[k]) * r.inv[k];
    if (t1 > t2) {
      const float t = t1;
      t1 = t2;
      t2 = t;
    }
    tn = tn > t1 ? tn : t1;
    tf = tf < t2 ? tf : t2;
  }
  if (tn > tf * 1.0001f + 1e-4f) return true;  // misses the box
  const float bf = best < 3.0e38 ? (float)best : 3.0e38f;
  return tn > bf * 1.0001f + 1e-3f;             // enters it beyond best
}

// Lower bound of a box daughter's SafetyToIn (BoxImplementation.h:801-818,
// max_i |l_i| - d_i) in float, minus a margin covering the float rounding of
// the transform and the subtraction.
VGB_HD float box_safety_lower(const BoxP &b, const DXform &X, const V3<double> &p) {
  const float ax = (float)(p.x - X.t[0]), ay = (float)(p.y - X.t[1]), az = (float)(p.z - X.t[2]);
  const bool tr = X.flags & kXfHasTrans;
  const float px = tr ? ax : (float)p.x, py = tr ? ay : (float)p.y, pz = tr ? az : (float)p.z;
  float lx = px, ly = py, lz = pz;
  if (X.flags & kXfHasRot) {
    lx = px * (float)X.r[0] + py * (float)X.r[3] + pz * (float)X.r[6];
    ly = px * (float)X.r[1] + py * (float)X.r[4] + pz * (float)X.r[7];
    lz = px * (float)X.r[2] + py * (float)X.r[5] + pz * (float)X.r[8];
  }
  float s = fabsf(lx) - (float)b.d[0];
  s = fmaxf(s, fabsf(ly) - (float)b.d[1]);
  s = fmaxf(s, fabsf(lz) - (float)b.d[2]);
  const float scale = fabsf(px) + fabsf(py) + fabsf(pz) + (float)(b.d[0] + b.d[1] + b.d[2]);
  return s - (1e-3f + 1e-5f * scale);
}

// ---------------------------------------------------------------------------
// the navigator
// ---------------------------------------------------------------------------
template <class L, uint32_t kMask, bool kScreen = false> struct Navigator {
  using R = double;
  using S = NavShapes<kMask>;

  // Descends from `vol` (already pushed) through the first (kFirst) or last
  // daughter containing the point, as LocatePoint (:204-240) and
  // LocatePointExclVolume (:246-283) do.  Returns false if the path would
  // exceed kNavMaxLevels.
  template <bool kFirst>
  static VGB_HD bool descend(const NavGeom &G, NavPath &s, int32_t vol, V3<R> tmp,
                             int32_t excluded) {
    int32_t cand = vol;
    for (;;) {
      const LogicalRec &lr = G.logicals[G.placed[cand].logical];
      const int32_t nd = lr.dcount;
      if (nd == 0) return true;
      const int32_t *dl = G.daughters + lr.dfirst;
      int found = -1;
      if (kFirst) {
        for (int base = 0; base < nd && found < 0; base += L::N) {
          const int d = base + L::lane();
          V3<R> loc;
          const bool hit = d < nd && dl[d] != excluded && S::contains(G, dl[d], tmp, loc);
          const uint32_t b = L::ballot(hit);
          if (b) found = base + nav_lowbit(b);
        }
      } else {
        for (int top = nd; top > 0 && found < 0; top -= L::N) {
          const int base = top - L::N;  // lanes base..top-1, some below 0
          const int d = base + L::lane();
          V3<R> loc;
          const bool hit = d >= 0 && dl[d] != excluded && S::contains(G, dl[d], tmp, loc);
          const uint32_t b = L::ballot(hit);
          if (b) found = base + nav_highbit(b);
        }
      }
      if (found < 0) return true;
      if (s.level >= kNavMaxLevels) return false;
      V3<R> loc;
      S::contains(G, dl[found], tmp, loc);
      s.push(dl[found]);
      tmp = loc;
      cand = dl[found];
    }
  }

  // LocatePoint(world, point, path, top=true)
  static VGB_HD bool locate_from_world(const NavGeom &G, NavPath &s, const V3<R> &p) {
    s.level = 0;
    s.boundary = false;
    for (int i = 0; i < kNavMaxLevels; ++i) s.v[i] = -1;
    if (!S::unplaced_contains(G, G.world, p)) return true;
    s.push(G.world);
    return descend<true>(G, s, G.world, p, -1);
  }

  // RelocatePointFromPath (:286-318)
  static VGB_HD bool relocate_from_path(const NavGeom &G, NavPath &s, V3<R> tmp) {
    int32_t mother = s.top();
    if (mother < 0) return true;
    while (mother >= 0 && !S::unplaced_contains(G, mother, tmp)) {
      s.pop();
      tmp = nav_inverse_point(G.raw[G.placed[mother].raw_xform], tmp);
      mother = s.top();
    }
    if (mother >= 0) {
      s.pop();
      s.push(mother);
      return descend<false>(G, s, mother, tmp, mother);
    }
    return true;
  }

  // GetSafety (:572-596) in the frame of the top volume
  static VGB_HD R safety(const NavGeom &G, const NavPath &s, const V3<R> &lp) {
    const int32_t cv = s.top();
    R best = S::safety_to_out(G, cv, lp);
    int bi = -1;
    const LogicalRec &lr = G.logicals[G.placed[cv].logical];
    const int32_t nd = lr.dcount;
    const int32_t *dl = G.daughters + lr.dfirst;
    // std::min(safety, tmp): a daughter replaces the running value only when
    // strictly smaller; NaN never replaces and a NaN mother value stays
    if (best == best) {
      R mine = best;
      int mi = -1;
      for (int d = L::lane(); d < nd; d += L::N) {
        if constexpr (kScreen && ((kMask >> VGB_SHAPE_BOX) & 1u)) {
          // a box daughter whose safety is certainly >= the running minimum
          // cannot replace it (strict <; the lane's earlier daughters hold it)
          const PlacedRec &pr = G.placed[dl[d]];
          const UnplacedRec &ur = G.unplaced[pr.unplaced];
          if (ur.type == VGB_SHAPE_BOX &&
              (double)box_safety_lower(*reinterpret_cast<const BoxP *>(G.params + ur.param_off),
                                       G.xforms[pr.xform], lp) >= mine)
            continue;
        }
        const R t = S::safety_to_in(G, dl[d], lp);
        if (t < mine) {
          mine = t;
          mi = d;
        }
      }
      nav_min_reduce<L>(mine, mi);
      best = mine;
      bi = mi;
    }
    (void)bi;
    return best;
  }

  // The basket form of FindNextBoundaryAndStep (:637-743) for one track: the
  // mother's DistanceToOut with its node index (-1 leaves within pstep, -2
  // stays; volumes/ShapeImplementationHelper.h:676-692), every daughter's
  // DistanceToInMinimize (:637-658: a strictly smaller distance takes the
  // daughter's index), then the relocation with a 1e-9 push.  Unlike the
  // single-track form there is no special case for a negative or infinite
  // distance.  The lanes share the daughters as in step().
  static VGB_HD bool step_basket(const NavGeom &G, const NavPath &cur, NavPath &next,
                                 const V3<R> &lp, const V3<R> &ld, R pstep, R &dist_out,
                                 int32_t &node_out) {
    const int32_t cv = cur.top();
    const R mother = S::distance_to_out(G, cv, lp, ld, pstep);
    const LogicalRec &lr = G.logicals[G.placed[cv].logical];
    const int32_t nd = lr.dcount;
    const int32_t *dl = G.daughters + lr.dfirst;
    R best = mother;
    int bi = mother < pstep ? -1 : -2;
    R mine = mother;
    int mi = 0x7fffffff;
    for (int d = L::lane(); d < nd; d += L::N) {
      const R dd = S::distance_to_in(G, dl[d], lp, ld, mother);
      if (dd < mine) {
        mine = dd;
        mi = d;
      }
    }
    nav_min_reduce<L>(mine, mi);
    if (mine < best) {
      best = mine;
      bi = mi;
    }
    dist_out = best;
    node_out = bi;
    next = cur;
    if (best > pstep) {
      dist_out = pstep;
      next.boundary = false;
      return true;
    }
    next.boundary = true;
    const R s9 = best + (R)1e-9;
    V3<R> np = {ld.x * s9, ld.y * s9, ld.z * s9};
    np = {np.x + lp.x, np.y + lp.y, np.z + lp.z};
    if (bi > -1) {
      const int32_t nv = dl[bi];
      if (next.level >= kNavMaxLevels) return false;
      next.push(nv);
      return descend<true>(G, next, nv, nav_generic_point(G.raw[G.placed[nv].raw_xform], np), -1);
    }
    return relocate_from_path(G, next, np);
  }

  // FindNextBoundaryAndStep (:340-470).  `next` is updated in place from `cur`.
  // Returns false if a path would exceed kNavMaxLevels.
  static VGB_HD bool step(const NavGeom &G, const NavPath &cur, NavPath &next, const V3<R> &lp,
                          const V3<R> &ld, R pstep, R &step_out) {
    const int32_t cv = cur.top();
    R step = S::distance_to_out(G, cv, lp, ld, pstep);
    if (step <= 0.) step = Lim<R>::inf();
    const LogicalRec &lr = G.logicals[G.placed[cv].logical];
    const int32_t nd = lr.dcount;
    const int32_t *dl = G.daughters + lr.dfirst;
    R best = step;
    int bi = -1;
    RayF rf;
    if constexpr (kScreen) rf = ray_f(lp, ld);
    for (int d = L::lane(); d < nd; d += L::N) {
      if constexpr (kScreen) {
        if (box_skips(G.pl_box + 6 * (int64_t)dl[d], rf, best)) continue;
      }
      const R dd = S::distance_to_in(G, dl[d], lp, ld, step);
      const bool valid = dd < best && !isinf(dd);
      if (valid) {
        best = dd;
        bi = d;
      }
    }
    nav_min_reduce<L>(best, bi);
    step = best;
    const int hit = bi;

    next = cur;
    if (step == Lim<R>::inf() && pstep > 0.) {
      step_out = 0.;
      next.pop();
      next.boundary = true;
      return true;
    }
    if (step > pstep) {
      step_out = pstep;
      next.boundary = false;
      return true;
    }
    next.boundary = true;
    if (step < 0.) step = 0.;
    step_out = step;
    const R s6 = step + (R)1e-6;
    V3<R> np = {ld.x * s6, ld.y * s6, ld.z * s6};
    np = {np.x + lp.x, np.y + lp.y, np.z + lp.z};
    if (hit != -1) {
      const int32_t nv = dl[hit];
      if (next.level >= kNavMaxLevels) return false;
      next.push(nv);
      return descend<true>(G, next, nv, nav_generic_point(G.raw[G.placed[nv].raw_xform], np), -1);
    }
    return relocate_from_path(G, next, np);
  }
};

}  // namespace vgb
