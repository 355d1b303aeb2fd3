// abbox.cuh -- ABBoxNavigator on the device: FindNextBoundaryAndStep with the
// daughters culled by their aligned bounding boxes and visited in the order of
// their box distance (navigation/ABBoxNavigator.h:200-420,
// source/ABBoxManager.cpp:88-126).
//
// Per step the reference
//   1. takes the mother's DistanceToOut (a negative value becomes kInfinity),
//   2. intersects the ray, in float, with the aligned box of every daughter
//      (ABBoxManager's boxes: the daughter's Extent moved into the mother's
//      frame, widened by 1e-3 and rounded to float) and lists the hits with
//      their entry distance b (negative when the point is inside the box),
//   3. sorts the list by b and walks it while b <= step: a daughter whose box
//      holds the point (b < 0) and that contains the point ends the walk with
//      step 0 and that daughter; otherwise its DistanceToIn (limited by the
//      running step) replaces the step when strictly smaller,
//   4. then decides the new state as ABBoxNavigator.h:327-420 does (which
//      differs from SimpleNavigator in its treatment of an infinite step and
//      of a relocation that ends in the volume it left).
//
// On the GPU one warp serves one track.  The lanes test the boxes in parallel
// and compact the hits, in daughter order (the order the reference pushes
// them), into a per-warp list in shared memory.  The list is then ordered as
// the reference's std::sort orders it: lists of up to 16 hits by rank (libstdc++
// sorts them by insertion, which keeps equal box distances in daughter order),
// longer ones by one lane with a restatement of libstdc++'s introsort (below),
// since its partitioning decides the order of equal box distances.  The
// sorted walk runs 32 candidates at a time: every lane evaluates its candidate
// (Contains when b < 0, else DistanceToIn with the running step at the start
// of the group as its limit), a warp prefix minimum gives each lane the step
// the reference holds when it reaches that candidate, the first lane where the
// reference stops (b above that step, or a containing box) ends the walk, and
// the minimum over the lanes before it, first lane on ties, is the reference's
// last strict improvement.  A DistanceToIn limit above the reference's only
// changes results that cannot improve the step (the kernels use the limit for
// early kInfinity returns only), so the outcome is the reference's.
//
// A list longer than the shared buffer is walked one candidate at a time, each
// the smallest (b, daughter index) above the previous one (a warp reduction
// over the mother's daughters per visit).  That order equals std::sort's
// unless such a list holds equal box distances, which then are visited in
// daughter order.
#pragma once
#include "navigation.cuh"

namespace vgb {

// one hit: box entry distance and the daughter's position in its mother's list
struct AbCand {
  float b;
  int32_t d;
};

// (box distance, daughter index): the order of the one-by-one walk and of the
// rank sort of short lists
VGB_HD bool ab_less(const AbCand &a, const AbCand &b) {
  return a.b < b.b || (a.b == b.b && a.d < b.d);
}

// ---------------------------------------------------------------------------
// std::sort(hits, HitBoxComparatorFunctor) as GCC's libstdc++ carries it out
// (the reference build's standard library): introsort over [0, n) with
// depth limit 2 floor(log2 n), ranges of more than 16 elements partitioned
// around the median of (second, middle, last) moved to the front (Hoare's
// unguarded scheme), heapsort for a range that reaches the depth limit, and
// one insertion pass at the end (guarded over the first 16, unguarded after).
// Only the box distance is compared, as HitBoxComparatorFunctor does.
// ---------------------------------------------------------------------------
VGB_HD bool ab_key_less(const AbCand &a, const AbCand &b) { return a.b < b.b; }

VGB_HD void ab_swap(AbCand *a, int i, int j) {
  const AbCand t = a[i];
  a[i] = a[j];
  a[j] = t;
}

VGB_HD void ab_median_to_front(AbCand *a, int front, int x, int y, int z) {
  if (ab_key_less(a[x], a[y])) {
    if (ab_key_less(a[y], a[z]))
      ab_swap(a, front, y);
    else if (ab_key_less(a[x], a[z]))
      ab_swap(a, front, z);
    else
      ab_swap(a, front, x);
  } else if (ab_key_less(a[x], a[z])) {
    ab_swap(a, front, x);
  } else if (ab_key_less(a[y], a[z])) {
    ab_swap(a, front, z);
  } else {
    ab_swap(a, front, y);
  }
}

// partitions [lo, hi) around a[pivot] (pivot < lo); returns the cut
VGB_HD int ab_partition(AbCand *a, int lo, int hi, int pivot) {
  for (;;) {
    while (ab_key_less(a[lo], a[pivot])) ++lo;
    --hi;
    while (ab_key_less(a[pivot], a[hi])) --hi;
    if (!(lo < hi)) return lo;
    ab_swap(a, lo, hi);
    ++lo;
  }
}

// sift the hole at `hole` down a max-heap of len elements, then place v
VGB_HD void ab_adjust_heap(AbCand *a, int hole, int len, AbCand v) {
  const int top = hole;
  int child = hole;
  while (child < (len - 1) / 2) {
    child = 2 * (child + 1);
    if (ab_key_less(a[child], a[child - 1])) --child;
    a[hole] = a[child];
    hole = child;
  }
  if ((len & 1) == 0 && child == (len - 2) / 2) {
    child = 2 * (child + 1);
    a[hole] = a[child - 1];
    hole = child - 1;
  }
  int parent = (hole - 1) / 2;
  while (hole > top && ab_key_less(a[parent], v)) {
    a[hole] = a[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  a[hole] = v;
}

VGB_HD void ab_heap_sort(AbCand *a, int len) {
  if (len >= 2) {
    for (int parent = (len - 2) / 2;; --parent) {
      ab_adjust_heap(a, parent, len, a[parent]);
      if (parent == 0) break;
    }
  }
  for (int last = len - 1; last > 0; --last) {
    const AbCand v = a[last];
    a[last] = a[0];
    ab_adjust_heap(a, 0, last, v);
  }
}

// insertion of a[i] into the sorted a[lo..i), stopping at lo only when guarded
VGB_HD void ab_insert(AbCand *a, int lo, int i, bool guarded) {
  const AbCand v = a[i];
  if (guarded && ab_key_less(v, a[lo])) {
    for (int k = i; k > lo; --k) a[k] = a[k - 1];
    a[lo] = v;
    return;
  }
  int k = i;
  while (ab_key_less(v, a[k - 1])) {
    a[k] = a[k - 1];
    --k;
  }
  a[k] = v;
}

constexpr int kAbSortThreshold = 16;

VGB_HD_NOINLINE void ab_sort_like_libstdcxx(AbCand *a, int n) {
  if (n < 2 || n >= (1 << 16)) return;
  int lg = 0;
  while ((n >> (lg + 1)) != 0) ++lg;
  // ranges still to partition: (first, last, depth left); the right part of
  // every cut is finished before the left, which does not change the result.
  // The stack never holds more entries than the depth limit (n < 2^16 here).
  int stack_first[32], stack_last[32], stack_depth[32];
  int top = 0;
  stack_first[0] = 0;
  stack_last[0] = n;
  stack_depth[0] = 2 * lg;
  top = 1;
  while (top > 0) {
    --top;
    const int first = stack_first[top];
    int last = stack_last[top];
    int depth = stack_depth[top];
    while (last - first > kAbSortThreshold) {
      if (depth == 0) {
        ab_heap_sort(a + first, last - first);
        break;
      }
      --depth;
      ab_median_to_front(a, first, first + 1, first + (last - first) / 2, last - 1);
      const int cut = ab_partition(a, first + 1, last, first);
      stack_first[top] = cut;
      stack_last[top] = last;
      stack_depth[top] = depth;
      ++top;
      last = cut;
    }
  }
  const int head = n > kAbSortThreshold ? kAbSortThreshold : n;
  for (int i = 1; i < head; ++i) ab_insert(a, 0, i, true);
  for (int i = head; i < n; ++i) ab_insert(a, 0, i, false);
}

// the ray as GetHitCandidates_v sets it up (source/ABBoxManager.cpp:110-114)
struct AbRay {
  float p[3], inv[3];
  int sign[3];
};

VGB_HD AbRay ab_ray(const V3<double> &p, const V3<double> &d) {
  AbRay r;
  r.inv[0] = 1.f / (float)d.x;
  r.inv[1] = 1.f / (float)d.y;
  r.inv[2] = 1.f / (float)d.z;
  r.p[0] = (float)p.x;
  r.p[1] = (float)p.y;
  r.p[2] = (float)p.z;
  for (int k = 0; k < 3; ++k) r.sign[k] = r.inv[k] < 0.f;
  return r;
}

// BoxImplementation::IntersectCachedKernel2<kScalarFloat, float>
// (volumes/kernel/BoxImplementation.h:337-384) with t0 = 0 and t1 = +inf on a
// box stored as lower and upper corner (two float4): the entry distance, or
// +inf when the ray misses.
VGB_HD float ab_intersect(const float4 *box, const AbRay &r) {
  const float inf = Lim<float>::inf();
  const float4 lo = box[0], hi = box[1];
  // corners[sign] and corners[1 - sign] of the reference, per axis
  const float xn = r.sign[0] ? hi.x : lo.x, xf = r.sign[0] ? lo.x : hi.x;
  const float yn = r.sign[1] ? hi.y : lo.y, yf = r.sign[1] ? lo.y : hi.y;
  const float zn = r.sign[2] ? hi.z : lo.z, zf = r.sign[2] ? lo.z : hi.z;
  float tmin = (xn - r.p[0]) * r.inv[0];
  float tymax = (yf - r.p[1]) * r.inv[1];
  if (tmin > tymax) return inf;
  float tmax = (xf - r.p[0]) * r.inv[0];
  const float tymin = (yn - r.p[1]) * r.inv[1];
  if (tymin > tmax) return inf;
  tmin = vmax(tmin, tymin);
  tmax = vmin(tmax, tymax);
  const float tzmin = (zn - r.p[2]) * r.inv[2];
  const float tzmax = (zf - r.p[2]) * r.inv[2];
  if ((tmin > tzmax) || (tzmin > tmax)) return inf;
  tmin = vmax(tmin, tzmin);
  tmax = vmin(tmax, tzmax);
  if (!((tmin < inf) && (tmax > 0.f))) return inf;
  return tmin;
}

template <class L, uint32_t kMask> struct ABBoxNavigator {
  using R = double;
  using S = NavShapes<kMask>;
  using Base = Navigator<L, kMask, false>;

  // ABBoxNavigator::GetSafety (navigation/ABBoxNavigator.h:424-452) is the
  // brute-force loop of SimpleNavigator::GetSafety.
  static VGB_HD R safety(const NavGeom &G, const NavPath &s, const V3<R> &lp) {
    return Base::safety(G, s, lp);
  }

  // Steps 2 and 3 above: updates step (entering with the mother's) and hit
  // (the daughter position, -1 for the mother).  buf holds cap + 16 entries.
  static VGB_HD void walk(const NavGeom &G, const int32_t *dl, const float4 *boxes, int nd,
                          const V3<R> &lp, const V3<R> &ld, R &step, int &hit, AbCand *buf,
                          int cap) {
    const AbRay ray = ab_ray(lp, ld);
    const float finf = Lim<float>::inf();
    L::sync();
    int m = 0;
    for (int base = 0; base < nd; base += L::N) {
      const int d = base + L::lane();
      float b = finf;
      if (d < nd) b = ab_intersect(boxes + 2 * d, ray);
      const bool keep = b < finf;
      const uint32_t bal = L::ballot(keep);
      if (keep) {
        const int pos = m + nav_popc(bal & L::lanes_below());
        if (pos < cap) buf[pos] = AbCand{b, d};
      }
      m += nav_popc(bal);
    }
    if (m == 0) return;
    if (m > cap) {
      walk_one_by_one(G, dl, boxes, nd, lp, ld, ray, step, hit);
      return;
    }
    L::sync();
    AbCand *sorted = buf;
    if (m <= kAbSortThreshold) {
      sorted = buf + cap;
      for (int i = L::lane(); i < m; i += L::N) {
        const AbCand c = buf[i];
        int r = 0;
        for (int j = 0; j < m; ++j) r += ab_less(buf[j], c) ? 1 : 0;
        sorted[r] = c;
      }
    } else if (L::lane() == 0) {
      ab_sort_like_libstdcxx(buf, m);
    }
    L::sync();
    const R inf = Lim<R>::inf();
    R t = step;
    int h = hit;
    for (int c0 = 0; c0 < m; c0 += L::N) {
      const int j = c0 + L::lane();
      const bool valid = j < m;
      const AbCand c = valid ? sorted[j] : AbCand{finf, -1};
      const R b = (R)c.b;
      R v = inf;  // what the candidate offers; +inf and NaN never improve
      bool inside = false;
      if (valid && !(t < b)) {
        const int32_t pv = dl[c.d];
        if (b < 0.) {
          V3<R> loc;
          inside = S::contains(G, pv, lp, loc);
        }
        if (!inside) {
          const R dd = S::distance_to_in(G, pv, lp, ld, t);
          if (dd == dd) v = dd;
        }
      }
      // the reference's running step when it reaches this lane's candidate
      R incl = v;
      for (int o = 1; o < L::N; o <<= 1) {
        const R u = L::shfl_up(incl, o);
        if (L::lane() >= o) incl = vmin(incl, u);
      }
      R excl = L::shfl_up(incl, 1);
      if (L::lane() == 0) excl = inf;
      const R before = vmin(t, excl);
      const bool stop_b = valid && (before < b);
      const bool stop_in = valid && !stop_b && inside;
      const uint32_t stops = L::ballot(stop_b || stop_in || !valid);
      const uint32_t ins = L::ballot(stop_in);
      const int f = stops ? nav_lowbit(stops) : L::N;
      R mv = (L::lane() < f) ? v : inf;
      int mi = L::lane();
      nav_min_reduce<L>(mv, mi);
      if (mv < t) {
        t = mv;
        h = sorted[c0 + mi].d;
      }
      if (f < L::N) {
        if ((ins >> f) & 1u) {
          t = 0.;
          h = sorted[c0 + f].d;
        }
        break;
      }
    }
    step = t;
    hit = h;
  }

  // The same walk for lists longer than the buffer: the next candidate is the
  // smallest (b, index) above the last one among the hits the step can reach.
  static VGB_HD_NOINLINE void walk_one_by_one(const NavGeom &G, const int32_t *dl,
                                              const float4 *boxes, int nd, const V3<R> &lp,
                                              const V3<R> &ld, const AbRay &ray, R &step,
                                              int &hit) {
    const float finf = Lim<float>::inf();
    R t = step;
    int h = hit;
    AbCand last = {-finf, -1};
    for (;;) {
      AbCand best = {finf, 0x7fffffff};
      for (int d = L::lane(); d < nd; d += L::N) {
        const float b = ab_intersect(boxes + 2 * d, ray);
        if (!(b < finf) || t < (R)b) continue;
        const AbCand c = {b, d};
        if (ab_less(last, c) && ab_less(c, best)) best = c;
      }
      for (int o = L::N / 2; o > 0; o >>= 1) {
        const AbCand oc = {L::shfl_xor(best.b, o), L::shfl_xor(best.d, o)};
        if (ab_less(oc, best)) best = oc;
      }
      if (best.d == 0x7fffffff) break;
      const int32_t pv = dl[best.d];
      if (best.b < 0.f) {
        V3<R> loc;
        if (S::contains(G, pv, lp, loc)) {
          t = 0.;
          h = best.d;
          break;
        }
      }
      const R dd = S::distance_to_in(G, pv, lp, ld, t);
      if (dd < t) {
        t = dd;
        h = best.d;
      }
      last = best;
    }
    step = t;
    hit = h;
  }

  // ABBoxNavigator::FindNextBoundaryAndStep (navigation/ABBoxNavigator.h:200-420).
  // `next` is updated from `cur`; false if a path would exceed kNavMaxLevels.
  static VGB_HD bool step(const NavGeom &G, const NavPath &cur, NavPath &next, const V3<R> &lp,
                          const V3<R> &ld, R pstep, R &step_out, AbCand *buf, int cap) {
    const int32_t cv = cur.top();
    R step = S::distance_to_out(G, cv, lp, ld, pstep);
    if (step < 0.) step = Lim<R>::inf();
    const LogicalRec &lr = G.logicals[G.placed[cv].logical];
    const int32_t nd = lr.dcount;
    const int32_t *dl = G.daughters + lr.dfirst;
    int hit = -1;
    if (nd > 0) walk(G, dl, G.ab_slot + 2 * (int64_t)lr.dfirst, nd, lp, ld, step, hit, buf, cap);

    next = cur;
    if (step > pstep) {
      step_out = pstep;
      next.boundary = false;
      return true;
    }
    next.boundary = true;
    if (step > 1E30) {
      step_out = 0.;
      next.pop();
      return true;
    }
    if (step < 0.) step = 0.;
    step_out = step;
    const R s6 = step + (R)1e-6;
    V3<R> np = {ld.x * s6, ld.y * s6, ld.z * s6};
    np = {np.x + lp.x, np.y + lp.y, np.z + lp.z};
    if (hit != -1) {
      const int32_t nv = dl[hit];
      if (next.level >= kNavMaxLevels) return false;
      next.push(nv);
      return Base::template descend<true>(G, next, nv,
                                          nav_generic_point(G.raw[G.placed[nv].raw_xform], np), -1);
    }
    const bool ok = Base::relocate_from_path(G, next, np);
    // leaving: pop while the relocation ends in the volume being left (:390-410)
    while (next.top() == cv) next.pop();
    return ok;
  }
};

}  // namespace vgb
