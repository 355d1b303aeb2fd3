// hostcheck.cu -- test infrastructure: the device shape arithmetic of libvgb
// (vecgeom_b200/csrc/*.cuh, all __host__ __device__) compiled for the host, so
// the parity tests can check every shape's math against the reference on a
// machine without a GPU.  The product never loads this library; on a GPU the
// tests check the real kernels through libvgb.so.
//
// Built with -ffp-contract=off, like the FP64 kernels (-fmad=false), so the
// host results round like the device results (transcendentals aside).
#include <algorithm>
#include <utility>
#include <vector>

#include "../../vecgeom_b200/csrc/batch.cuh"
#include "../../vecgeom_b200/csrc/geometry.h"
#include "../../vecgeom_b200/csrc/abbox.cuh"

using namespace vgb;

namespace {

template <class Ops, class P>
int run(const P &prm, const DXform &X, int op, int64_t n, const double *x, const double *y,
        const double *z, const double *dx, const double *dy, const double *dz, const double *st,
        void *out) {
  for (int64_t i = 0; i < n; ++i) {
    const V3<double> m = {x[i], y[i], z[i]};
    V3<double> d = {0, 0, 0};
    if (dx) d = {dx[i], dy[i], dz[i]};
    switch (op) {
    case VGB_OP_CONTAINS: static_cast<uint8_t *>(out)[i] = Ops::contains(prm, xf_point(X, m)); break;
    case VGB_OP_INSIDE: static_cast<int32_t *>(out)[i] = Ops::inside(prm, xf_point(X, m)); break;
    case VGB_OP_DISTANCE_TO_IN:
      static_cast<double *>(out)[i] = Ops::distance_to_in(prm, xf_point(X, m), dti_dir<Ops>(X, d), st[i]);
      break;
    case VGB_OP_DISTANCE_TO_OUT:
      static_cast<double *>(out)[i] = Ops::distance_to_out(prm, m, d, st[i]);
      break;
    case VGB_OP_SAFETY_TO_IN: static_cast<double *>(out)[i] = Ops::safety_to_in(prm, xf_point(X, m)); break;
    case VGB_OP_SAFETY_TO_OUT: static_cast<double *>(out)[i] = Ops::safety_to_out(prm, m); break;
    default: return -1;
    }
  }
  return 0;
}

}  // namespace

extern "C" int hc_batch(const vgb_geometry *g, int32_t placed, int32_t op, int64_t n,
                        const double *x, const double *y, const double *z, const double *dx,
                        const double *dy, const double *dz, const double *st, void *out) {
  const PlacedRec &pr = g->placed[placed];
  const DXform &X = g->xforms[pr.xform];
  const int type = g->unplaced[pr.unplaced].type;
  const void *prm = shape_params(g, pr.unplaced);
  switch (type) {
#define VGB_SHAPE_CASE(TYPE, OPS, P) \
  case TYPE:                         \
    return run<OPS<double>>(bind_params(*static_cast<const P *>(prm),                    \
                                        static_cast<const double *>(prm)),                \
                            X, op, n, x, y, z, dx, dy, dz, st, out);
    VGB_FOR_EACH_SHAPE(VGB_SHAPE_CASE)
#undef VGB_SHAPE_CASE
  default:
    return -2;
  }
}

// The navigator of navigation.cuh with a single lane, over the host tables of an
// (unclosed) geometry: the same loop as vgb_nav_trace's kernel.
template <class Nav>
int trace_host(const NavGeom &G, int64_t n, const double *x, const double *y, const double *z,
               const double *dx, const double *dy, const double *dz, double pstep,
               int32_t max_steps, int32_t *next_ids, double *steps, double *safeties,
               int32_t *nsteps);

extern "C" int hc_nav_trace(vgb_geometry *g, int64_t n, const double *x, const double *y,
                            const double *z, const double *dx, const double *dy,
                            const double *dz, double pstep, int32_t max_steps, int32_t *next_ids,
                            double *steps, double *safeties, int32_t *nsteps, int32_t screen) {
  if (prepare_tables(g) != VGB_OK) return -1;
  const NavGeom G = {g->params.data(),    g->unplaced.data(), g->placed.data(),
                     g->xforms.data(),    g->nav_raw.data(),  g->logicals.data(),
                     g->daughters.data(), g->pl_box.data(),   g->ab_box.data(), g->ab_slot.data(), g->world,
                     g->max_depth};
  if (screen) return trace_host<Navigator<OneLane, kNavMaskAll, true>>(G, n, x, y, z, dx, dy, dz, pstep,
                                                                       max_steps, next_ids, steps,
                                                                       safeties, nsteps);
  return trace_host<Navigator<OneLane, kNavMaskAll, false>>(G, n, x, y, z, dx, dy, dz, pstep,
                                                            max_steps, next_ids, steps, safeties,
                                                            nsteps);
}

template <class Nav>
int trace_host(const NavGeom &G, int64_t n, const double *x, const double *y, const double *z,
               const double *dx, const double *dy, const double *dz, double pstep,
               int32_t max_steps, int32_t *next_ids, double *steps, double *safeties,
               int32_t *nsteps) {
  for (int64_t i = 0; i < n; ++i) {
    V3<double> p = {x[i], y[i], z[i]};
    const V3<double> d = {dx[i], dy[i], dz[i]};
    NavPath cur, nxt;
    bool ok = Nav::locate_from_world(G, cur, p);
    int32_t k = 0;
    while (ok && cur.level > 0 && k < max_steps) {
      const DXform m = nav_top_matrix(G, cur);
      const V3<double> lp = xf_point(m, p);
      const V3<double> ld = xf_dir(m, d);
      const double sf = Nav::safety(G, cur, lp);
      double st = 0.;
      ok = Nav::step(G, cur, nxt, lp, ld, pstep, st);
      if (!ok) break;
      const int64_t r = i * (int64_t)max_steps + k;
      next_ids[r] = nxt.top();
      steps[r] = st;
      safeties[r] = sf;
      p = {p.x + d.x * st, p.y + d.y * st, p.z + d.z * st};
      cur = nxt;
      ++k;
    }
    nsteps[i] = ok ? k : -1;
  }
  return 0;
}

// ABBoxNavigator (abbox.cuh) with a single lane and a hit list of `cap`
// entries (a small cap exercises the one-by-one walk of long lists).
extern "C" int hc_abbox_trace(vgb_geometry *g, int64_t n, const double *x, const double *y,
                              const double *z, const double *dx, const double *dy,
                              const double *dz, double pstep, int32_t max_steps,
                              int32_t *next_ids, double *steps, double *safeties, int32_t *nsteps,
                              int32_t cap) {
  if (prepare_tables(g) != VGB_OK || cap < 1) return -1;
  const NavGeom G = {g->params.data(),    g->unplaced.data(), g->placed.data(),
                     g->xforms.data(),    g->nav_raw.data(),  g->logicals.data(),
                     g->daughters.data(), g->pl_box.data(),   g->ab_box.data(), g->ab_slot.data(), g->world,
                     g->max_depth};
  using Nav = ABBoxNavigator<OneLane, kNavMaskAll>;
  std::vector<AbCand> buf((size_t)cap + kAbSortThreshold);
  for (int64_t i = 0; i < n; ++i) {
    V3<double> p = {x[i], y[i], z[i]};
    const V3<double> d = {dx[i], dy[i], dz[i]};
    NavPath cur, nxt;
    bool ok = Navigator<OneLane, kNavMaskAll>::locate_from_world(G, cur, p);
    int32_t k = 0;
    while (ok && cur.level > 0 && k < max_steps) {
      const DXform m = nav_top_matrix(G, cur);
      const V3<double> lp = xf_point(m, p);
      const V3<double> ld = xf_dir(m, d);
      const double sf = Nav::safety(G, cur, lp);
      double st = 0.;
      ok = Nav::step(G, cur, nxt, lp, ld, pstep, st, buf.data(), cap);
      if (!ok) break;
      const int64_t r = i * (int64_t)max_steps + k;
      next_ids[r] = nxt.top();
      steps[r] = st;
      safeties[r] = sf;
      p = {p.x + d.x * st, p.y + d.y * st, p.z + d.z * st};
      cur = nxt;
      ++k;
    }
    nsteps[i] = ok ? k : -1;
  }
  return 0;
}

// The introsort restatement of abbox.cuh next to the standard library's
// std::sort (of this build, libstdc++) on the same (distance, index) pairs with
// HitBoxComparatorFunctor's comparison; writes both orders of indices.
extern "C" int hc_abbox_sort_check(const float *b, int32_t n, int32_t *ours, int32_t *std_order) {
  std::vector<AbCand> a((size_t)n);
  std::vector<std::pair<int, double>> h((size_t)n);
  for (int i = 0; i < n; ++i) {
    a[i] = AbCand{b[i], i};
    h[i] = std::pair<int, double>(i, (double)b[i]);
  }
  ab_sort_like_libstdcxx(a.data(), n);
  std::sort(h.begin(), h.end(), [](const std::pair<int, double> &l, const std::pair<int, double> &r) {
    return l.second < r.second;
  });
  for (int i = 0; i < n; ++i) {
    ours[i] = a[i].d;
    std_order[i] = h[i].first;
  }
  return 0;
}

// The basket step (Navigator::step_basket) with one lane, after `prior`
// single-track steps from the located start point (the same sequence as the
// reference driver's vgref_nav_basket_step); outputs per track as there.
extern "C" int hc_nav_basket(vgb_geometry *g, int64_t n, const double *x, const double *y,
                             const double *z, const double *dx, const double *dy,
                             const double *dz, const double *pstep, int32_t prior, double *px,
                             double *py, double *pz, double *dist, double *safety,
                             int32_t *nextnode, int32_t *newtop, int32_t *boundary) {
  if (prepare_tables(g) != VGB_OK) return -1;
  const NavGeom G = {g->params.data(),    g->unplaced.data(), g->placed.data(),
                     g->xforms.data(),    g->nav_raw.data(),  g->logicals.data(),
                     g->daughters.data(), g->pl_box.data(),   g->ab_box.data(), g->ab_slot.data(),
                     g->world,            g->max_depth};
  using Nav = Navigator<OneLane, kNavMaskAll>;
  for (int64_t i = 0; i < n; ++i) {
    V3<double> p = {x[i], y[i], z[i]};
    const V3<double> d = {dx[i], dy[i], dz[i]};
    NavPath cur, nxt;
    if (!Nav::locate_from_world(G, cur, p)) return -2;
    for (int k = 0; k < prior && cur.level > 0; ++k) {
      const DXform m = nav_top_matrix(G, cur);
      double st = 0.;
      if (!Nav::step(G, cur, nxt, xf_point(m, p), xf_dir(m, d), 1e30, st)) return -2;
      p = {p.x + d.x * st, p.y + d.y * st, p.z + d.z * st};
      cur = nxt;
    }
    px[i] = p.x;
    py[i] = p.y;
    pz[i] = p.z;
    dist[i] = safety[i] = Lim<double>::quiet_nan();
    nextnode[i] = newtop[i] = boundary[i] = -7;
    if (cur.level == 0) continue;
    const DXform m = nav_top_matrix(G, cur);
    const V3<double> lp = xf_point(m, p), ld = xf_dir(m, d);
    safety[i] = Nav::safety(G, cur, lp);
    double st = 0.;
    int32_t node = 0;
    if (!Nav::step_basket(G, cur, nxt, lp, ld, pstep[i], st, node)) return -2;
    dist[i] = st;
    nextnode[i] = node;
    newtop[i] = nxt.top();
    boundary[i] = nxt.boundary ? 1 : 0;
  }
  return 0;
}

// The correctly rounded functions of crmath.cuh, element-wise over arrays
// (fn: 0 atan2(a, b), 1 sin(a), 2 cos(a), 3 cbrt(a)).
#include "../../vecgeom_b200/csrc/crmath.cuh"
extern "C" int hc_crmath(int32_t fn, int64_t n, const double *a, const double *b, double *out) {
  for (int64_t i = 0; i < n; ++i) {
    switch (fn) {
    case 0: out[i] = cr_atan2(a[i], b[i]); break;
    case 1: out[i] = cr_sin(a[i]); break;
    case 2: out[i] = cr_cos(a[i]); break;
    case 3: out[i] = cr_cbrt(a[i]); break;
    default: return -1;
    }
  }
  return 0;
}

// The FP32+refine DistanceToIn of a sphere placed volume on the host: the float
// selection and the FP64 value of the winning root where it certifies, the FP64
// DistanceToIn elsewhere (the GPU kernel runs the same functions).  winners[i]
// is the selection's result (0: uncertain).
#include "../../vecgeom_b200/csrc/refine.cuh"
extern "C" int hc_refine_dti(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                             const double *y, const double *z, const double *dx,
                             const double *dy, const double *dz, const double *st, double *out,
                             int32_t *winners) {
  const PlacedRec &pr = g->placed[placed];
  const DXform &X = g->xforms[pr.xform];
  if (g->unplaced[pr.unplaced].type != VGB_SHAPE_SPHERE) return -2;
  const SphereP &s = *static_cast<const SphereP *>(shape_params(g, pr.unplaced));
  for (int64_t i = 0; i < n; ++i) {
    const V3<double> p = xf_point(X, V3<double>{x[i], y[i], z[i]});
    const V3<double> v = dti_dir<SphereOps<double>>(X, V3<double>{dx[i], dy[i], dz[i]});
    const int w = SphereRefine::select(s, p, v);
    winners[i] = w;
    out[i] = w ? SphereRefine::eval(s, p, v, w) : SphereOps<double>::distance_to_in(s, p, v, st[i]);
  }
  return 0;
}
