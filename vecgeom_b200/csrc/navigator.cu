// navigator.cu -- navigation kernels and their C ABI (vgb_navpool_*, vgb_nav_*).
//
// One warp per track: the warp's lanes share the daughter loops of the track's
// current volume (navigation.cuh).  The kernels are instantiated for two shape
// sets, the box/tube/trd set of layered detectors and every shape, and the
// launch picks the smallest set that covers the geometry.
#include <cstring>

#include "abbox.cuh"

using namespace vgb;

struct vgb_navpool {
  int device = -1;
  unsigned char *dev = nullptr;
  int64_t stride = 0;
  int64_t n = 0;
  int32_t max_depth = 0;
};

namespace vgb {
namespace {

constexpr int kNavBlock = 128;  // 4 warps, one track each
constexpr int kNavWarps = kNavBlock / 32;

int nav_grid(int64_t n) {
  const int64_t want = (n + kNavWarps - 1) / kNavWarps;
  const int64_t cap = 148 * 16;
  return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

NavGeom nav_geom(const vgb_geometry *g) {
  NavGeom G;
  G.params = g->dev.params;
  G.unplaced = g->dev.unplaced;
  G.placed = g->dev.placed;
  G.xforms = g->dev.xforms;
  G.raw = g->dev.raw;
  G.logicals = g->dev.logicals;
  G.daughters = g->dev.daughters;
  G.pl_box = g->dev.pl_box;
  G.ab_box = g->dev.ab_box;
  G.ab_slot = g->dev.ab_slot;
  G.world = g->world;
  G.max_depth = g->max_depth;
  return G;
}

VGB_D void nav_raise(uint32_t *flags, uint32_t bits) { atomicOr(flags, bits); }

template <uint32_t kMask>
__global__ void __launch_bounds__(kNavBlock) k_nav_locate(const NavGeom G, int64_t n,
                                                          const double *x, const double *y,
                                                          const double *z, unsigned char *states,
                                                          int64_t stride, uint32_t *flags) {
  using Nav = Navigator<WarpLanes, kMask>;
  const int64_t warps = (int64_t)gridDim.x * kNavWarps;
  for (int64_t i = (int64_t)blockIdx.x * kNavWarps + threadIdx.x / 32; i < n; i += warps) {
    NavPath s;
    const V3<double> p = {x[i], y[i], z[i]};
    const bool ok = Nav::locate_from_world(G, s, p);
    if (WarpLanes::lane() == 0) {
      if (!ok) {
        nav_raise(flags, VGB_NAV_ERR_DEPTH);
        s.level = 0;
      }
      nav_store(s, NavStateRef{states + i * stride}, G.max_depth);
    }
  }
}

template <uint32_t kMask, bool kScreen>
__global__ void __launch_bounds__(kNavBlock)
    k_nav_step(const NavGeom G, int64_t n, const double *x, const double *y, const double *z,
               const double *dx, const double *dy, const double *dz, const unsigned char *cur,
               unsigned char *next, int64_t stride, const double *pstep, double *step_out,
               double *safety_out, uint32_t *flags) {
  using Nav = Navigator<WarpLanes, kMask, kScreen>;
  const int64_t warps = (int64_t)gridDim.x * kNavWarps;
  for (int64_t i = (int64_t)blockIdx.x * kNavWarps + threadIdx.x / 32; i < n; i += warps) {
    NavPath c, nx;
    nav_load(c, NavStateRef{const_cast<unsigned char *>(cur) + i * stride});
    const V3<double> p = {x[i], y[i], z[i]};
    const V3<double> d = {dx[i], dy[i], dz[i]};
    double st = 0., sf = 0.;
    bool ok = true;
    nx = c;
    if (c.level > 0) {
      const DXform m = nav_top_matrix(G, c);
      const V3<double> lp = xf_point(m, p);
      const V3<double> ld = xf_dir(m, d);
      if (safety_out) sf = Nav::safety(G, c, lp);
      ok = Nav::step(G, c, nx, lp, ld, pstep[i], st);
    }
    if (WarpLanes::lane() == 0) {
      if (!ok) nav_raise(flags, VGB_NAV_ERR_DEPTH);
      nav_store(nx, NavStateRef{next + i * stride}, G.max_depth);
      step_out[i] = st;
      if (safety_out) safety_out[i] = sf;
    }
  }
}

// basket form of the step (SimpleNavigator.h:637-743) with GetSafeties (:599-632)
template <uint32_t kMask, bool>
__global__ void __launch_bounds__(kNavBlock)
    k_nav_basket(const NavGeom G, int64_t n, const double *x, const double *y, const double *z,
                 const double *dx, const double *dy, const double *dz, const unsigned char *cur,
                 unsigned char *next, int64_t stride, const double *pstep, double *dist_out,
                 double *safety_out, int32_t *node_out, uint32_t *flags) {
  using Nav = Navigator<WarpLanes, kMask>;
  const int64_t warps = (int64_t)gridDim.x * kNavWarps;
  for (int64_t i = (int64_t)blockIdx.x * kNavWarps + threadIdx.x / 32; i < n; i += warps) {
    NavPath c, nx;
    nav_load(c, NavStateRef{const_cast<unsigned char *>(cur) + i * stride});
    const V3<double> p = {x[i], y[i], z[i]};
    const V3<double> d = {dx[i], dy[i], dz[i]};
    double st = 0., sf = 0.;
    int32_t node = -2;
    bool ok = true;
    nx = c;
    if (c.level > 0) {
      const DXform m = nav_top_matrix(G, c);
      const V3<double> lp = xf_point(m, p);
      const V3<double> ld = xf_dir(m, d);
      if (safety_out) sf = Nav::safety(G, c, lp);
      ok = Nav::step_basket(G, c, nx, lp, ld, pstep[i], st, node);
    }
    if (WarpLanes::lane() == 0) {
      if (!ok) nav_raise(flags, VGB_NAV_ERR_DEPTH);
      nav_store(nx, NavStateRef{next + i * stride}, G.max_depth);
      dist_out[i] = st;
      if (safety_out) safety_out[i] = sf;
      if (node_out) node_out[i] = node;
    }
  }
}

template <uint32_t kMask, bool kScreen>
__global__ void __launch_bounds__(kNavBlock)
    k_nav_trace(const NavGeom G, int64_t n, const double *x, const double *y, const double *z,
                const double *dx, const double *dy, const double *dz, double pstep,
                int32_t max_steps, int32_t *next_ids, double *steps, double *safeties,
                int32_t *nsteps, uint32_t *flags) {
  using Nav = Navigator<WarpLanes, kMask, kScreen>;
  const int64_t warps = (int64_t)gridDim.x * kNavWarps;
  const bool lane0 = WarpLanes::lane() == 0;
  for (int64_t i = (int64_t)blockIdx.x * kNavWarps + threadIdx.x / 32; i < n; i += warps) {
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
      if (lane0) {
        const int64_t r = i * (int64_t)max_steps + k;
        if (next_ids) next_ids[r] = nxt.top();
        if (steps) steps[r] = st;
        if (safeties) safeties[r] = sf;
      }
      // the client advances to the boundary: p + d * step
      p = {p.x + d.x * st, p.y + d.y * st, p.z + d.z * st};
      cur = nxt;
      ++k;
    }
    if (lane0) {
      if (!ok) nav_raise(flags, VGB_NAV_ERR_DEPTH);
      nsteps[i] = ok ? k : -1;
    }
  }
}

// ABBoxNavigator kernels: the same loops with the box-culled step; each warp
// keeps its hit list in dynamic shared memory (cap hits, and the rank-sorted
// copy of a list of up to 16 beside them).  Volumes with more than kAbMaxCap
// daughters fall back to the one-by-one walk when a ray hits more boxes.
constexpr int kAbMaxCap = 6144;
extern __shared__ AbCand vgb_ab_lists[];

template <uint32_t kMask>
__global__ void __launch_bounds__(kNavBlock)
    k_abbox_step(const NavGeom G, int32_t cap, int64_t n, const double *x, const double *y, const double *z,
                 const double *dx, const double *dy, const double *dz, const unsigned char *cur,
                 unsigned char *next, int64_t stride, const double *pstep, double *step_out,
                 double *safety_out, uint32_t *flags) {
  using Nav = ABBoxNavigator<WarpLanes, kMask>;
  AbCand *buf = vgb_ab_lists + (threadIdx.x / 32) * (cap + kAbSortThreshold);
  const int64_t warps = (int64_t)gridDim.x * kNavWarps;
  for (int64_t i = (int64_t)blockIdx.x * kNavWarps + threadIdx.x / 32; i < n; i += warps) {
    NavPath c, nx;
    nav_load(c, NavStateRef{const_cast<unsigned char *>(cur) + i * stride});
    const V3<double> p = {x[i], y[i], z[i]};
    const V3<double> d = {dx[i], dy[i], dz[i]};
    double st = 0., sf = 0.;
    bool ok = true;
    nx = c;
    if (c.level > 0) {
      const DXform m = nav_top_matrix(G, c);
      const V3<double> lp = xf_point(m, p);
      const V3<double> ld = xf_dir(m, d);
      if (safety_out) sf = Nav::safety(G, c, lp);
      ok = Nav::step(G, c, nx, lp, ld, pstep[i], st, buf, cap);
    }
    if (WarpLanes::lane() == 0) {
      if (!ok) nav_raise(flags, VGB_NAV_ERR_DEPTH);
      nav_store(nx, NavStateRef{next + i * stride}, G.max_depth);
      step_out[i] = st;
      if (safety_out) safety_out[i] = sf;
    }
  }
}

template <uint32_t kMask>
__global__ void __launch_bounds__(kNavBlock)
    k_abbox_trace(const NavGeom G, int32_t cap, int64_t n, const double *x, const double *y, const double *z,
                  const double *dx, const double *dy, const double *dz, double pstep,
                  int32_t max_steps, int32_t *next_ids, double *steps, double *safeties,
                  int32_t *nsteps, uint32_t *flags) {
  using Nav = ABBoxNavigator<WarpLanes, kMask>;
  AbCand *buf = vgb_ab_lists + (threadIdx.x / 32) * (cap + kAbSortThreshold);
  const int64_t warps = (int64_t)gridDim.x * kNavWarps;
  const bool lane0 = WarpLanes::lane() == 0;
  for (int64_t i = (int64_t)blockIdx.x * kNavWarps + threadIdx.x / 32; i < n; i += warps) {
    V3<double> p = {x[i], y[i], z[i]};
    const V3<double> d = {dx[i], dy[i], dz[i]};
    NavPath cur, nxt;
    bool ok = Navigator<WarpLanes, kMask>::locate_from_world(G, cur, p);
    int32_t k = 0;
    while (ok && cur.level > 0 && k < max_steps) {
      const DXform m = nav_top_matrix(G, cur);
      const V3<double> lp = xf_point(m, p);
      const V3<double> ld = xf_dir(m, d);
      const double sf = Nav::safety(G, cur, lp);
      double st = 0.;
      ok = Nav::step(G, cur, nxt, lp, ld, pstep, st, buf, cap);
      if (!ok) break;
      if (lane0) {
        const int64_t r = i * (int64_t)max_steps + k;
        if (next_ids) next_ids[r] = nxt.top();
        if (steps) steps[r] = st;
        if (safeties) safeties[r] = sf;
      }
      p = {p.x + d.x * st, p.y + d.y * st, p.z + d.z * st};
      cur = nxt;
      ++k;
    }
    if (lane0) {
      if (!ok) nav_raise(flags, VGB_NAV_ERR_DEPTH);
      nsteps[i] = ok ? k : -1;
    }
  }
}

// Launches K<kMask, kScreen> for the smallest shape set covering the geometry;
// kScreen (the float screen of the FP32+refine form) when precision asks for it.
template <template <uint32_t, bool> class K, class... A>
vgb_status nav_launch(const vgb_geometry *g, int64_t n, cudaStream_t s, int precision, size_t smem,
                      A... args) {
  const int grid = nav_grid(n);
  const bool small = (g->type_mask & ~kNavMaskBoxTubeTrd) == 0;
  const bool screen = precision == VGB_PREC_FP32_REFINE;
  if (small && screen)
    K<kNavMaskBoxTubeTrd, true>::launch(grid, smem, s, args...);
  else if (small)
    K<kNavMaskBoxTubeTrd, false>::launch(grid, smem, s, args...);
  else if (screen)
    K<kNavMaskAll, true>::launch(grid, smem, s, args...);
  else
    K<kNavMaskAll, false>::launch(grid, smem, s, args...);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "navigation kernel launch");
  return VGB_OK;
}

template <uint32_t M, bool> struct LocateK {
  template <class... A> static void launch(int grid, size_t, cudaStream_t s, A... a) {
    k_nav_locate<M><<<grid, kNavBlock, 0, s>>>(a...);
  }
};
template <uint32_t M, bool S> struct StepK {
  template <class... A> static void launch(int grid, size_t, cudaStream_t s, A... a) {
    k_nav_step<M, S><<<grid, kNavBlock, 0, s>>>(a...);
  }
};
template <uint32_t M, bool S> struct BasketK {
  template <class... A> static void launch(int grid, size_t, cudaStream_t s, A... a) {
    k_nav_basket<M, S><<<grid, kNavBlock, 0, s>>>(a...);
  }
};
template <uint32_t M, bool S> struct TraceK {
  template <class... A> static void launch(int grid, size_t, cudaStream_t s, A... a) {
    k_nav_trace<M, S><<<grid, kNavBlock, 0, s>>>(a...);
  }
};

template <uint32_t M, bool> struct AbStepK {
  template <class... A> static void launch(int grid, size_t smem, cudaStream_t s, A... a) {
    cudaFuncSetAttribute(k_abbox_step<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_abbox_step<M><<<grid, kNavBlock, smem, s>>>(a...);
  }
};
template <uint32_t M, bool> struct AbTraceK {
  template <class... A> static void launch(int grid, size_t smem, cudaStream_t s, A... a) {
    cudaFuncSetAttribute(k_abbox_trace<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_abbox_trace<M><<<grid, kNavBlock, smem, s>>>(a...);
  }
};

// Hit-list capacity per warp: the most daughters of any volume (so every list
// fits and is ordered as the reference orders it), rounded up to 32 and kept
// within kAbMaxCap; dynamic shared memory of a block for it.
int abbox_cap(const vgb_geometry *g) {
  int cap = (g->max_daughters + 31) / 32 * 32;
  if (cap < 32) cap = 32;
  return cap > kAbMaxCap ? kAbMaxCap : cap;
}
size_t abbox_smem(int cap) { return (size_t)kNavWarps * (cap + kAbSortThreshold) * sizeof(AbCand); }

vgb_status check_nav_geometry(const vgb_geometry *g, const char *fn) {
  if (!g) return set_error(VGB_EINVAL, "%s: geometry is NULL", fn);
  if (!g->closed) return set_error(VGB_EINVAL, "%s: geometry is not closed", fn);
  if (g->world < 0) return set_error(VGB_EINVAL, "%s: no world volume set", fn);
  if (g->max_depth > kNavMaxLevels)
    return set_error(VGB_ENOTSUP, "%s: geometry is %d levels deep; at most %d are supported", fn,
                     g->max_depth, kNavMaxLevels);
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, fn);
  if (dev != g->device)
    return set_error(VGB_EINVAL, "%s: geometry lives on device %d, current device is %d", fn,
                     g->device, dev);
  return VGB_OK;
}

bool is_device_ptr(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace vgb

extern "C" {

vgb_status vgb_navpool_create(const vgb_geometry *g, int64_t n, vgb_navpool **pool) {
  if (!pool) return set_error(VGB_EINVAL, "vgb_navpool_create: pool is NULL");
  *pool = nullptr;
  vgb_status s = check_nav_geometry(g, "vgb_navpool_create");
  if (s != VGB_OK) return s;
  if (n < 0) return set_error(VGB_EINVAL, "vgb_navpool_create: n < 0");
  vgb_navpool *p = new vgb_navpool;
  p->device = g->device;
  p->max_depth = g->max_depth;
  p->stride = nav_state_stride(g->max_depth);
  p->n = n;
  const size_t bytes = (size_t)(n > 0 ? n : 1) * (size_t)p->stride;
  cudaError_t e = cudaMalloc((void **)&p->dev, bytes);
  if (e != cudaSuccess) {
    delete p;
    return cuda_error(e, "vgb_navpool_create: cudaMalloc");
  }
  e = cudaMemset(p->dev, 0, bytes);
  if (e != cudaSuccess) {
    cudaFree(p->dev);
    delete p;
    return cuda_error(e, "vgb_navpool_create: cudaMemset");
  }
  *pool = p;
  return VGB_OK;
}

vgb_status vgb_navpool_destroy(vgb_navpool *pool) {
  if (!pool) return VGB_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(pool->device);
  cudaFree(pool->dev);
  cudaSetDevice(prev);
  delete pool;
  return VGB_OK;
}

vgb_status vgb_navpool_info(const vgb_navpool *pool, void **device, int64_t *stride, int64_t *n) {
  if (!pool) return set_error(VGB_EINVAL, "vgb_navpool_info: pool is NULL");
  if (device) *device = pool->dev;
  if (stride) *stride = pool->stride;
  if (n) *n = pool->n;
  return VGB_OK;
}

vgb_status vgb_navpool_upload(vgb_navpool *pool, const void *host, int64_t n, void *stream) {
  if (!pool || (!host && n > 0)) return set_error(VGB_EINVAL, "vgb_navpool_upload: NULL argument");
  if (n < 0 || n > pool->n) return set_error(VGB_EINVAL, "vgb_navpool_upload: n out of range");
  if (n == 0) return VGB_OK;
  cudaError_t e = cudaMemcpyAsync(pool->dev, host, (size_t)(n * pool->stride),
                                  cudaMemcpyHostToDevice, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "vgb_navpool_upload");
  e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "vgb_navpool_upload");
  return VGB_OK;
}

vgb_status vgb_navpool_download(const vgb_navpool *pool, void *host, int64_t n, void *stream) {
  if (!pool || (!host && n > 0))
    return set_error(VGB_EINVAL, "vgb_navpool_download: NULL argument");
  if (n < 0 || n > pool->n) return set_error(VGB_EINVAL, "vgb_navpool_download: n out of range");
  if (n == 0) return VGB_OK;
  cudaError_t e = cudaMemcpyAsync(host, pool->dev, (size_t)(n * pool->stride),
                                  cudaMemcpyDeviceToHost, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "vgb_navpool_download");
  e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "vgb_navpool_download");
  return VGB_OK;
}

vgb_status vgb_nav_locate(const vgb_geometry *g, int64_t n, const double *x, const double *y,
                          const double *z, vgb_navpool *states, void *stream) {
  vgb_status s = check_nav_geometry(g, "vgb_nav_locate");
  if (s != VGB_OK) return s;
  if (!states || n < 0 || n > states->n || states->max_depth != g->max_depth)
    return set_error(VGB_EINVAL, "vgb_nav_locate: pool missing, too small or of another depth");
  if (n == 0) return VGB_OK;
  if (!is_device_ptr(x) || !is_device_ptr(y) || !is_device_ptr(z))
    return set_error(VGB_EINVAL, "vgb_nav_locate: points must be device memory");
  return nav_launch<LocateK>(g, n, (cudaStream_t)stream, VGB_PREC_FP64, 0, nav_geom(g), n, x, y, z,
                             states->dev,
                             states->stride, g->dev.nav_flags);
}

vgb_status vgb_nav_find_next_boundary_and_step(const vgb_geometry *g, int64_t n, const double *x,
                                               const double *y, const double *z,
                                               const double *dx, const double *dy,
                                               const double *dz, const vgb_navpool *cur,
                                               vgb_navpool *next, const double *pstep,
                                               double *step, double *safety, int32_t precision,
                                               void *stream) {
  const char *fn = "vgb_nav_find_next_boundary_and_step";
  if (precision != VGB_PREC_FP64 && precision != VGB_PREC_FP32_REFINE)
    return set_error(VGB_EINVAL, "%s: unknown precision %d", fn, precision);
  vgb_status s = check_nav_geometry(g, fn);
  if (s != VGB_OK) return s;
  if (!cur || !next || cur == next || n < 0 || n > cur->n || n > next->n ||
      cur->max_depth != g->max_depth || next->max_depth != g->max_depth)
    return set_error(VGB_EINVAL, "%s: need two distinct pools of the geometry's depth", fn);
  if (n == 0) return VGB_OK;
  const void *ptrs[] = {x, y, z, dx, dy, dz, pstep, step};
  for (const void *p : ptrs)
    if (!is_device_ptr(p)) return set_error(VGB_EINVAL, "%s: arrays must be device memory", fn);
  if (safety && !is_device_ptr(safety))
    return set_error(VGB_EINVAL, "%s: safety must be device memory or NULL", fn);
  return nav_launch<StepK>(g, n, (cudaStream_t)stream, precision, 0, nav_geom(g), n, x, y, z, dx,
                           dy, dz,
                           (const unsigned char *)cur->dev, next->dev, cur->stride, pstep, step,
                           safety, g->dev.nav_flags);
}

vgb_status vgb_nav_find_next_boundary_and_step_basket(
    const vgb_geometry *g, int64_t n, const double *x, const double *y, const double *z,
    const double *dx, const double *dy, const double *dz, const vgb_navpool *cur,
    vgb_navpool *next, const double *pstep, double *distance, double *safety, int32_t *nextnode,
    void *stream) {
  const char *fn = "vgb_nav_find_next_boundary_and_step_basket";
  vgb_status s = check_nav_geometry(g, fn);
  if (s != VGB_OK) return s;
  if (!cur || !next || cur == next || n < 0 || n > cur->n || n > next->n ||
      cur->max_depth != g->max_depth || next->max_depth != g->max_depth)
    return set_error(VGB_EINVAL, "%s: need two distinct pools of the geometry's depth", fn);
  if (n == 0) return VGB_OK;
  const void *ptrs[] = {x, y, z, dx, dy, dz, pstep, distance};
  for (const void *p : ptrs)
    if (!is_device_ptr(p)) return set_error(VGB_EINVAL, "%s: arrays must be device memory", fn);
  if ((safety && !is_device_ptr(safety)) || (nextnode && !is_device_ptr(nextnode)))
    return set_error(VGB_EINVAL, "%s: safety / nextnode must be device memory or NULL", fn);
  return nav_launch<BasketK>(g, n, (cudaStream_t)stream, VGB_PREC_FP64, 0, nav_geom(g), n, x, y,
                             z, dx, dy, dz, (const unsigned char *)cur->dev, next->dev,
                             cur->stride, pstep, distance, safety, nextnode, g->dev.nav_flags);
}

vgb_status vgb_nav_trace(const vgb_geometry *g, int64_t n, const double *x, const double *y,
                         const double *z, const double *dx, const double *dy, const double *dz,
                         double pstep, int32_t max_steps, int32_t *next_ids, double *steps,
                         double *safeties, int32_t *nsteps, int32_t precision, void *stream) {
  const char *fn = "vgb_nav_trace";
  if (precision != VGB_PREC_FP64 && precision != VGB_PREC_FP32_REFINE)
    return set_error(VGB_EINVAL, "%s: unknown precision %d", fn, precision);
  vgb_status s = check_nav_geometry(g, fn);
  if (s != VGB_OK) return s;
  if (n < 0 || max_steps < 0) return set_error(VGB_EINVAL, "%s: n or max_steps < 0", fn);
  if (n == 0) return VGB_OK;
  const void *ptrs[] = {x, y, z, dx, dy, dz, nsteps};
  for (const void *p : ptrs)
    if (!is_device_ptr(p)) return set_error(VGB_EINVAL, "%s: arrays must be device memory", fn);
  const void *opt[] = {next_ids, steps, safeties};
  for (const void *p : opt)
    if (p && !is_device_ptr(p))
      return set_error(VGB_EINVAL, "%s: records must be device memory or NULL", fn);
  return nav_launch<TraceK>(g, n, (cudaStream_t)stream, precision, 0, nav_geom(g), n, x, y, z, dx,
                            dy, dz,
                            pstep, max_steps, next_ids, steps, safeties, nsteps,
                            g->dev.nav_flags);
}

vgb_status vgb_abbox_nav_find_next_boundary_and_step(const vgb_geometry *g, int64_t n,
                                                     const double *x, const double *y,
                                                     const double *z, const double *dx,
                                                     const double *dy, const double *dz,
                                                     const vgb_navpool *cur, vgb_navpool *next,
                                                     const double *pstep, double *step,
                                                     double *safety, void *stream) {
  const char *fn = "vgb_abbox_nav_find_next_boundary_and_step";
  vgb_status s = check_nav_geometry(g, fn);
  if (s != VGB_OK) return s;
  if (!g->abbox_ok)
    return set_error(VGB_ENOTSUP, "%s: a volume's shape has no Extent (parallelepiped), so no "
                     "aligned box", fn);
  if (!cur || !next || cur == next || n < 0 || n > cur->n || n > next->n ||
      cur->max_depth != g->max_depth || next->max_depth != g->max_depth)
    return set_error(VGB_EINVAL, "%s: need two distinct pools of the geometry's depth", fn);
  if (n == 0) return VGB_OK;
  const void *ptrs[] = {x, y, z, dx, dy, dz, pstep, step};
  for (const void *p : ptrs)
    if (!is_device_ptr(p)) return set_error(VGB_EINVAL, "%s: arrays must be device memory", fn);
  if (safety && !is_device_ptr(safety))
    return set_error(VGB_EINVAL, "%s: safety must be device memory or NULL", fn);
  const int cap = abbox_cap(g);
  return nav_launch<AbStepK>(g, n, (cudaStream_t)stream, VGB_PREC_FP64, abbox_smem(cap),
                             nav_geom(g), (int32_t)cap, n, x, y, z,
                             dx, dy, dz, (const unsigned char *)cur->dev, next->dev, cur->stride,
                             pstep, step, safety, g->dev.nav_flags);
}

vgb_status vgb_abbox_nav_trace(const vgb_geometry *g, int64_t n, const double *x, const double *y,
                               const double *z, const double *dx, const double *dy,
                               const double *dz, double pstep, int32_t max_steps,
                               int32_t *next_ids, double *steps, double *safeties,
                               int32_t *nsteps, void *stream) {
  const char *fn = "vgb_abbox_nav_trace";
  vgb_status s = check_nav_geometry(g, fn);
  if (s != VGB_OK) return s;
  if (!g->abbox_ok)
    return set_error(VGB_ENOTSUP, "%s: a volume's shape has no Extent (parallelepiped), so no "
                     "aligned box", fn);
  if (n < 0 || max_steps < 0) return set_error(VGB_EINVAL, "%s: n or max_steps < 0", fn);
  if (n == 0) return VGB_OK;
  const void *ptrs[] = {x, y, z, dx, dy, dz, nsteps};
  for (const void *p : ptrs)
    if (!is_device_ptr(p)) return set_error(VGB_EINVAL, "%s: arrays must be device memory", fn);
  const void *opt[] = {next_ids, steps, safeties};
  for (const void *p : opt)
    if (p && !is_device_ptr(p))
      return set_error(VGB_EINVAL, "%s: records must be device memory or NULL", fn);
  const int cap = abbox_cap(g);
  return nav_launch<AbTraceK>(g, n, (cudaStream_t)stream, VGB_PREC_FP64, abbox_smem(cap),
                              nav_geom(g), (int32_t)cap, n, x, y, z,
                              dx, dy, dz, pstep, max_steps, next_ids, steps, safeties, nsteps,
                              g->dev.nav_flags);
}

vgb_status vgb_nav_error_flags(const vgb_geometry *g, uint32_t *flags) {
  if (!g || !flags) return set_error(VGB_EINVAL, "vgb_nav_error_flags: NULL argument");
  if (!g->closed) return set_error(VGB_EINVAL, "vgb_nav_error_flags: geometry is not closed");
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_error(e, "vgb_nav_error_flags");
  e = cudaMemcpy(flags, g->dev.nav_flags, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_error(e, "vgb_nav_error_flags");
  e = cudaMemset(g->dev.nav_flags, 0, sizeof(uint32_t));
  if (e != cudaSuccess) return cuda_error(e, "vgb_nav_error_flags");
  return VGB_OK;
}

}  // extern "C"
