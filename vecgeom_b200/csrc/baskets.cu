// baskets.cu -- many baskets (placed volume + its points) in one persistent launch,
// the autotuner that picks its launch shape, and its CUDA-graph replay.
//
// A plan keeps its baskets sorted by shape kind and splits every basket into
// tiles of `tile` points; tile t belongs to the basket found by a binary search
// over the per-basket tile prefix.  Each kind present has its own kernel
// (k_baskets_kind: that shape's per-point code only, registers sized for it),
// and the kinds' kernels run as concurrent branches forked from the caller's
// stream, so a captured graph holds them as parallel nodes of one launch.  A
// CTA takes its kind's tiles t0 + blockIdx.x, + gridDim.x, ... (the grid is
// sized to the kernel's resident CTAs on every SM), stages the tile's shape
// record and transform in shared memory (one broadcast read per tile instead of
// a parameter bank) and runs the fused per-point ops of batch.cuh over the
// tile's points.  The allocation-free entry point (below) runs all kinds in one
// kernel with a switch over the shapes (k_baskets).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "batch.cuh"
#include "geometry.h"

using namespace vgb;

namespace vgb {
namespace {

struct BasketRec {
  int32_t unplaced;
  int32_t xform;
  int64_t offset;
  int64_t count;
};

struct BasketGeom {
  const double *params;
  const UnplacedRec *unplaced;
  const DXform *xforms;
};

constexpr int kRecDoubles = 128;  // largest fixed shape record staged per tile (1 KB)

template <class P> struct HasBase : std::false_type {};
template <> struct HasBase<PolyconeP> : std::true_type {};
template <> struct HasBase<PolyhedronP> : std::true_type {};
template <> struct HasBase<BooleanP> : std::true_type {};

// kRegroup: the kind kernels run the section/segment walks regrouped; the
// all-shape kernel keeps one point per lane (the walk's state inside its
// switch over every shape would spill)
template <class Ops, class P, int kBlock, uint32_t kOps, bool kRegroup = false>
__device__ __forceinline__ void run_tile(const double *rec, const DXform *xg, int64_t first,
                                         int64_t end, const FusedIO &io, double *srec,
                                         DXform *sx) {
  static_assert(sizeof(P) <= kRecDoubles * sizeof(double), "shape record too large to stage");
  constexpr int nd = (int)((sizeof(P) + 7) / 8);
  for (int k = threadIdx.x; k < nd; k += kBlock) srec[k] = rec[k];
  if (threadIdx.x == 0) *sx = *xg;
  __syncthreads();
  P *sp = reinterpret_cast<P *>(srec);
  if constexpr (HasBase<P>::value) {
    if (threadIdx.x == 0) sp->base = rec;
    __syncthreads();
  }
  const P &prm = *sp;
  constexpr uint32_t kDtiSti = (1u << VGB_OP_DISTANCE_TO_IN) | (1u << VGB_OP_SAFETY_TO_IN);
  if constexpr (kRegroup && kOps == kDtiSti && RegroupedWalk<Ops, VGB_OP_DISTANCE_TO_IN>::value) {
    // section/segment walks: SafetyToIn one point per lane, then DistanceToIn as
    // the warp-regrouped walk over the tile (each warp's block-stride points)
    if ((io.ops & kDtiSti) == kDtiSti) {
      double *sti = static_cast<double *>(io.out[VGB_OP_SAFETY_TO_IN]);
      for (int64_t i = first + threadIdx.x; i < end; i += kBlock) {
        const V3<double> m = {ldg(io.x + i), ldg(io.y + i), ldg(io.z + i)};
        sti[i] = Ops::safety_to_in(prm, xf_point(*sx, m));
      }
      const int64_t base = first + 32 * (threadIdx.x >> 5);
      walk_regrouped<Ops, P, VGB_OP_DISTANCE_TO_IN>(
          prm, *sx, io, static_cast<double *>(io.out[VGB_OP_DISTANCE_TO_IN]),
          [=](int64_t s) { return base + (int64_t)kBlock * (s >> 5) + (s & 31); }, end);
      __syncthreads();  // the next tile overwrites the staged record
      return;
    }
  }
  for (int64_t i = first + threadIdx.x; i < end; i += kBlock)
    fused_point<Ops, P, kOps>(prm, *sx, io, i);
  __syncthreads();  // the next tile overwrites the staged record
}

// Op sets with their own instantiation: DistanceToIn + SafetyToIn (the mixed
// basket workload) and every fused op.
constexpr uint32_t kOpsDtiSti = (1u << VGB_OP_DISTANCE_TO_IN) | (1u << VGB_OP_SAFETY_TO_IN);
constexpr uint32_t kOpsAll = 0x3fu;

template <int kBlock, uint32_t kOps>
__global__ void __launch_bounds__(kBlock, 1)
    k_baskets(const BasketGeom G, const BasketRec *__restrict__ baskets,
              const int64_t *__restrict__ prefix, int32_t nb, int64_t ntiles, int32_t tile,
              const FusedIO io) {
  __shared__ __align__(16) double srec[kRecDoubles];
  __shared__ DXform sx;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int lo = 0, hi = nb;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (prefix[mid] <= t) lo = mid; else hi = mid;
    }
    const BasketRec b = baskets[lo];
    const int64_t first = b.offset + (t - prefix[lo]) * tile;
    const int64_t last = b.offset + b.count;
    const int64_t end = first + tile < last ? first + tile : last;
    const UnplacedRec u = G.unplaced[b.unplaced];
    const double *rec = G.params + u.param_off;
    const DXform *xg = G.xforms + b.xform;
    switch (u.type) {
#define VGB_BASKET_CASE(T, OPS, P)                                                 \
  case T:                                                                          \
    run_tile<OPS<double>, P, kBlock, kOps>(rec, xg, first, end, io, srec, &sx);    \
    break;
      VGB_FOR_EACH_SHAPE(VGB_BASKET_CASE)
#undef VGB_BASKET_CASE
      default:
        break;
    }
  }
}

// One shape kind: the tiles [t0, t1) of the baskets [b0, b1) (the plan keeps
// its baskets sorted by kind), with the kind's own per-point code, so the
// kernel carries no switch over every shape and its registers fit its shape.
template <class Ops, class P, int kBlock, uint32_t kOps>
__global__ void __launch_bounds__(kBlock)
    k_baskets_kind(const BasketGeom G, const BasketRec *__restrict__ baskets,
                   const int64_t *__restrict__ prefix, int32_t b0, int32_t b1, int64_t t0,
                   int64_t t1, int32_t tile, const FusedIO io) {
  __shared__ __align__(16) double srec[kRecDoubles];
  __shared__ DXform sx;
  for (int64_t t = t0 + blockIdx.x; t < t1; t += gridDim.x) {
    int lo = b0, hi = b1;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (prefix[mid] <= t) lo = mid; else hi = mid;
    }
    const BasketRec b = baskets[lo];
    const int64_t first = b.offset + (t - prefix[lo]) * tile;
    const int64_t last = b.offset + b.count;
    const int64_t end = first + tile < last ? first + tile : last;
    const UnplacedRec u = G.unplaced[b.unplaced];
    run_tile<Ops, P, kBlock, kOps, true>(G.params + u.param_off, G.xforms + b.xform, first,
                                         end, io, srec, &sx);
  }
}

// resident CTAs of the all-shape kernel on every SM (the allocation-free entry
// point launches it with 256-thread CTAs)
template <uint32_t kOps> int occupancy_grid() {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_baskets<256, kOps>, 256, 0);
  if (e != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return sms * per_sm;
}

bool valid_shape(int block, int tile) {
  return (block == 256 || block == 512) && tile >= block && tile % block == 0 &&
         tile <= (1 << 16);
}

}  // namespace
}  // namespace vgb

struct vgb_basket_plan {
  const vgb_geometry *g = nullptr;
  int device = -1;
  uint32_t ops = 0;
  int32_t nb = 0;
  int64_t points = 0;
  std::vector<vgb::BasketRec> host;
  vgb::BasketRec *d_baskets = nullptr;
  int64_t *d_prefix = nullptr;  // nb + 1 tile prefix for the current tile size
  int64_t ntiles = 0;
  int32_t block = 256;
  int32_t tile = 1024;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  // the shape kinds present: type, basket range [b0, b1) and tile range
  // [t0, t1) of the kind in the kind-sorted basket order
  struct Kind {
    int32_t type, sub, b0, b1;  // sub: the component pair of a boolean kind
    int64_t t0, t1;
  };
  std::vector<Kind> kinds;
  // one stream and join event per kind after the first, and the fork event:
  // the kinds' kernels run as concurrent branches (nodes of one captured graph)
  std::vector<cudaStream_t> kstreams;
  std::vector<cudaEvent_t> kjoin;
  cudaEvent_t kfork = nullptr;
};

namespace vgb {
namespace {

// Uploads the tile prefix for `tile` (stream-ordered; the host copy must live
// until the copy ran, so it is synchronous).
vgb_status set_tile(vgb_basket_plan *p, int32_t tile, cudaStream_t s) {
  std::vector<int64_t> prefix(p->nb + 1, 0);
  for (int b = 0; b < p->nb; ++b)
    prefix[b + 1] = prefix[b] + (p->host[b].count + tile - 1) / tile;
  cudaError_t e = cudaMemcpyAsync(p->d_prefix, prefix.data(), prefix.size() * sizeof(int64_t),
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_error(e, "basket plan: tile prefix upload");
  p->ntiles = prefix[p->nb];
  p->tile = tile;
  for (auto &k : p->kinds) {
    k.t0 = prefix[k.b0];
    k.t1 = prefix[k.b1];
  }
  return VGB_OK;
}

FusedIO make_io(const vgb_basket_plan *p, const double *x, const double *y, const double *z,
                const double *dx, const double *dy, const double *dz, const double *step,
                void *const *outs, uint32_t flags) {
  FusedIO io;
  std::memset(&io, 0, sizeof(io));
  io.x = x; io.y = y; io.z = z;
  io.dx = dx; io.dy = dy; io.dz = dz;
  io.step = step;
  for (int k = 0; k < 6; ++k) io.out[k] = (p->ops >> k) & 1u ? outs[k] : nullptr;
  io.n = p->points;
  io.ops = p->ops;
  io.flags = flags;
  return io;
}

template <uint32_t kOps, int kBlock, class Ops, class P>
void launch_kind_t(const vgb_basket_plan *p, const vgb_basket_plan::Kind &k, const FusedIO &io,
                   cudaStream_t s) {
  const BasketGeom G = {p->g->dev.params, p->g->dev.unplaced, p->g->dev.xforms};
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_baskets_kind<Ops, P, kBlock, kOps>,
                                                    kBlock, 0) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int grid = (int)std::min<int64_t>(k.t1 - k.t0, (int64_t)sms * per_sm);
  if (grid > 0)
    k_baskets_kind<Ops, P, kBlock, kOps><<<grid, kBlock, 0, s>>>(
        G, p->d_baskets, p->d_prefix, k.b0, k.b1, k.t0, k.t1, p->tile, io);
}

// A kind is a shape type; booleans are further told apart by their component
// types, so the common pairs run their compile-time specialisations.
constexpr int32_t kKindPairBox = 1, kKindPairBoxTube = 2;

template <uint32_t kOps, int kBlock>
void launch_kind(const vgb_basket_plan *p, const vgb_basket_plan::Kind &k, const FusedIO &io,
                 cudaStream_t s) {
  if (k.type == VGB_SHAPE_BOOLEAN) {
    if (k.sub == kKindPairBoxTube)
      launch_kind_t<kOps, kBlock, BoolBoxTube<double>, BooleanP>(p, k, io, s);
    else if (k.sub == kKindPairBox)
      launch_kind_t<kOps, kBlock, BoolBoxBox<double>, BooleanP>(p, k, io, s);
    else
      launch_kind_t<kOps, kBlock, BoolOps<double>, BooleanP>(p, k, io, s);
    return;
  }
  switch (k.type) {
#define VGB_KIND_CASE(T, OPS, P) \
  case T: launch_kind_t<kOps, kBlock, OPS<double>, P>(p, k, io, s); break;
    VGB_FOR_EACH_SHAPE(VGB_KIND_CASE)
#undef VGB_KIND_CASE
    default: break;
  }
}

template <uint32_t kOps>
void launch_kinds(const vgb_basket_plan *p, const FusedIO &io, cudaStream_t s) {
  const int nk = (int)p->kinds.size();
  if (nk > 1) cudaEventRecord(p->kfork, s);
  for (int i = 0; i < nk; ++i) {
    cudaStream_t ks = i == 0 ? s : p->kstreams[i - 1];
    if (i > 0) cudaStreamWaitEvent(ks, p->kfork, 0);
    if (p->block == 256)
      launch_kind<kOps, 256>(p, p->kinds[i], io, ks);
    else
      launch_kind<kOps, 512>(p, p->kinds[i], io, ks);
    if (i > 0) cudaEventRecord(p->kjoin[i - 1], ks);
  }
  for (int i = 1; i < nk; ++i) cudaStreamWaitEvent(s, p->kjoin[i - 1], 0);
}

vgb_status launch(const vgb_basket_plan *p, const FusedIO &io, cudaStream_t s) {
  if (p->ntiles == 0) return VGB_OK;
  if ((p->ops & ~kOpsDtiSti) == 0)
    launch_kinds<kOpsDtiSti>(p, io, s);
  else
    launch_kinds<kOpsAll>(p, io, s);
  count_launch((int)p->kinds.size());
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "vgb_basket_run: kernel launch");
  return VGB_OK;
}

vgb_status check_io(const vgb_basket_plan *p, const double *x, const double *y, const double *z,
                    const double *dx, const double *dy, const double *dz, const double *step,
                    void *const *outs, const char *fn) {
  if (!p) return set_error(VGB_EINVAL, "%s: plan is NULL", fn);
  if (!x || !y || !z) return set_error(VGB_EINVAL, "%s: points are NULL", fn);
  const uint32_t dist = (1u << VGB_OP_DISTANCE_TO_IN) | (1u << VGB_OP_DISTANCE_TO_OUT);
  if ((p->ops & dist) && (!dx || !dy || !dz || !step))
    return set_error(VGB_EINVAL, "%s: distances need directions and step_max", fn);
  if (!outs) return set_error(VGB_EINVAL, "%s: outs is NULL", fn);
  for (int k = 0; k < 6; ++k)
    if (((p->ops >> k) & 1u) && !outs[k])
      return set_error(VGB_EINVAL, "%s: output of op %d is NULL", fn, k);
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device)
    return set_error(VGB_EINVAL, "%s: current device %d is not the plan's device %d", fn, dev,
                     p->device);
  return VGB_OK;
}

}  // namespace
}  // namespace vgb

extern "C" {

vgb_status vgb_basket_plan_create(const vgb_geometry *g, const vgb_basket *baskets, int32_t nb,
                                  uint32_t ops, int32_t block, int32_t tile,
                                  vgb_basket_plan **plan) {
  if (!plan) return set_error(VGB_EINVAL, "vgb_basket_plan_create: plan is NULL");
  *plan = nullptr;
  if (!g || !g->closed) return set_error(VGB_EINVAL, "vgb_basket_plan_create: geometry not closed");
  if (nb < 0 || (nb > 0 && !baskets))
    return set_error(VGB_EINVAL, "vgb_basket_plan_create: bad basket array");
  if (ops == 0 || (ops & ~0x3fu))
    return set_error(VGB_EINVAL, "vgb_basket_plan_create: ops must be a mask over ops 0..5");
  if (block == 0) block = 256;
  if (tile == 0) tile = 1024;
  if (!valid_shape(block, tile))
    return set_error(VGB_EINVAL, "vgb_basket_plan_create: block %d / tile %d not supported", block,
                     tile);
  vgb_basket_plan *p = new vgb_basket_plan;
  p->g = g;
  p->device = g->device;
  p->ops = ops;
  p->nb = nb;
  p->block = block;
  p->host.resize(nb);
  for (int b = 0; b < nb; ++b) {
    const vgb_basket &k = baskets[b];
    if (k.placed < 0 || k.placed >= (int32_t)g->placed.size() || k.offset < 0 || k.count < 0) {
      delete p;
      return set_error(VGB_EINVAL, "vgb_basket_plan_create: basket %d is invalid", b);
    }
    const PlacedRec &pr = g->placed[k.placed];
    p->host[b] = BasketRec{pr.unplaced, pr.xform, k.offset, k.count};
    p->points = std::max<int64_t>(p->points, k.offset + k.count);
  }
  // baskets in shape-kind order (each writes only its own points, so the order
  // changes no result), one range per kind
  auto sub_of = [&](const BasketRec &r) {
    if (g->unplaced[r.unplaced].type != VGB_SHAPE_BOOLEAN) return 0;
    const BooleanP &bp = *static_cast<const BooleanP *>(shape_params(g, r.unplaced));
    if (bp.left.type == VGB_SHAPE_BOX && bp.right.type == VGB_SHAPE_TUBE) return kKindPairBoxTube;
    if (bp.left.type == VGB_SHAPE_BOX && bp.right.type == VGB_SHAPE_BOX) return kKindPairBox;
    return 0;
  };
  auto key_of = [&](const BasketRec &r) {
    return g->unplaced[r.unplaced].type * 16 + sub_of(r);
  };
  std::stable_sort(p->host.begin(), p->host.end(), [&](const BasketRec &a, const BasketRec &b) {
    return key_of(a) < key_of(b);
  });
  for (int b = 0; b < nb;) {
    const int key = key_of(p->host[b]);
    int e = b;
    while (e < nb && key_of(p->host[e]) == key) ++e;
    p->kinds.push_back({key / 16, key % 16, b, e, 0, 0});
    b = e;
  }
  for (size_t k = 1; k < p->kinds.size(); ++k) {
    cudaStream_t ks = nullptr;
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&ks, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (ks) p->kstreams.push_back(ks);
    if (ev) p->kjoin.push_back(ev);
    if (e != cudaSuccess) {
      vgb_basket_plan_destroy(p);
      return cuda_error(e, "vgb_basket_plan_create: kind streams");
    }
  }
  if (p->kinds.size() > 1) {
    cudaError_t e = cudaEventCreateWithFlags(&p->kfork, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      vgb_basket_plan_destroy(p);
      return cuda_error(e, "vgb_basket_plan_create: fork event");
    }
  }
  cudaError_t e = cudaMalloc((void **)&p->d_baskets, std::max(1, nb) * sizeof(BasketRec));
  if (e == cudaSuccess) e = cudaMalloc((void **)&p->d_prefix, (nb + 1) * sizeof(int64_t));
  if (e == cudaSuccess && nb > 0)
    e = cudaMemcpy(p->d_baskets, p->host.data(), nb * sizeof(BasketRec), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    vgb_basket_plan_destroy(p);
    return cuda_error(e, "vgb_basket_plan_create");
  }
  vgb_status s = set_tile(p, tile, nullptr);
  if (s != VGB_OK) {
    vgb_basket_plan_destroy(p);
    return s;
  }
  *plan = p;
  return VGB_OK;
}

vgb_status vgb_basket_plan_destroy(vgb_basket_plan *p) {
  if (!p) return VGB_OK;
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  cudaFree(p->d_baskets);
  cudaFree(p->d_prefix);
  for (cudaStream_t ks : p->kstreams) cudaStreamDestroy(ks);
  for (cudaEvent_t ev : p->kjoin) cudaEventDestroy(ev);
  if (p->kfork) cudaEventDestroy(p->kfork);
  delete p;
  return VGB_OK;
}

vgb_status vgb_basket_plan_info(const vgb_basket_plan *p, int64_t *points, int64_t *tiles,
                                int32_t *block, int32_t *tile) {
  if (!p) return set_error(VGB_EINVAL, "vgb_basket_plan_info: plan is NULL");
  if (points) *points = p->points;
  if (tiles) *tiles = p->ntiles;
  if (block) *block = p->block;
  if (tile) *tile = p->tile;
  return VGB_OK;
}

vgb_status vgb_basket_run(vgb_basket_plan *p, const double *x, const double *y, const double *z,
                          const double *dx, const double *dy, const double *dz,
                          const double *step_max, void *const *outs, uint32_t flags,
                          void *stream) {
  vgb_status s = check_io(p, x, y, z, dx, dy, dz, step_max, outs, "vgb_basket_run");
  if (s != VGB_OK) return s;
  return launch(p, make_io(p, x, y, z, dx, dy, dz, step_max, outs, flags), (cudaStream_t)stream);
}

vgb_status vgb_basket_tune(vgb_basket_plan *p, const double *x, const double *y, const double *z,
                           const double *dx, const double *dy, const double *dz,
                           const double *step_max, void *const *outs, uint32_t flags, int32_t reps,
                           void *stream, int32_t *best_block, int32_t *best_tile,
                           float *best_ms) {
  vgb_status s = check_io(p, x, y, z, dx, dy, dz, step_max, outs, "vgb_basket_tune");
  if (s != VGB_OK) return s;
  if (reps < 1) reps = 1;
  cudaStream_t st = (cudaStream_t)stream;
  const FusedIO io = make_io(p, x, y, z, dx, dy, dz, step_max, outs, flags);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = -1.f;
  int bb = p->block, bt = p->tile;
  const int blocks[] = {256, 512};
  const int mults[] = {1, 2, 4, 8, 16};
  for (int b : blocks) {
    for (int m : mults) {
      const int t = b * m;
      if (!valid_shape(b, t)) continue;
      p->block = b;
      if ((s = set_tile(p, t, st)) != VGB_OK) break;
      if ((s = launch(p, io, st)) != VGB_OK) break;  // warm-up
      cudaEventRecord(e0, st);
      for (int r = 0; r < reps && s == VGB_OK; ++r) s = launch(p, io, st);
      cudaEventRecord(e1, st);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        s = cuda_error(e, "vgb_basket_tune");
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)reps;
      if (best < 0.f || ms < best) {
        best = ms;
        bb = b;
        bt = t;
      }
    }
    if (s != VGB_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != VGB_OK) return s;
  p->block = bb;
  if ((s = set_tile(p, bt, st)) != VGB_OK) return s;
  if (best_block) *best_block = bb;
  if (best_tile) *best_tile = bt;
  if (best_ms) *best_ms = best;
  return VGB_OK;
}

vgb_status vgb_basket_graph_capture(vgb_basket_plan *p, const double *x, const double *y,
                                    const double *z, const double *dx, const double *dy,
                                    const double *dz, const double *step_max, void *const *outs,
                                    uint32_t flags) {
  vgb_status s = check_io(p, x, y, z, dx, dy, dz, step_max, outs, "vgb_basket_graph_capture");
  if (s != VGB_OK) return s;
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->graph_exec = nullptr;
  p->graph = nullptr;
  cudaStream_t cs;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_error(e, "vgb_basket_graph_capture: stream");
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    s = launch(p, make_io(p, x, y, z, dx, dy, dz, step_max, outs, flags), cs);
    cudaError_t e2 = cudaStreamEndCapture(cs, &p->graph);
    if (s == VGB_OK && e2 != cudaSuccess) s = cuda_error(e2, "vgb_basket_graph_capture: end");
  } else {
    s = cuda_error(e, "vgb_basket_graph_capture: begin");
  }
  if (s == VGB_OK) {
    e = cudaGraphInstantiate(&p->graph_exec, p->graph, 0);
    if (e != cudaSuccess) s = cuda_error(e, "vgb_basket_graph_capture: instantiate");
  }
  cudaStreamDestroy(cs);
  return s;
}

vgb_status vgb_basket_graph_launch(vgb_basket_plan *p, void *stream) {
  if (!p || !p->graph_exec)
    return set_error(VGB_EINVAL, "vgb_basket_graph_launch: no graph captured");
  cudaError_t e = cudaGraphLaunch(p->graph_exec, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "vgb_basket_graph_launch");
  count_launch();
  return VGB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// vgb_basket_run_noalloc: the basket launch with its tables in a fixed array
// compiled into the library, for callers that cannot allocate device memory.
// ---------------------------------------------------------------------------
namespace vgb {
namespace {

constexpr int32_t kNoallocMax = VGB_NOALLOC_MAX_BASKETS;
constexpr int32_t kNoallocBlock = 256;
constexpr int32_t kNoallocTile = 1024;
// layout: the caller's vgb_basket records as copied, the resolved BasketRec
// records, then the nb + 1 tile prefix
constexpr size_t kNoallocRawOff = 0;
constexpr size_t kNoallocRecOff = kNoallocRawOff + sizeof(vgb_basket) * kNoallocMax;
constexpr size_t kNoallocPrefixOff = kNoallocRecOff + sizeof(BasketRec) * kNoallocMax;
constexpr size_t kNoallocBytes = kNoallocPrefixOff + sizeof(int64_t) * (kNoallocMax + 1);
static_assert(kNoallocRecOff % 16 == 0 && kNoallocPrefixOff % 16 == 0, "table alignment");

// Every GPU that loads the library holds this array until the process exits.
// In host code the name is only a stand-in: its device address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_tables[kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kMaxDevices] = {};
// Host copy of the caller's basket records.  The library allocated it, so it is
// plain pageable memory: cudaMemcpyAsync from it returns only once the driver has
// staged the bytes, and the caller's own array (pinned or not) is never read after
// the call returns.  Filled and copied under g_noalloc_mu.
vgb_basket g_noalloc_host[kNoallocMax];

// Device address of the array on `dev` (the current device); looked up once.
vgb_status noalloc_tables(int dev, unsigned char **p) {
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(VGB_EINVAL, "vgb_basket_run_noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_tables);
    if (e != cudaSuccess) return cuda_error(e, "vgb_basket_run_noalloc: cudaGetSymbolAddress");
    g_noalloc_addr[dev] = ptr;
  }
  *p = static_cast<unsigned char *>(g_noalloc_addr[dev]);
  return VGB_OK;
}

// Resolves the copied records into BasketRec and writes the tile prefix
// (one CTA: every thread scans up to 8 consecutive baskets, then a block scan).
__global__ void __launch_bounds__(1024)
    k_noalloc_tables(const vgb_basket *raw, int32_t nb, const PlacedRec *placed, int32_t tile,
                     BasketRec *rec, int64_t *prefix) {
  __shared__ int64_t part[1024];
  const int per = (nb + 1023) / 1024;
  const int b0 = threadIdx.x * per;
  int64_t sum = 0;
  for (int k = 0; k < per; ++k) {
    const int b = b0 + k;
    if (b < nb) {
      const vgb_basket r = raw[b];
      const PlacedRec pr = placed[r.placed];
      rec[b] = BasketRec{pr.unplaced, pr.xform, r.offset, r.count};
      sum += (r.count + tile - 1) / tile;
    }
  }
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int64_t v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int64_t run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  if (threadIdx.x == 0) prefix[0] = 0;
  for (int k = 0; k < per; ++k) {
    const int b = b0 + k;
    if (b < nb) {
      run += (raw[b].count + tile - 1) / tile;
      prefix[b + 1] = run;
    }
  }
}

template <uint32_t kOps>
void noalloc_launch(const vgb_geometry *g, const BasketRec *rec, const int64_t *prefix,
                    int32_t nb, int64_t ntiles, const FusedIO &io, cudaStream_t s) {
  const BasketGeom G = {g->dev.params, g->dev.unplaced, g->dev.xforms};
  static_assert(kNoallocBlock == 256, "the all-shape kernel is built for 256-thread CTAs");
  const int grid = (int)std::min<int64_t>(ntiles, occupancy_grid<kOps>());
  k_baskets<kNoallocBlock, kOps><<<grid, kNoallocBlock, 0, s>>>(G, rec, prefix, nb, ntiles,
                                                                 kNoallocTile, io);
}

}  // namespace
}  // namespace vgb

extern "C" vgb_status vgb_basket_run_noalloc(const vgb_geometry *g, const vgb_basket *baskets,
                                             int32_t nb, uint32_t ops, const double *x,
                                             const double *y, const double *z, const double *dx,
                                             const double *dy, const double *dz,
                                             const double *step_max, void *const *outs,
                                             uint32_t flags, void *stream) {
  const char *fn = "vgb_basket_run_noalloc";
  if (!g || !g->closed) return set_error(VGB_EINVAL, "%s: geometry not closed", fn);
  if (nb < 0 || (nb > 0 && !baskets)) return set_error(VGB_EINVAL, "%s: bad basket array", fn);
  if (nb > kNoallocMax)
    return set_error(VGB_ENOSPC, "%s: %d baskets exceed the fixed table of %d", fn, nb,
                     kNoallocMax);
  if (ops == 0 || (ops & ~0x3fu))
    return set_error(VGB_EINVAL, "%s: ops must be a mask over ops 0..5", fn);
  if (!x || !y || !z || !outs) return set_error(VGB_EINVAL, "%s: points or outs are NULL", fn);
  const uint32_t dist = (1u << VGB_OP_DISTANCE_TO_IN) | (1u << VGB_OP_DISTANCE_TO_OUT);
  if ((ops & dist) && (!dx || !dy || !dz || !step_max))
    return set_error(VGB_EINVAL, "%s: distances need directions and step_max", fn);
  for (int k = 0; k < 6; ++k)
    if (((ops >> k) & 1u) && !outs[k])
      return set_error(VGB_EINVAL, "%s: output of op %d is NULL", fn, k);
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, fn);
  if (dev != g->device)
    return set_error(VGB_EINVAL, "%s: current device %d is not the geometry's device %d", fn,
                     dev, g->device);
  int64_t ntiles = 0, npoints = 0;
  for (int32_t b = 0; b < nb; ++b) {
    const vgb_basket &k = baskets[b];
    if (k.placed < 0 || k.placed >= (int32_t)g->placed.size() || k.offset < 0 || k.count < 0)
      return set_error(VGB_EINVAL, "%s: basket %d is invalid", fn, b);
    ntiles += (k.count + kNoallocTile - 1) / kNoallocTile;
    npoints = std::max<int64_t>(npoints, k.offset + k.count);
  }
  if (ntiles == 0) return VGB_OK;
  unsigned char *tables = nullptr;
  vgb_status st = noalloc_tables(dev, &tables);
  if (st != VGB_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  vgb_basket *raw = reinterpret_cast<vgb_basket *>(tables + kNoallocRawOff);
  BasketRec *rec = reinterpret_cast<BasketRec *>(tables + kNoallocRecOff);
  int64_t *prefix = reinterpret_cast<int64_t *>(tables + kNoallocPrefixOff);
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    std::memcpy(g_noalloc_host, baskets, sizeof(vgb_basket) * nb);
    e = cudaMemcpyAsync(raw, g_noalloc_host, sizeof(vgb_basket) * nb, cudaMemcpyHostToDevice, s);
  }
  if (e != cudaSuccess) return cuda_error(e, "vgb_basket_run_noalloc: basket copy");
  k_noalloc_tables<<<1, 1024, 0, s>>>(raw, nb, g->dev.placed, kNoallocTile, rec, prefix);
  FusedIO io;
  std::memset(&io, 0, sizeof(io));
  io.x = x; io.y = y; io.z = z;
  io.dx = dx; io.dy = dy; io.dz = dz;
  io.step = step_max;
  for (int k = 0; k < 6; ++k) io.out[k] = ((ops >> k) & 1u) ? outs[k] : nullptr;
  io.n = npoints;
  io.ops = ops;
  io.flags = flags;
  if ((ops & ~kOpsDtiSti) == 0)
    noalloc_launch<kOpsDtiSti>(g, rec, prefix, nb, ntiles, io, s);
  else
    noalloc_launch<kOpsAll>(g, rec, prefix, nb, ntiles, io, s);
  count_launch(2);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "vgb_basket_run_noalloc: kernel launch");
  return VGB_OK;
}
