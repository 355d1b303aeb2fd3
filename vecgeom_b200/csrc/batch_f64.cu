// batch_f64.cu -- FP64 instantiations of the batch kernels.
//
// Compiled with -fmad=false (see the Makefile): no a*b+c is contracted into an
// FMA, so each result rounds exactly as the reference Scalar build compiled
// with -ffp-contract=off.
#include "batch.cuh"
#include "dispatch.h"
#include "geometry.h"
#include "refine.cuh"

namespace vgb {

static int grid_for(int64_t n) {
  // enough CTAs to fill 148 SMs x 8 resident 256-thread CTAs; grid-stride beyond
  const int64_t want = (n + kBatchBlock - 1) / kBatchBlock;
  const int64_t cap = 148 * 8 * 4;
  return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

// The regrouped walks (polycone and polyhedron distances) refill a warp's lanes
// from the warp's own stream of points, so they keep lanes busier when each warp
// owns more points: a quarter of the grid above (measured: polyhedron
// DistanceToIn/Out 7.0 k/5.7 k -> 7.9 k/7.4 k Mpoints/s, polycone DistanceToIn
// 5.8 k -> 6.2 k, and polycone DistanceToOut regrouped 7.6 k, against 6.8 k on
// one lane), while the other kernels run fastest with the full grid.
constexpr int kWalkGridCap = 148 * 8;

template <class Ops, class P>
static vgb_status launch_ops(const P &prm, const DXform &X, int op, BatchIO io, cudaStream_t s,
                             int32_t rec_len = 0, int precision = VGB_PREC_FP64) {
  // FP32+refine: DistanceToIn of the shapes with a float selector (refine.cuh);
  // every other (shape, op) computes in FP64 in both forms
  if constexpr (!std::is_void<typename RefineDti<Ops>::type>::value) {
    if (precision == VGB_PREC_FP32_REFINE && op == VGB_OP_DISTANCE_TO_IN) {
      const int64_t tiles = (io.n + kRefineTile - 1) / kRefineTile;
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, 148 * 8));
      k_refine_dti<typename RefineDti<Ops>::type, Ops, P><<<grid, kRefineBlock, 0, s>>>(prm, X, io);
      count_launch();
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_error(e, "vgb_batch: kernel launch");
      return VGB_OK;
    }
  }
  const int grid = grid_for(io.n);
  io.stage = (Stageable<P>::value && rec_len > 0 && rec_len <= kStageMaxDoubles) ? rec_len : 0;
  const size_t smem = (size_t)io.stage * sizeof(double);
  switch (op) {
#define VGB_OP_CASE(OPC)                                                      \
  case OPC:                                                                   \
    k_batch<Ops, P, OPC><<<RegroupedWalk<Ops, OPC>::value ? std::min(grid, kWalkGridCap) \
                                                          : grid,                    \
                           kBatchBlock, smem, s>>>(prm, X, io);                      \
    break;
    VGB_OP_CASE(VGB_OP_CONTAINS)
    VGB_OP_CASE(VGB_OP_INSIDE)
    VGB_OP_CASE(VGB_OP_DISTANCE_TO_IN)
    VGB_OP_CASE(VGB_OP_DISTANCE_TO_OUT)
    VGB_OP_CASE(VGB_OP_SAFETY_TO_IN)
    VGB_OP_CASE(VGB_OP_SAFETY_TO_OUT)
    VGB_OP_CASE(VGB_OP_DISTANCE_TO_IN_MINIMIZE)
    VGB_OP_CASE(VGB_OP_SAFETY_TO_IN_MINIMIZE)
    VGB_OP_CASE(VGB_OP_SAFETY_TO_OUT_MINIMIZE)
    VGB_OP_CASE(VGB_OP_DISTANCE_TO_OUT_NODE)
    VGB_OP_CASE(VGB_OP_PLACED_DISTANCE_TO_OUT)
#undef VGB_OP_CASE
  default:
    return set_error(VGB_EINVAL, "vgb_batch: unknown op %d", op);
  }
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "vgb_batch: kernel launch");
  return VGB_OK;
}

template <class Ops, class P>
static vgb_status launch_fused(const P &prm, const DXform &X, const FusedIO &io,
                               cudaStream_t s) {
  k_fused<Ops, P><<<grid_for(io.n), kBatchBlock, 0, s>>>(prm, X, io);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "vgb_batch_fused: kernel launch");
  return VGB_OK;
}

// Boolean subtraction: compile-time components for the common pairs, the
// switch over primitive shapes for every other pair.
template <class F> static vgb_status with_boolean_ops(const BooleanP &b, F &&f) {
  const int lt = b.left.type, rt = b.right.type;
  if (lt == VGB_SHAPE_BOX && rt == VGB_SHAPE_TUBE) return f(BoolBoxTube<double>{});
  if (lt == VGB_SHAPE_BOX && rt == VGB_SHAPE_BOX) return f(BoolBoxBox<double>{});
  return f(BoolOps<double>{});
}

static BooleanP boolean_params(const vgb_geometry *g, int32_t unplaced) {
  return bind_params(*static_cast<const BooleanP *>(shape_params(g, unplaced)),
                     shape_params_dev(g, unplaced));
}

vgb_status launch_batch_f64(const vgb_geometry *g, int32_t placed, int op, const BatchIO &io0,
                            cudaStream_t s, int precision) {
  const PlacedRec &pr = g->placed[placed];
  const DXform &X = g->xforms[pr.xform];
  const int type = g->unplaced[pr.unplaced].type;
  const void *prm = shape_params(g, pr.unplaced);
  const BatchIO &io = io0;
  if (type == VGB_SHAPE_BOOLEAN) {
    const BooleanP b = boolean_params(g, pr.unplaced);
    return with_boolean_ops(
        b, [&](auto o) { return launch_ops<decltype(o)>(b, X, op, io, s, 0, precision); });
  }
  switch (type) {
#define VGB_SHAPE_CASE(TYPE, OPS, P) \
  case TYPE:                         \
    return launch_ops<OPS<double>>(                                                     \
        bind_params(*static_cast<const P *>(prm), shape_params_dev(g, pr.unplaced)), X, op, io, s, \
        g->unplaced[pr.unplaced].param_len, precision);
    VGB_FOR_EACH_SHAPE(VGB_SHAPE_CASE)
#undef VGB_SHAPE_CASE
  default:
    return set_error(VGB_ENOTSUP, "vgb_batch: shape type %d not supported", type);
  }
}

vgb_status launch_fused_f64(const vgb_geometry *g, int32_t placed, const FusedIO &io,
                            cudaStream_t s) {
  const PlacedRec &pr = g->placed[placed];
  const DXform &X = g->xforms[pr.xform];
  const int type = g->unplaced[pr.unplaced].type;
  const void *prm = shape_params(g, pr.unplaced);
  if (type == VGB_SHAPE_BOOLEAN) {
    const BooleanP b = boolean_params(g, pr.unplaced);
    return with_boolean_ops(b, [&](auto o) { return launch_fused<decltype(o)>(b, X, io, s); });
  }
  switch (type) {
#define VGB_SHAPE_CASE(TYPE, OPS, P) \
  case TYPE:                         \
    return launch_fused<OPS<double>>(                                                   \
        bind_params(*static_cast<const P *>(prm), shape_params_dev(g, pr.unplaced)), X, io, s);
    VGB_FOR_EACH_SHAPE(VGB_SHAPE_CASE)
#undef VGB_SHAPE_CASE
  default:
    return set_error(VGB_ENOTSUP, "vgb_batch_fused: shape type %d not supported", type);
  }
}

}  // namespace vgb

extern "C" vgb_status vgb_refine_counts(int64_t *certified, int64_t *fallback, int32_t reset) {
  vgb::RefineCounts c = {0, 0};
  cudaError_t e = cudaMemcpyFromSymbol(&c, vgb::g_refine_counts, sizeof(c));
  if (e != cudaSuccess) return vgb::cuda_error(e, "vgb_refine_counts");
  if (certified) *certified = (int64_t)c.certified;
  if (fallback) *fallback = (int64_t)c.fallback;
  if (reset) {
    const vgb::RefineCounts z = {0, 0};
    e = cudaMemcpyToSymbol(vgb::g_refine_counts, &z, sizeof(z));
    if (e != cudaSuccess) return vgb::cuda_error(e, "vgb_refine_counts");
  }
  return VGB_OK;
}
