// batch.cuh -- the SOA batch kernels behind vgb_batch / vgb_batch_fused.
//
// One thread per point, grid-stride over the batch.  The shape's parameter
// record and the placement transform are kernel arguments, so every thread
// reads them from the constant bank (a broadcast) and the only global traffic
// is the coalesced SOA stream: x,y,z (+ dx,dy,dz, step_max) in, one result out.
// Replaces the reference's per-op CUDA kernels (source/benchmarking/Benchmarker.cu:13-79),
// which make a device virtual call per point, with shape and op resolved at
// compile time.
#pragma once
#include <type_traits>

#include "shapes.cuh"

namespace vgb {

constexpr int kBatchBlock = 256;

struct BatchIO {
  const double *x, *y, *z;
  const double *dx, *dy, *dz;
  const double *step;
  void *out;
  int32_t *aux;
  int64_t n;
  int32_t daughter;
  int32_t stage;  // doubles of the shape record staged in shared memory (0: none)
};

// Fused: the outputs of every op of the mask, one read of the inputs.
struct FusedIO {
  const double *x, *y, *z;
  const double *dx, *dy, *dz;
  const double *step;
  void *out[6];
  int64_t n;
  uint32_t ops;
  uint32_t flags;
};

template <class T> VGB_D T ldg(const T *p) { return __ldg(p); }

// Shapes whose tables hang off the record (polycone sections, polyhedron
// segments and quadrilaterals) can run with the record and its tables staged in
// shared memory: every thread of a block reads the same table entries, which a
// shared-memory copy serves without the global-load latency.
template <class P> struct Stageable : std::false_type {};
template <> struct Stageable<PolyconeP> : std::true_type {};
template <> struct Stageable<PolyhedronP> : std::true_type {};
constexpr int kStageMaxDoubles = 6144;  // 48 KB of dynamic shared memory
extern __shared__ double vgb_stage[];

// Distance kernels carry the most live state; they are compiled for four
// resident 256-thread blocks per SM (64 registers), or the shape's own
// `kDistanceBlocks` (five for tube and cone: 51 registers, more warps to hide
// the FP64 latency; measured 5 % faster DistanceToIn, while the sphere and the
// composite shapes spill at five); the others keep the compiler's own choice
// (0: no minimum).
template <class Ops, class = void> struct DistanceBlocks {
  static constexpr int value = 4;
};
template <class Ops>
struct DistanceBlocks<Ops, std::void_t<decltype(Ops::kDistanceBlocks)>> {
  static constexpr int value = Ops::kDistanceBlocks;
};
template <class Ops, int OP> struct MinBlocks {
  static constexpr int value =
      (OP == VGB_OP_DISTANCE_TO_IN || OP == VGB_OP_DISTANCE_TO_OUT ||
       OP == VGB_OP_DISTANCE_TO_IN_MINIMIZE || OP == VGB_OP_DISTANCE_TO_OUT_NODE ||
       OP == VGB_OP_PLACED_DISTANCE_TO_OUT) ? DistanceBlocks<Ops>::value : 0;
};

template <class Ops, class P, int OP>
__device__ __forceinline__ void batch_point(const P &prm, const DXform &X, const BatchIO &io,
                                            int64_t i) {
  using R = double;
  const V3<R> m = {ldg(io.x + i), ldg(io.y + i), ldg(io.z + i)};
  if constexpr (OP == VGB_OP_CONTAINS) {
    static_cast<uint8_t *>(io.out)[i] = (uint8_t)Ops::contains(prm, xf_point(X, m));
  } else if constexpr (OP == VGB_OP_INSIDE) {
    static_cast<int32_t *>(io.out)[i] = Ops::inside(prm, xf_point(X, m));
  } else if constexpr (OP == VGB_OP_SAFETY_TO_IN) {
    static_cast<double *>(io.out)[i] = Ops::safety_to_in(prm, xf_point(X, m));
  } else if constexpr (OP == VGB_OP_SAFETY_TO_OUT) {
    static_cast<double *>(io.out)[i] = Ops::safety_to_out(prm, m);
  } else if constexpr (OP == VGB_OP_SAFETY_TO_IN_MINIMIZE) {
    // volumes/ShapeImplementationHelper.h:708-720
    double *o = static_cast<double *>(io.out);
    const R r = Ops::safety_to_in(prm, xf_point(X, m));
    const R cur = o[i];
    o[i] = (r < cur) ? r : cur;
  } else if constexpr (OP == VGB_OP_SAFETY_TO_OUT_MINIMIZE) {
    // volumes/ShapeImplementationHelper.h:734-746
    double *o = static_cast<double *>(io.out);
    const R r = Ops::safety_to_out(prm, m);
    const R cur = o[i];
    o[i] = (r < cur) ? r : cur;
  } else {
    const V3<R> d = {ldg(io.dx + i), ldg(io.dy + i), ldg(io.dz + i)};
    if constexpr (OP == VGB_OP_DISTANCE_TO_IN) {
      static_cast<double *>(io.out)[i] =
          Ops::distance_to_in(prm, xf_point(X, m), dti_dir<Ops>(X, d), ldg(io.step + i));
    } else if constexpr (OP == VGB_OP_DISTANCE_TO_OUT) {
      static_cast<double *>(io.out)[i] = Ops::distance_to_out(prm, m, d, ldg(io.step + i));
    } else if constexpr (OP == VGB_OP_DISTANCE_TO_OUT_NODE) {
      // volumes/ShapeImplementationHelper.h:676-692: -1 leaves, -2 stays
      const R s = ldg(io.step + i);
      const R r = Ops::distance_to_out(prm, m, d, s);
      static_cast<double *>(io.out)[i] = r;
      io.aux[i] = (r < s) ? -1 : -2;
    } else if constexpr (OP == VGB_OP_PLACED_DISTANCE_TO_OUT) {
      // volumes/ShapeImplementationHelper.h:243-270
      static_cast<double *>(io.out)[i] =
          Ops::distance_to_out(prm, xf_point(X, m), xf_dir(X, d), ldg(io.step + i));
    } else if constexpr (OP == VGB_OP_DISTANCE_TO_IN_MINIMIZE) {
      // volumes/ShapeImplementationHelper.h:637-658 (Scalar form): the current
      // distance is the step limit; update only on a strictly smaller result.
      double *o = static_cast<double *>(io.out);
      const R cur = o[i];
      const R r = Ops::distance_to_in(prm, xf_point(X, m), dti_dir<Ops>(X, d), cur);
      if (r < cur) {
        o[i] = r;
        io.aux[i] = io.daughter;
      }
    }
  }
}

// Distance walks with warp-regrouped steps: polycone DistanceToIn/DistanceToOut
// (walks over cone sections) and polyhedron DistanceToIn/DistanceToOut (walks
// over z-segments).  A point's walk takes from one to all of its sections; run
// one point per lane to the end and a warp waits for its longest walk with its
// other lanes idle.  Here each iteration evaluates one step for the point each
// lane holds, and the lanes whose walk ended (a __ballot_sync over the warp)
// take the warp's next points at once (ranked by __popc), so the warp stays
// full until its points run out; the steps of each point are the ones the
// scalar function takes, so every result is the same.  A warp owns the points
// point_of(0), point_of(1), ... below `end` (point_of increasing, the same for
// the whole warp); the batch kernels give it the grid-stride order (slot s of
// global warp gw is point 32 gw + 32 W (s / 32) + s % 32, W warps in the grid),
// the basket kernels the block-stride order of one tile.  IO holds the input
// arrays (x, y, z, dx, dy, dz, step); out receives the distances.
template <class Ops, int OP> struct RegroupedWalk : std::false_type {};
template <> struct RegroupedWalk<PolyconeOps<double>, VGB_OP_DISTANCE_TO_IN> : std::true_type {};
template <> struct RegroupedWalk<PolyconeOps<double>, VGB_OP_DISTANCE_TO_OUT> : std::true_type {};
template <> struct RegroupedWalk<PolyhedronOps<double>, VGB_OP_DISTANCE_TO_IN> : std::true_type {};
template <> struct RegroupedWalk<PolyhedronOps<double>, VGB_OP_DISTANCE_TO_OUT> : std::true_type {};

template <class Ops, class P, int OP, class IO, class PointOf>
__device__ __forceinline__ void walk_regrouped(const P &prm, const DXform &X, const IO &io,
                                               double *out, PointOf point_of, int64_t end) {
  using R = double;
  constexpr bool kIn = OP == VGB_OP_DISTANCE_TO_IN;
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int64_t next = 0;  // the warp's next slot (warp-uniform)
  int64_t i = -1;    // the lane's point, -1: none
  V3<R> q = {0, 0, 0}, v = {0, 0, 0};
  R smax = 0;
  typename Ops::Walk w;
  while (true) {
    const bool free_lane = i < 0;
    const unsigned m = __ballot_sync(kFull, free_lane);
    if (free_lane) {
      const int64_t pi = point_of(next + __popc(m & ((1u << lane) - 1u)));
      if (pi < end) {
        const V3<R> mq = {ldg(io.x + pi), ldg(io.y + pi), ldg(io.z + pi)};
        const V3<R> md = {ldg(io.dx + pi), ldg(io.dy + pi), ldg(io.dz + pi)};
        smax = ldg(io.step + pi);
        R res;
        bool done;
        if constexpr (kIn) {
          q = xf_point(X, mq);
          v = dti_dir<Ops>(X, md);
          done = Ops::dti_begin(prm, q, v, smax, w, res);
        } else {
          q = mq;
          v = md;
          done = Ops::dto_begin(prm, q, v, smax, w, res);
        }
        if (done)
          out[pi] = res;  // settled in the set-up; the lane stays free
        else
          i = pi;
      }
    }
    next += __popc(m);
    const bool more = point_of(next) < end;  // warp-uniform
    if (!__any_sync(kFull, i >= 0) && !more) break;
    if (i >= 0) {
      bool ended;
      if constexpr (kIn)
        ended = Ops::dti_step(prm, q, v, smax, w);
      else
        ended = Ops::dto_step(prm, q, v, smax, w);
      if (ended) {
        if constexpr (kIn)
          out[i] = Ops::dti_end(prm, q, v, smax, w);
        else
          out[i] = Ops::dto_end(prm, q, v, smax, w);
        i = -1;
      }
    }
  }
}

template <class Ops, class P, int OP>
__device__ __forceinline__ void batch_loop(const P &prm, const DXform &X, const BatchIO &io) {
  if constexpr (RegroupedWalk<Ops, OP>::value) {
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    walk_regrouped<Ops, P, OP>(
        prm, X, io, static_cast<double *>(io.out),
        [=](int64_t s) { return 32 * gw + 32 * nw * (s >> 5) + (s & 31); }, io.n);
    return;
  }
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < io.n; i += stride)
    batch_point<Ops, P, OP>(prm, X, io, i);
}

template <class Ops, class P, int OP>
__global__ void __launch_bounds__(kBatchBlock, MinBlocks<Ops, OP>::value)
    k_batch(const P prm, const DXform X, const BatchIO io) {
  if constexpr (Stageable<P>::value) {
    if (io.stage > 0) {
      for (int k = threadIdx.x; k < io.stage; k += blockDim.x) vgb_stage[k] = prm.base[k];
      __syncthreads();
      P sp = prm;
      sp.base = vgb_stage;
      batch_loop<Ops, P, OP>(sp, X, io);
      return;
    }
  }
  batch_loop<Ops, P, OP>(prm, X, io);
}

// All requested ops for one point.  With VGB_FUSED_DTO_INSIDE_ONLY the
// DistanceToOut result is computed only where Contains() holds.  kOps bounds the
// ops at compile time (callers that know their op set drop the other paths).
template <class Ops, class P, uint32_t kOps = 0x3fu>
__device__ __forceinline__ void fused_point(const P &prm, const DXform &X, const FusedIO &io,
                                            int64_t i) {
  using R = double;
  const uint32_t ops = io.ops & kOps;
  const bool need_dir = ops & ((1u << VGB_OP_DISTANCE_TO_IN) | (1u << VGB_OP_DISTANCE_TO_OUT));
  const V3<R> m = {ldg(io.x + i), ldg(io.y + i), ldg(io.z + i)};
  const V3<R> l = xf_point(X, m);
  V3<R> d = {0, 0, 0};
  if (need_dir) d = {ldg(io.dx + i), ldg(io.dy + i), ldg(io.dz + i)};
  bool c = false;
  const bool dto_inside = io.flags & (VGB_FUSED_DTO_INSIDE_ONLY | VGB_FUSED_LOCAL_INSIDE_ONLY);
  const bool sto_inside = io.flags & VGB_FUSED_LOCAL_INSIDE_ONLY;
  if ((ops & (1u << VGB_OP_CONTAINS)) || dto_inside) c = Ops::contains(prm, l);
  if (ops & (1u << VGB_OP_CONTAINS)) static_cast<uint8_t *>(io.out[VGB_OP_CONTAINS])[i] = c;
  if (ops & (1u << VGB_OP_INSIDE))
    static_cast<int32_t *>(io.out[VGB_OP_INSIDE])[i] = Ops::inside(prm, l);
  if (ops & (1u << VGB_OP_SAFETY_TO_IN))
    static_cast<double *>(io.out[VGB_OP_SAFETY_TO_IN])[i] = Ops::safety_to_in(prm, l);
  if (ops & (1u << VGB_OP_SAFETY_TO_OUT)) {
    R r = Lim<R>::inf();
    if (!sto_inside || c) r = Ops::safety_to_out(prm, m);
    static_cast<double *>(io.out[VGB_OP_SAFETY_TO_OUT])[i] = r;
  }
  if (ops & (1u << VGB_OP_DISTANCE_TO_IN))
    static_cast<double *>(io.out[VGB_OP_DISTANCE_TO_IN])[i] =
        Ops::distance_to_in(prm, l, dti_dir<Ops>(X, d), ldg(io.step + i));
  if (ops & (1u << VGB_OP_DISTANCE_TO_OUT)) {
    R r = Lim<R>::inf();
    if (!dto_inside || c) r = Ops::distance_to_out(prm, m, d, ldg(io.step + i));
    static_cast<double *>(io.out[VGB_OP_DISTANCE_TO_OUT])[i] = r;
  }
}

template <class Ops, class P>
__global__ void __launch_bounds__(kBatchBlock) k_fused(const P prm, const DXform X,
                                                       const FusedIO io) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < io.n; i += stride)
    fused_point<Ops, P>(prm, X, io, i);
}

}  // namespace vgb
