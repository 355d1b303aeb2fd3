// api.cu -- the batch entry points of the C ABI (vgb_batch, vgb_batch_fused and
// the per-op forms).  Device pointers go straight to the kernels; host pointers
// are staged through device slots in chunks: copies in on one internal stream,
// kernels on a second, copies out on a third, so PCIe carries the inputs of one
// chunk and the results of an earlier one at the same time.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "dispatch.h"
#include "geometry.h"

using namespace vgb;

namespace {

enum PtrKind { kPtrNull = 0, kPtrDevice = 1, kPtrHost = 2 };

PtrKind classify(const void *p) {
  if (!p) return kPtrNull;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return kPtrHost;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return kPtrDevice;
  return kPtrHost;
}

bool op_needs_dir(int op) {
  return op == VGB_OP_DISTANCE_TO_IN || op == VGB_OP_DISTANCE_TO_OUT ||
         op == VGB_OP_DISTANCE_TO_IN_MINIMIZE || op == VGB_OP_DISTANCE_TO_OUT_NODE ||
         op == VGB_OP_PLACED_DISTANCE_TO_OUT;
}
bool op_needs_step(int op) {
  return op == VGB_OP_DISTANCE_TO_IN || op == VGB_OP_DISTANCE_TO_OUT ||
         op == VGB_OP_DISTANCE_TO_OUT_NODE || op == VGB_OP_PLACED_DISTANCE_TO_OUT;
}
bool op_needs_aux(int op) {
  return op == VGB_OP_DISTANCE_TO_IN_MINIMIZE || op == VGB_OP_DISTANCE_TO_OUT_NODE;
}
bool op_reads_out(int op) {
  return op == VGB_OP_DISTANCE_TO_IN_MINIMIZE || op == VGB_OP_SAFETY_TO_IN_MINIMIZE ||
         op == VGB_OP_SAFETY_TO_OUT_MINIMIZE;
}
bool op_reads_aux(int op) { return op == VGB_OP_DISTANCE_TO_IN_MINIMIZE; }
size_t out_size(int op) {
  if (op == VGB_OP_CONTAINS) return 1;
  if (op == VGB_OP_INSIDE) return 4;
  return 8;
}

vgb_status check_geometry(const vgb_geometry *g, int32_t placed, const char *fn) {
  if (!g) return set_error(VGB_EINVAL, "%s: geometry is NULL", fn);
  if (!g->closed) return set_error(VGB_EINVAL, "%s: geometry is not closed", fn);
  if (placed < 0 || placed >= (int32_t)g->placed.size())
    return set_error(VGB_EINVAL, "%s: unknown placed volume %d", fn, placed);
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != g->device)
    return set_error(VGB_EINVAL, "%s: current device %d is not the geometry's device %d", fn,
                     dev, g->device);
  return VGB_OK;
}

// Staged host-buffer calls.  A batch crosses PCIe in chunks through
// vgb_geometry::kStageSlots device slots.  One stream copies the chunks in, in
// order, so the copy engine finishes each chunk before it starts the next (two
// streams copying in at once would both finish late, and their kernels and
// copies out would then queue at the end); a second runs the kernels; a third
// copies the results out, in order.  Chunk c's copy-in waits for the copy-out of
// chunk c - kStageSlots (the slot's previous occupant), its kernel for its
// copy-in, its copy-out for its kernel.  The chunks shrink towards the end of the
// batch (halving down to kStageMin points), so the copy-out left after the last
// copy-in is short.  Measured on one B200 (55.6 GB/s in, 57.2 GB/s out, both at
// once 8 % slower than in alone): a fused 2^22-point call became copy-in bound.
constexpr int64_t kStageChunk = 1 << 20;  // points per chunk, at most
constexpr int64_t kStageMin = 1 << 16;    // the smallest chunk but the remainder

// Points of the next chunk when r points are left and slots hold cap points.
int64_t next_chunk(int64_t r, int64_t cap) {
  if (r <= kStageMin) return r;
  return std::min(cap, std::max(kStageMin, (r + 1) / 2));
}

// Internal streams, events and the staging buffer of a geometry (created on first use).
vgb_status ensure_staging(vgb_geometry *g, size_t bytes) {
  if (!g->staging_streams[0]) {
    cudaError_t e = cudaSuccess;
    for (cudaStream_t &st : g->staging_streams)
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->staging_start, cudaEventDisableTiming);
    for (auto &slot : g->staging_ev)
      for (cudaEvent_t &ev : slot)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_error(e, "vgb staging: stream/event create");
  }
  if (g->staging_bytes < bytes) {
    cudaFree(g->staging);
    g->staging = nullptr;
    g->staging_bytes = 0;
    cudaError_t e = cudaMalloc(&g->staging, bytes);
    if (e != cudaSuccess) return cuda_error(e, "vgb staging: cudaMalloc");
    g->staging_bytes = bytes;
  }
  return VGB_OK;
}

// Runs a host-buffer call over n points in chunks through slots of slot_bytes
// (sized by the caller for cap = min(n, kStageChunk) points):
//   copy_in(slot, b, m, stream)  -> cudaError_t: points [b, b + m) into the slot
//   launch(slot, m, stream)      -> vgb_status:  the kernel over the slot
//   copy_out(slot, b, m, stream) -> cudaError_t: the slot's results back
// Ordered after the work already on the caller's stream s; returns when every
// result is in host memory.  On an error it waits for the chunks in flight, so
// the buffer is free when the lock is released.
template <class In, class Run, class Out>
vgb_status staged_call(vgb_geometry *g, cudaStream_t s, int64_t n, int64_t cap,
                       size_t slot_bytes, In &&copy_in, Run &&launch, Out &&copy_out,
                       const char *fn) {
  constexpr int S = vgb_geometry::kStageSlots;
  std::lock_guard<std::mutex> lock(g->staging_mu);
  vgb_status st = ensure_staging(g, S * slot_bytes);
  if (st != VGB_OK) return st;
  cudaStream_t sin = g->staging_streams[0], sk = g->staging_streams[1],
               sout = g->staging_streams[2];
  auto drain = [&] {
    for (cudaStream_t q : g->staging_streams) cudaStreamSynchronize(q);
    cudaGetLastError();
  };
  auto fail = [&](cudaError_t err, const char *what) {
    char msg[128];
    std::snprintf(msg, sizeof msg, "%s: %s", fn, what);
    return cuda_error(err, msg);
  };
  cudaError_t e = cudaEventRecord(g->staging_start, s);
  for (cudaStream_t q : g->staging_streams)
    if (e == cudaSuccess) e = cudaStreamWaitEvent(q, g->staging_start, 0);
  if (e != cudaSuccess) return fail(e, "stream ordering");
  char *base = static_cast<char *>(g->staging);
  int64_t m = 0;
  for (int64_t b = 0, c = 0; b < n; b += m, ++c) {
    m = next_chunk(n - b, cap);
    const int sl = (int)(c % S);
    char *slot = base + sl * slot_bytes;
    cudaEvent_t *ev = g->staging_ev[sl];
    if (c >= S) e = cudaStreamWaitEvent(sin, ev[2], 0);
    if (e == cudaSuccess) e = copy_in(slot, b, m, sin);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], sin);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sk, ev[0], 0);
    if (e != cudaSuccess) {
      drain();
      return fail(e, "host-to-device copy");
    }
    if ((st = launch(slot, m, sk)) != VGB_OK) {
      drain();
      return st;
    }
    e = cudaEventRecord(ev[1], sk);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sout, ev[1], 0);
    if (e == cudaSuccess) e = copy_out(slot, b, m, sout);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2], sout);
    if (e != cudaSuccess) {
      drain();
      return fail(e, "device-to-host copy");
    }
  }
  for (cudaStream_t q : {sin, sk, sout})
    if (e == cudaSuccess) e = cudaStreamSynchronize(q);
  if (e != cudaSuccess) return fail(e, "synchronize");
  return VGB_OK;
}

}  // namespace

extern "C" {

vgb_status vgb_batch(const vgb_geometry *gc, int32_t placed, int32_t op, int64_t n,
                     const double *x, const double *y, const double *z, const double *dx,
                     const double *dy, const double *dz, const double *step_max, void *out,
                     int32_t *aux, int32_t daughter, int32_t precision, void *stream) {
  vgb_status st = check_geometry(gc, placed, "vgb_batch");
  if (st != VGB_OK) return st;
  vgb_geometry *g = const_cast<vgb_geometry *>(gc);
  if (op < 0 || op >= VGB_OP_COUNT) return set_error(VGB_EINVAL, "vgb_batch: unknown op %d", op);
  if (precision != VGB_PREC_FP64 && precision != VGB_PREC_FP32_REFINE)
    return set_error(VGB_EINVAL, "vgb_batch: unknown precision %d", precision);
  if (n < 0) return set_error(VGB_EINVAL, "vgb_batch: n < 0");
  if (n == 0) return VGB_OK;
  if (!x || !y || !z || !out) return set_error(VGB_EINVAL, "vgb_batch: NULL point or output");
  if (op_needs_dir(op) && (!dx || !dy || !dz))
    return set_error(VGB_EINVAL, "vgb_batch: op %d needs directions", op);
  if (op_needs_step(op) && !step_max)
    return set_error(VGB_EINVAL, "vgb_batch: op %d needs step_max", op);
  if (op_needs_aux(op) && !aux) return set_error(VGB_EINVAL, "vgb_batch: op %d needs aux", op);
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  const PtrKind kx = classify(x);
  const PtrKind ko = classify(out);
  if (kx == kPtrDevice && ko == kPtrDevice) {
    BatchIO io{x, y, z, dx, dy, dz, step_max, out, aux, n, daughter, 0};
    return launch_batch_f64(g, placed, op, io, s, precision);
  }
  if (kx != kPtrHost || ko != kPtrHost)
    return set_error(VGB_EINVAL, "vgb_batch: inputs and outputs must all be device or all host");

  // host buffers: staged chunk by chunk
  const bool nd = op_needs_dir(op), ns = op_needs_step(op), na = op_needs_aux(op);
  const size_t osz = out_size(op);
  const int64_t cap = n < kStageChunk ? n : kStageChunk;
  // every staged array starts on a 256-byte boundary
  auto span = [&](size_t elem) { return ((cap * elem + 255) / 256) * 256; };
  const size_t slot_bytes = 3 * span(8) + (nd ? 3 * span(8) : 0) + (ns ? span(8) : 0) +
                            span(osz) + (na ? span(4) : 0);
  struct Slot {
    double *x, *y, *z, *dx, *dy, *dz, *st;
    void *out;
    int32_t *aux;
  };
  auto carve = [&](char *p) {
    auto take = [&](size_t elem) {
      char *r = p;
      p += span(elem);
      return r;
    };
    Slot sl{};
    sl.x = (double *)take(8), sl.y = (double *)take(8), sl.z = (double *)take(8);
    if (nd) sl.dx = (double *)take(8), sl.dy = (double *)take(8), sl.dz = (double *)take(8);
    if (ns) sl.st = (double *)take(8);
    sl.out = take(osz);
    if (na) sl.aux = (int32_t *)take(4);
    return sl;
  };
  auto copy_in = [&](char *slot, int64_t b, int64_t m, cudaStream_t q) {
    const Slot sl = carve(slot);
    const size_t db = m * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(sl.x, x + b, db, cudaMemcpyHostToDevice, q);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.y, y + b, db, cudaMemcpyHostToDevice, q);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.z, z + b, db, cudaMemcpyHostToDevice, q);
    if (nd && e == cudaSuccess) e = cudaMemcpyAsync(sl.dx, dx + b, db, cudaMemcpyHostToDevice, q);
    if (nd && e == cudaSuccess) e = cudaMemcpyAsync(sl.dy, dy + b, db, cudaMemcpyHostToDevice, q);
    if (nd && e == cudaSuccess) e = cudaMemcpyAsync(sl.dz, dz + b, db, cudaMemcpyHostToDevice, q);
    if (ns && e == cudaSuccess)
      e = cudaMemcpyAsync(sl.st, step_max + b, db, cudaMemcpyHostToDevice, q);
    if (op_reads_out(op) && e == cudaSuccess)
      e = cudaMemcpyAsync(sl.out, static_cast<char *>(out) + b * osz, m * osz,
                          cudaMemcpyHostToDevice, q);
    if (op_reads_aux(op) && e == cudaSuccess)
      e = cudaMemcpyAsync(sl.aux, aux + b, m * 4, cudaMemcpyHostToDevice, q);
    return e;
  };
  auto run = [&](char *slot, int64_t m, cudaStream_t q) {
    const Slot sl = carve(slot);
    BatchIO io{sl.x, sl.y, sl.z, sl.dx, sl.dy, sl.dz, sl.st, sl.out, sl.aux, m, daughter, 0};
    return launch_batch_f64(g, placed, op, io, q, precision);
  };
  auto copy_out = [&](char *slot, int64_t b, int64_t m, cudaStream_t q) {
    const Slot sl = carve(slot);
    cudaError_t e = cudaMemcpyAsync(static_cast<char *>(out) + b * osz, sl.out, m * osz,
                                    cudaMemcpyDeviceToHost, q);
    if (na && e == cudaSuccess) e = cudaMemcpyAsync(aux + b, sl.aux, m * 4, cudaMemcpyDeviceToHost, q);
    return e;
  };
  return staged_call(g, s, n, cap, slot_bytes, copy_in, run, copy_out, "vgb_batch");
}

vgb_status vgb_batch_fused(const vgb_geometry *gc, int32_t placed, uint32_t ops, int64_t n,
                           const double *x, const double *y, const double *z, const double *dx,
                           const double *dy, const double *dz, const double *step_max,
                           void *const *outs, uint32_t flags, int32_t precision, void *stream) {
  vgb_status st = check_geometry(gc, placed, "vgb_batch_fused");
  if (st != VGB_OK) return st;
  const uint32_t allowed = (1u << VGB_OP_CONTAINS) | (1u << VGB_OP_INSIDE) |
                           (1u << VGB_OP_DISTANCE_TO_IN) | (1u << VGB_OP_DISTANCE_TO_OUT) |
                           (1u << VGB_OP_SAFETY_TO_IN) | (1u << VGB_OP_SAFETY_TO_OUT);
  if (ops & ~allowed) return set_error(VGB_EINVAL, "vgb_batch_fused: unsupported op mask 0x%x", ops);
  if (precision != VGB_PREC_FP64 && precision != VGB_PREC_FP32_REFINE)
    return set_error(VGB_EINVAL, "vgb_batch_fused: unknown precision %d", precision);
  if (precision == VGB_PREC_FP32_REFINE)
    return set_error(VGB_ENOTSUP, "vgb_batch_fused: the FP32+refine form is not available");
  if (n < 0) return set_error(VGB_EINVAL, "vgb_batch_fused: n < 0");
  if (n == 0 || ops == 0) return VGB_OK;
  if (!x || !y || !z || !outs) return set_error(VGB_EINVAL, "vgb_batch_fused: NULL argument");
  const bool nd = ops & ((1u << VGB_OP_DISTANCE_TO_IN) | (1u << VGB_OP_DISTANCE_TO_OUT));
  if (nd && (!dx || !dy || !dz || !step_max))
    return set_error(VGB_EINVAL, "vgb_batch_fused: distances need directions and step_max");
  FusedIO io;
  std::memset(&io, 0, sizeof(io));
  io.x = x; io.y = y; io.z = z; io.dx = dx; io.dy = dy; io.dz = dz; io.step = step_max;
  for (int k = 0; k < 6; ++k) {
    if (!(ops & (1u << k))) continue;
    if (!outs[k]) return set_error(VGB_EINVAL, "vgb_batch_fused: output %d is NULL", k);
    io.out[k] = outs[k];
  }
  io.n = n;
  io.ops = ops;
  io.flags = flags;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const PtrKind kx = classify(x);
  bool all_host = kx == kPtrHost, all_dev = kx == kPtrDevice;
  for (int k = 0; k < 6; ++k) {
    if (!io.out[k]) continue;
    const PtrKind ko = classify(io.out[k]);
    all_host = all_host && ko == kPtrHost;
    all_dev = all_dev && ko == kPtrDevice;
  }
  if (all_dev) return launch_fused_f64(gc, placed, io, s);
  if (!all_host)
    return set_error(VGB_EINVAL, "vgb_batch_fused: inputs and outputs must all be device or all host");

  // host buffers: the points (and directions, steps) cross once per chunk for
  // all the ops, staged as in vgb_batch
  vgb_geometry *g = const_cast<vgb_geometry *>(gc);
  const int64_t cap = n < kStageChunk ? n : kStageChunk;
  auto span = [&](size_t elem) { return ((cap * elem + 255) / 256) * 256; };
  const int nin = nd ? 7 : 3;
  size_t slot_bytes = nin * span(8);
  for (int k = 0; k < 6; ++k)
    if (io.out[k]) slot_bytes += span(out_size(k));
  const double *hin[7] = {x, y, z, dx, dy, dz, step_max};
  // the slot: the nin input arrays, then each requested output
  auto carve = [&](char *p, int64_t m) {
    FusedIO cio = io;
    double *din[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int i = 0; i < nin; ++i) {
      din[i] = reinterpret_cast<double *>(p);
      p += span(8);
    }
    cio.x = din[0], cio.y = din[1], cio.z = din[2];
    cio.dx = din[3], cio.dy = din[4], cio.dz = din[5], cio.step = din[6];
    for (int k = 0; k < 6; ++k) {
      if (!io.out[k]) continue;
      cio.out[k] = p;
      p += span(out_size(k));
    }
    cio.n = m;
    return cio;
  };
  auto copy_in = [&](char *slot, int64_t b, int64_t m, cudaStream_t q) {
    const FusedIO cio = carve(slot, m);
    const double *din[7] = {cio.x, cio.y, cio.z, cio.dx, cio.dy, cio.dz, cio.step};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < nin && e == cudaSuccess; ++i)
      e = cudaMemcpyAsync(const_cast<double *>(din[i]), hin[i] + b, m * sizeof(double),
                          cudaMemcpyHostToDevice, q);
    return e;
  };
  auto run = [&](char *slot, int64_t m, cudaStream_t q) {
    return launch_fused_f64(gc, placed, carve(slot, m), q);
  };
  auto copy_out = [&](char *slot, int64_t b, int64_t m, cudaStream_t q) {
    const FusedIO cio = carve(slot, m);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 6 && e == cudaSuccess; ++k) {
      if (!io.out[k]) continue;
      const size_t osz = out_size(k);
      e = cudaMemcpyAsync(static_cast<char *>(io.out[k]) + b * osz, cio.out[k], m * osz,
                          cudaMemcpyDeviceToHost, q);
    }
    return e;
  };
  return staged_call(g, s, n, cap, slot_bytes, copy_in, run, copy_out, "vgb_batch_fused");
}

vgb_status vgb_Contains(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                        const double *y, const double *z, uint8_t *out, void *stream) {
  return vgb_batch(g, placed, VGB_OP_CONTAINS, n, x, y, z, nullptr, nullptr, nullptr, nullptr,
                   out, nullptr, 0, VGB_PREC_FP64, stream);
}
vgb_status vgb_Inside(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                      const double *y, const double *z, int32_t *out, void *stream) {
  return vgb_batch(g, placed, VGB_OP_INSIDE, n, x, y, z, nullptr, nullptr, nullptr, nullptr, out,
                   nullptr, 0, VGB_PREC_FP64, stream);
}
vgb_status vgb_DistanceToIn(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                            const double *y, const double *z, const double *dx,
                            const double *dy, const double *dz, const double *step_max,
                            double *out, void *stream) {
  return vgb_batch(g, placed, VGB_OP_DISTANCE_TO_IN, n, x, y, z, dx, dy, dz, step_max, out,
                   nullptr, 0, VGB_PREC_FP64, stream);
}
vgb_status vgb_DistanceToOut(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                             const double *y, const double *z, const double *dx,
                             const double *dy, const double *dz, const double *step_max,
                             double *out, void *stream) {
  return vgb_batch(g, placed, VGB_OP_DISTANCE_TO_OUT, n, x, y, z, dx, dy, dz, step_max, out,
                   nullptr, 0, VGB_PREC_FP64, stream);
}
vgb_status vgb_SafetyToIn(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                          const double *y, const double *z, double *out, void *stream) {
  return vgb_batch(g, placed, VGB_OP_SAFETY_TO_IN, n, x, y, z, nullptr, nullptr, nullptr,
                   nullptr, out, nullptr, 0, VGB_PREC_FP64, stream);
}
vgb_status vgb_SafetyToOut(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                           const double *y, const double *z, double *out, void *stream) {
  return vgb_batch(g, placed, VGB_OP_SAFETY_TO_OUT, n, x, y, z, nullptr, nullptr, nullptr,
                   nullptr, out, nullptr, 0, VGB_PREC_FP64, stream);
}

}  // extern "C"
