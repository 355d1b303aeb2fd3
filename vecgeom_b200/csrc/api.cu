// api.cu -- the batch entry points of the C ABI (vgb_batch, vgb_batch_fused and
// the per-op forms).  Device pointers go straight to the kernels; host pointers
// are staged through device buffers in chunks, on two internal streams so the
// copy engines overlap the kernels of neighbouring chunks.
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

// Points per staged chunk of a host-buffer call (measured: 512 K-point chunks
// gave no faster end-to-end rate than 1 M; the copies are PCIe-bound either way).
constexpr int64_t kStageChunk = 1 << 20;

// Internal streams and the staging buffer of a geometry (created on first use).
vgb_status ensure_staging(vgb_geometry *g, size_t bytes) {
  if (!g->staging_streams[0]) {
    cudaError_t e = cudaStreamCreateWithFlags(&g->staging_streams[0], cudaStreamNonBlocking);
    if (e == cudaSuccess)
      e = cudaStreamCreateWithFlags(&g->staging_streams[1], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->staging_start, cudaEventDisableTiming);
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

  // host buffers: stage chunk by chunk
  const bool nd = op_needs_dir(op), ns = op_needs_step(op), na = op_needs_aux(op);
  const size_t osz = out_size(op);
  const int64_t chunk = n < kStageChunk ? n : kStageChunk;
  // every staged array starts on a 256-byte boundary; one half per stream
  auto span = [&](size_t elem) { return ((chunk * elem + 255) / 256) * 256; };
  const size_t half = 3 * span(8) + (nd ? 3 * span(8) : 0) + (ns ? span(8) : 0) + span(osz) +
                      (na ? span(4) : 0);
  std::lock_guard<std::mutex> lock(g->staging_mu);
  if ((st = ensure_staging(g, 2 * half)) != VGB_OK) return st;
  cudaStream_t *sts = g->staging_streams;
  cudaError_t e = cudaEventRecord(g->staging_start, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(sts[0], g->staging_start, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(sts[1], g->staging_start, 0);
  if (e != cudaSuccess) return cuda_error(e, "vgb_batch: stream ordering");
  char *base = static_cast<char *>(g->staging);
  for (int64_t b = 0, k = 0; b < n; b += chunk, ++k) {
    const int64_t m = (n - b < chunk) ? (n - b) : chunk;
    cudaStream_t cs = sts[k & 1];
    char *p = base + (k & 1) * half;
    auto carve = [&](size_t elem) {
      char *r = p;
      p += ((chunk * elem + 255) / 256) * 256;
      return r;
    };
    double *dxp = (double *)carve(8), *dyp = (double *)carve(8), *dzp = (double *)carve(8);
    double *ddx = nd ? (double *)carve(8) : nullptr;
    double *ddy = nd ? (double *)carve(8) : nullptr;
    double *ddz = nd ? (double *)carve(8) : nullptr;
    double *dst = ns ? (double *)carve(8) : nullptr;
    void *dout = carve(osz);
    int32_t *daux = na ? (int32_t *)carve(4) : nullptr;
    const size_t db = m * sizeof(double);
    e = cudaMemcpyAsync(dxp, x + b, db, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dyp, y + b, db, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dzp, z + b, db, cudaMemcpyHostToDevice, cs);
    if (nd && e == cudaSuccess) e = cudaMemcpyAsync(ddx, dx + b, db, cudaMemcpyHostToDevice, cs);
    if (nd && e == cudaSuccess) e = cudaMemcpyAsync(ddy, dy + b, db, cudaMemcpyHostToDevice, cs);
    if (nd && e == cudaSuccess) e = cudaMemcpyAsync(ddz, dz + b, db, cudaMemcpyHostToDevice, cs);
    if (ns && e == cudaSuccess)
      e = cudaMemcpyAsync(dst, step_max + b, db, cudaMemcpyHostToDevice, cs);
    if (op_reads_out(op) && e == cudaSuccess)
      e = cudaMemcpyAsync(dout, static_cast<char *>(out) + b * osz, m * osz,
                          cudaMemcpyHostToDevice, cs);
    if (op_reads_aux(op) && e == cudaSuccess)
      e = cudaMemcpyAsync(daux, aux + b, m * 4, cudaMemcpyHostToDevice, cs);
    if (e != cudaSuccess) return cuda_error(e, "vgb_batch: host-to-device copy");
    BatchIO io{dxp, dyp, dzp, ddx, ddy, ddz, dst, dout, daux, m, daughter, 0};
    if ((st = launch_batch_f64(g, placed, op, io, cs, precision)) != VGB_OK) return st;
    e = cudaMemcpyAsync(static_cast<char *>(out) + b * osz, dout, m * osz,
                        cudaMemcpyDeviceToHost, cs);
    if (na && e == cudaSuccess)
      e = cudaMemcpyAsync(aux + b, daux, m * 4, cudaMemcpyDeviceToHost, cs);
    if (e != cudaSuccess) return cuda_error(e, "vgb_batch: device-to-host copy");
  }
  e = cudaStreamSynchronize(sts[0]);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sts[1]);
  if (e != cudaSuccess) return cuda_error(e, "vgb_batch: synchronize");
  return VGB_OK;
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
  // all the ops, on the two internal streams as in vgb_batch
  vgb_geometry *g = const_cast<vgb_geometry *>(gc);
  const int64_t chunk = n < kStageChunk ? n : kStageChunk;
  auto span = [&](size_t elem) { return ((chunk * elem + 255) / 256) * 256; };
  size_t half = 3 * span(8) + (nd ? 4 * span(8) : 0);
  for (int k = 0; k < 6; ++k)
    if (io.out[k]) half += span(out_size(k));
  std::lock_guard<std::mutex> lock(g->staging_mu);
  if ((st = ensure_staging(g, 2 * half)) != VGB_OK) return st;
  cudaStream_t *sts = g->staging_streams;
  cudaError_t e = cudaEventRecord(g->staging_start, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(sts[0], g->staging_start, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(sts[1], g->staging_start, 0);
  if (e != cudaSuccess) return cuda_error(e, "vgb_batch_fused: stream ordering");
  char *base = static_cast<char *>(g->staging);
  const double *hin[7] = {x, y, z, dx, dy, dz, step_max};
  for (int64_t b = 0, c = 0; b < n; b += chunk, ++c) {
    const int64_t m = (n - b < chunk) ? (n - b) : chunk;
    cudaStream_t cs = sts[c & 1];
    char *p = base + (c & 1) * half;
    double *din[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int i = 0; i < (nd ? 7 : 3); ++i) {
      din[i] = reinterpret_cast<double *>(p);
      p += span(8);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(din[i], hin[i] + b, m * sizeof(double), cudaMemcpyHostToDevice, cs);
    }
    if (e != cudaSuccess) return cuda_error(e, "vgb_batch_fused: host-to-device copy");
    FusedIO cio = io;
    cio.x = din[0]; cio.y = din[1]; cio.z = din[2];
    cio.dx = din[3]; cio.dy = din[4]; cio.dz = din[5]; cio.step = din[6];
    for (int k = 0; k < 6; ++k) {
      if (!io.out[k]) continue;
      cio.out[k] = p;
      p += span(out_size(k));
    }
    cio.n = m;
    if ((st = launch_fused_f64(gc, placed, cio, cs)) != VGB_OK) return st;
    for (int k = 0; k < 6 && e == cudaSuccess; ++k) {
      if (!io.out[k]) continue;
      const size_t osz = out_size(k);
      e = cudaMemcpyAsync(static_cast<char *>(io.out[k]) + b * osz, cio.out[k], m * osz,
                          cudaMemcpyDeviceToHost, cs);
    }
    if (e != cudaSuccess) return cuda_error(e, "vgb_batch_fused: device-to-host copy");
  }
  e = cudaStreamSynchronize(sts[0]);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sts[1]);
  if (e != cudaSuccess) return cuda_error(e, "vgb_batch_fused: synchronize");
  return VGB_OK;
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
