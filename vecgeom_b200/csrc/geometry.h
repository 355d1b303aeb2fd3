// geometry.h -- host-side geometry registry of libvgb and its device image.
//
// The reference keeps an object graph (Unplaced*, LogicalVolume, VPlacedVolume,
// Transformation3D) and copies it to the GPU object by object with one
// constructor kernel each (source/CudaManager.cpp:39-322,
// backend/cuda/Interface.h:24-32).  Here the same graph is recorded in flat
// tables and vgb_geometry_close() uploads each table with one copy:
//   params    double pool; each unplaced shape owns a 16-byte aligned record
//   xforms    DXform per Transformation3D (effective matrix, see vgb_core.cuh)
//   placed    {unplaced, logical, xform} per placed volume
//   logicals  {unplaced, first daughter, daughter count} per logical volume
//   daughters placed ids, CSR over logicals, in insertion order
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vgb.h"
#include "vgb_core.cuh"

namespace vgb {

struct UnplacedRec {
  int32_t type;       // vgb_shape_type
  int32_t param_off;  // offset in doubles into the param pool (16-byte aligned)
  int32_t param_len;  // length in doubles
  int32_t extra;      // shape-specific (e.g. boolean left placed id)
};

struct PlacedRec {
  int32_t unplaced;
  int32_t logical;
  int32_t xform;      // index of the placement's effective DXform
  int32_t raw_xform;  // the Transformation3D it was placed with
};

struct LogicalRec {
  int32_t unplaced;
  int32_t dfirst;
  int32_t dcount;
  int32_t pad;
};

struct RawXform {
  double t[3];
  double r[9];
  int trans_code;  // 0 kIdentity, -1 kGeneric
  int rot_code;    // specialised code, 0x200 identity or -1 generic
};

// Transformation3D with its property flags, as the navigator composes it
// (base/Transformation3D.h:674-743 MultiplyFromRight, :598-632 InverseTransform;
// flags from SetProperties, source/Transformation3D.cpp:81-90).
enum : uint32_t { kNavHasTrans = 1, kNavHasRot = 2, kNavIdentity = 4 };
struct NavXform {
  double t[3];
  double r[9];
  uint32_t flags;
  uint32_t pad;
};

struct DeviceImage {
  double *params = nullptr;
  UnplacedRec *unplaced = nullptr;
  DXform *xforms = nullptr;
  NavXform *raw = nullptr;
  PlacedRec *placed = nullptr;
  LogicalRec *logicals = nullptr;
  int32_t *daughters = nullptr;
  uint32_t *nav_flags = nullptr;  // navigation error bits (VGB_NAV_ERR_*)
  float *pl_box = nullptr;        // per placed: enclosing box in the mother's frame
  float *ab_box = nullptr;        // per placed: ABBoxManager's aligned box (float), mother frame
  float4 *ab_slot = nullptr;      // per daughter slot (CSR order): the same box as 2 float4
  int64_t bytes = 0;
};

}  // namespace vgb

namespace vgb {
// Constructor forms of a shape (the trapezoid has two)
enum : int32_t { kCtorDefault = 0, kCtorCorners = 1 };
}  // namespace vgb

struct vgb_geometry {
  std::vector<vgb::UnplacedRec> unplaced;
  std::vector<int32_t> ctor_form;               // per unplaced: kCtorDefault / kCtorCorners
  std::vector<std::vector<double>> ctor_args;   // per unplaced: its constructor's arguments
  std::vector<double> params;
  std::vector<vgb::RawXform> raw_xforms;
  std::vector<vgb::DXform> xforms;  // per (placed volume), effective for its shape
  std::vector<std::string> labels;
  std::vector<vgb::LogicalRec> logicals;
  std::vector<std::vector<int32_t>> logical_daughters;
  std::vector<vgb::PlacedRec> placed;
  std::vector<int32_t> daughters;
  std::vector<vgb::NavXform> nav_raw;  // per Transformation3D, for the navigator
  std::vector<float> bbox;             // per unplaced: 6 floats, enclosing box (own frame)
  std::vector<float> pl_box;           // per placed: 6 floats, enclosing box (mother frame)
  std::vector<double> ab_box_d;        // per placed: ABBoxManager::ComputeABBox (lower, upper)
  std::vector<float> ab_box;           // the same boxes rounded to float, as navigated
  std::vector<float4> ab_slot;         // per daughter slot: (lower, 0), (upper, 0)
  bool abbox_ok = true;                // every placed volume's shape has an Extent
  uint32_t type_mask = 0;              // bit t set when a shape of type t exists
  int32_t world = -1;
  int32_t max_depth = 0;
  int32_t max_daughters = 0;  // the most daughters of any logical volume
  bool closed = false;
  int device = -1;
  vgb::DeviceImage dev;
  // host-pointer calls stage through one device buffer of kStageSlots chunk slots on
  // three internal streams (copies in, kernels, copies out) ordered by per-slot events
  static constexpr int kStageSlots = 3;
  std::mutex staging_mu;  // serialises host-pointer calls that share the buffer
  void *staging = nullptr;
  size_t staging_bytes = 0;
  cudaStream_t staging_streams[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t staging_start = nullptr;
  // per slot: its copy-in done, its kernel done, its copy-out done
  cudaEvent_t staging_ev[kStageSlots][3] = {};
};

namespace vgb {
// Error reporting (thread-local message, status return).
vgb_status set_error(vgb_status s, const char *fmt, ...);
vgb_status cuda_error(cudaError_t e, const char *what);
void count_launch(int n = 1);
// The device transform of a placement: the specialised form the reference
// picks for it, or Transform<kGeneric,kGeneric> when generic_only is set.
DXform effective_xform(const RawXform &x, bool generic_only);
// Host tables derived at close: daughters CSR, depth, navigator transforms and
// the shape-type mask.  No device work.
vgb_status prepare_tables(vgb_geometry *g);
// Axis-aligned box (min xyz, max xyz) in the shape's own frame that encloses
// the shape; false for unknown types.
bool shape_bbox(const vgb_geometry *g, int32_t unplaced, double box[6]);
// The reference's Extent of a shape record (lower and upper corner in its own
// frame, VPlacedVolume::Extent, volumes/PlacedVolume.h:260); false for unknown types.
bool reference_extent(int type, const double *rec, double lo[3], double hi[3]);
// Appends a shape record to the parameter pool (16-byte aligned).
vgb_status add_unplaced(vgb_geometry *g, int type, const void *rec, size_t bytes, int32_t extra,
                        int32_t *id);

// The host copy of a shape's parameter record (for passing by value).
inline const void *shape_params(const vgb_geometry *g, int32_t unplaced) {
  return g->params.data() + g->unplaced[unplaced].param_off;
}
// Device address of a shape's parameter record.
inline const double *shape_params_dev(const vgb_geometry *g, int32_t unplaced) {
  return g->dev.params + g->unplaced[unplaced].param_off;
}
}  // namespace vgb

#define VGB_CHECK_G(g)                                                          \
  do {                                                                          \
    if (!(g)) return vgb::set_error(VGB_EINVAL, "%s: geometry is NULL", __func__);   \
  } while (0)
#define VGB_CHECK_OPEN(g)                                                       \
  do {                                                                          \
    VGB_CHECK_G(g);                                                             \
    if ((g)->closed)                                                            \
      return vgb::set_error(VGB_EINVAL, "%s: geometry is closed", __func__);         \
  } while (0)
