// geometry.cu -- geometry construction, derived shape parameters and the bulk
// device upload (replaces CudaManager, source/CudaManager.cpp:39-322).
//
// Host code here is compiled with -ffp-contract=off: the derived parameters of
// each shape are computed with the same formulas and rounding as the reference
// constructors, so the device kernels see bit-identical constants.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>

#include "geometry.h"
#include "shapes.cuh"

namespace vgb {

static thread_local char g_err[512] = "";
static thread_local int64_t g_launches = 0;

vgb_status set_error(vgb_status s, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return s;
}

vgb_status cuda_error(cudaError_t e, const char *what) {
  if (e == cudaErrorMemoryAllocation)
    return set_error(VGB_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
  return set_error(VGB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

void count_launch(int n) { g_launches += n; }

// ---------------------------------------------------------------------------
// Transformation3D (source/Transformation3D.cpp)
// ---------------------------------------------------------------------------

// :138-150 GenerateRotationCode
static int gen_rot_code(const double *r) {
  int code = 0;
  for (int i = 0; i < 9; ++i) code |= (1 << i) * (std::fabs(r[i]) > kTolerance);
  if (code == 0x111 && (r[0] == 1. && r[4] == 1. && r[8] == 1.)) code = 0x200;
  return code;
}

// management/TransformationSpecializations.icc: codes with a specialised
// placed volume; everything else runs the generic rotation.
static int specialised_rot(int code) {
  static const int codes[] = {0x1b1, 0x18e, 0x076, 0x16a, 0x155, 0x0ad, 0x0dc, 0x0e3,
                              0x11b, 0x0a1, 0x10a, 0x046, 0x062, 0x054, 0x111, 0x200};
  for (int c : codes)
    if (c == code) return code;
  return -1;
}

static void set_codes(RawXform &x) {
  // :80-89 SetProperties; source/UnplacedVolume.cpp:23-24
  const bool has_t = std::fabs(x.t[0]) > kTolerance || std::fabs(x.t[1]) > kTolerance ||
                     std::fabs(x.t[2]) > kTolerance;
  x.trans_code = has_t ? -1 : 0;
  x.rot_code = specialised_rot(gen_rot_code(x.r));
}

// The effective device transform of one placement.  generic_only mirrors
// shapes whose placed volumes always take Transform<kGeneric,kGeneric>
// (source/UnplacedPolyhedron.cpp:321-333).
DXform effective_xform(const RawXform &x, bool generic_only) {
  DXform d;
  std::memset(&d, 0, sizeof(d));
  const int tcode = generic_only ? -1 : x.trans_code;
  const int rcode = generic_only ? -1 : x.rot_code;
  if (tcode != 0) {
    d.flags |= kXfHasTrans;
    for (int i = 0; i < 3; ++i) d.t[i] = x.t[i];
  }
  if (rcode != 0x200) {
    d.flags |= kXfHasRot;
    for (int i = 0; i < 9; ++i) {
      const bool keep = (rcode == -1) || ((rcode >> i) & 1);
      d.r[i] = keep ? x.r[i] : 0.;
    }
    if (rcode == 0x16a) d.flags |= kXfQuirk16A;
  } else {
    d.r[0] = d.r[4] = d.r[8] = 1.;
  }
  return d;
}

}  // namespace vgb

using namespace vgb;

vgb_status vgb::add_unplaced(vgb_geometry *g, int type, const void *rec, size_t bytes,
                             int32_t extra, int32_t *id) {
  // 16-byte aligned records in the pool
  while (g->params.size() % 2) g->params.push_back(0.);
  const size_t nd = (bytes + sizeof(double) - 1) / sizeof(double);
  UnplacedRec u;
  u.type = type;
  u.param_off = (int32_t)g->params.size();
  u.param_len = (int32_t)nd;
  u.extra = extra;
  g->params.resize(g->params.size() + nd + (nd % 2), 0.);
  std::memcpy(g->params.data() + u.param_off, rec, bytes);
  g->unplaced.push_back(u);
  g->ctor_form.push_back(kCtorDefault);
  g->ctor_args.emplace_back();
  if (id) *id = (int32_t)g->unplaced.size() - 1;
  return VGB_OK;
}

// Depth of the tree below a logical volume (GeoManager::getMaxDepth counts
// levels from the world, management/GeoManager.h:191).
static int depth_of(const vgb_geometry *g, int32_t logical, int guard) {
  if (guard > 64) return -1;
  int best = 0;
  for (int32_t d : g->logical_daughters[logical]) {
    const int sub = depth_of(g, g->placed[d].logical, guard + 1);
    if (sub < 0) return -1;
    if (sub > best) best = sub;
  }
  return best + 1;
}

template <class T>
static vgb_status upload(const std::vector<T> &h, T **d, int64_t *bytes) {
  const size_t n = h.empty() ? 1 : h.size();
  cudaError_t e = cudaMalloc((void **)d, n * sizeof(T));
  if (e != cudaSuccess) return cuda_error(e, "vgb_geometry_close: cudaMalloc");
  *bytes += (int64_t)(n * sizeof(T));
  if (!h.empty()) {
    e = cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "vgb_geometry_close: cudaMemcpy");
  }
  return VGB_OK;
}

extern "C" {

const char *vgb_last_error(void) { return vgb::g_err; }
const char *vgb_version(void) { return "vgb 0.1 (sm_100a)"; }
int64_t vgb_launch_count(void) { return vgb::g_launches; }
void vgb_launch_count_reset(void) { vgb::g_launches = 0; }

vgb_status vgb_geometry_create(vgb_geometry **g) {
  if (!g) return set_error(VGB_EINVAL, "vgb_geometry_create: out pointer is NULL");
  *g = new (std::nothrow) vgb_geometry();
  if (!*g) return set_error(VGB_ENOMEM, "vgb_geometry_create: out of host memory");
  return VGB_OK;
}

vgb_status vgb_geometry_destroy(vgb_geometry *g) {
  if (!g) return VGB_OK;
  if (g->device >= 0) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    cudaFree(g->dev.params);
    cudaFree(g->dev.unplaced);
    cudaFree(g->dev.xforms);
    cudaFree(g->dev.raw);
    cudaFree(g->dev.nav_flags);
    cudaFree(g->dev.pl_box);
    cudaFree(g->dev.ab_box);
    cudaFree(g->dev.ab_slot);
    cudaFree(g->dev.placed);
    cudaFree(g->dev.logicals);
    cudaFree(g->dev.daughters);
    cudaFree(g->staging);
    for (cudaStream_t st : g->staging_streams)
      if (st) cudaStreamDestroy(st);
    if (g->staging_start) cudaEventDestroy(g->staging_start);
    for (auto &slot : g->staging_ev)
      for (cudaEvent_t ev : slot)
        if (ev) cudaEventDestroy(ev);
    cudaSetDevice(prev);
  }
  delete g;
  return VGB_OK;
}

vgb_status vgb_transformation(vgb_geometry *g, double tx, double ty, double tz, double phi,
                              double theta, double psi, int32_t *id) {
  VGB_CHECK_OPEN(g);
  RawXform x;
  // source/Transformation3D.cpp:93-114 SetRotation(phi, theta, psi), degrees
  const double sinphi = std::sin(kDegToRad * phi), cosphi = std::cos(kDegToRad * phi);
  const double sinthe = std::sin(kDegToRad * theta), costhe = std::cos(kDegToRad * theta);
  const double sinpsi = std::sin(kDegToRad * psi), cospsi = std::cos(kDegToRad * psi);
  x.t[0] = tx;
  x.t[1] = ty;
  x.t[2] = tz;
  x.r[0] = cospsi * cosphi - costhe * sinphi * sinpsi;
  x.r[1] = -sinpsi * cosphi - costhe * sinphi * cospsi;
  x.r[2] = sinthe * sinphi;
  x.r[3] = cospsi * sinphi + costhe * cosphi * sinpsi;
  x.r[4] = -sinpsi * sinphi + costhe * cosphi * cospsi;
  x.r[5] = -sinthe * cosphi;
  x.r[6] = sinpsi * sinthe;
  x.r[7] = cospsi * sinthe;
  x.r[8] = costhe;
  set_codes(x);
  g->raw_xforms.push_back(x);
  if (id) *id = (int32_t)g->raw_xforms.size() - 1;
  return VGB_OK;
}

vgb_status vgb_transformation_matrix(vgb_geometry *g, double tx, double ty, double tz,
                                     const double *r9, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!r9) return set_error(VGB_EINVAL, "vgb_transformation_matrix: r9 is NULL");
  RawXform x;
  x.t[0] = tx;
  x.t[1] = ty;
  x.t[2] = tz;
  for (int i = 0; i < 9; ++i) x.r[i] = r9[i];
  set_codes(x);
  g->raw_xforms.push_back(x);
  if (id) *id = (int32_t)g->raw_xforms.size() - 1;
  return VGB_OK;
}

vgb_status vgb_logical_volume(vgb_geometry *g, const char *label, int32_t unplaced,
                              int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (unplaced < 0 || unplaced >= (int32_t)g->unplaced.size())
    return set_error(VGB_EINVAL, "vgb_logical_volume: unknown unplaced id %d", unplaced);
  LogicalRec l;
  l.unplaced = unplaced;
  l.dfirst = 0;
  l.dcount = 0;
  l.pad = 0;
  g->logicals.push_back(l);
  g->logical_daughters.emplace_back();
  g->labels.push_back(label ? label : "");
  if (id) *id = (int32_t)g->logicals.size() - 1;
  return VGB_OK;
}

vgb_status vgb_place(vgb_geometry *g, int32_t logical, int32_t transformation,
                     int32_t *placed) {
  VGB_CHECK_OPEN(g);
  if (logical < 0 || logical >= (int32_t)g->logicals.size())
    return set_error(VGB_EINVAL, "vgb_place: unknown logical volume %d", logical);
  if (transformation < 0 || transformation >= (int32_t)g->raw_xforms.size())
    return set_error(VGB_EINVAL, "vgb_place: unknown transformation %d", transformation);
  PlacedRec p;
  p.logical = logical;
  p.unplaced = g->logicals[logical].unplaced;
  p.xform = (int32_t)g->xforms.size();
  p.raw_xform = transformation;
  const int type = g->unplaced[p.unplaced].type;
  g->xforms.push_back(
      effective_xform(g->raw_xforms[transformation], type == VGB_SHAPE_POLYHEDRON));
  g->placed.push_back(p);
  if (placed) *placed = (int32_t)g->placed.size() - 1;
  return VGB_OK;
}

vgb_status vgb_place_daughter(vgb_geometry *g, int32_t mother_logical, int32_t daughter_logical,
                              int32_t transformation, int32_t *placed) {
  VGB_CHECK_OPEN(g);
  if (mother_logical < 0 || mother_logical >= (int32_t)g->logicals.size())
    return set_error(VGB_EINVAL, "vgb_place_daughter: unknown mother %d", mother_logical);
  int32_t id = -1;
  vgb_status s = vgb_place(g, daughter_logical, transformation, &id);
  if (s != VGB_OK) return s;
  g->logical_daughters[mother_logical].push_back(id);
  if (placed) *placed = id;
  return VGB_OK;
}

vgb_status vgb_set_world(vgb_geometry *g, int32_t placed) {
  VGB_CHECK_OPEN(g);
  if (placed < 0 || placed >= (int32_t)g->placed.size())
    return set_error(VGB_EINVAL, "vgb_set_world: unknown placed volume %d", placed);
  g->world = placed;
  return VGB_OK;
}

}  // extern "C"

vgb_status vgb::prepare_tables(vgb_geometry *g) {
  // CSR of daughters in insertion order (source/LogicalVolume.cpp:84-102)
  g->daughters.clear();
  for (size_t l = 0; l < g->logicals.size(); ++l) {
    g->logicals[l].dfirst = (int32_t)g->daughters.size();
    g->logicals[l].dcount = (int32_t)g->logical_daughters[l].size();
    for (int32_t d : g->logical_daughters[l]) g->daughters.push_back(d);
  }
  g->max_daughters = 0;
  for (const LogicalRec &l : g->logicals)
    if (l.dcount > g->max_daughters) g->max_daughters = l.dcount;
  if (g->world >= 0) {
    g->max_depth = depth_of(g, g->placed[g->world].logical, 0);
    if (g->max_depth < 0)
      return set_error(VGB_EINVAL, "vgb_geometry_close: volume tree deeper than 64 levels");
  }
  g->nav_raw.resize(g->raw_xforms.size());
  for (size_t i = 0; i < g->raw_xforms.size(); ++i) {
    const RawXform &x = g->raw_xforms[i];
    NavXform &n = g->nav_raw[i];
    std::memset(&n, 0, sizeof(n));
    for (int k = 0; k < 3; ++k) n.t[k] = x.t[k];
    for (int k = 0; k < 9; ++k) n.r[k] = x.r[k];
    const bool has_t = x.trans_code != 0, has_r = x.rot_code != 0x200;
    n.flags = (has_t ? kNavHasTrans : 0u) | (has_r ? kNavHasRot : 0u) |
              ((!has_t && !has_r) ? kNavIdentity : 0u);
  }
  g->type_mask = 0;
  for (const UnplacedRec &u : g->unplaced) g->type_mask |= 1u << u.type;
  // the FP32 screen's boxes, widened so that float rounding of the point, the
  // direction and the slab arithmetic cannot move a ray across them
  g->bbox.assign(6 * g->unplaced.size(), 0.f);
  for (size_t u = 0; u < g->unplaced.size(); ++u) {
    double b[6];
    if (!shape_bbox(g, (int32_t)u, b)) {
      for (int k = 0; k < 3; ++k) {
        g->bbox[6 * u + k] = -3.0e38f;
        g->bbox[6 * u + 3 + k] = 3.0e38f;
      }
      continue;
    }
    double ext = 0.;
    for (int k = 0; k < 6; ++k) ext = std::max(ext, std::fabs(b[k]));
    const double pad = 1e-3 + 1e-5 * ext;
    for (int k = 0; k < 3; ++k) {
      g->bbox[6 * u + k] = std::nextafter((float)(b[k] - pad), -3.0e38f);
      g->bbox[6 * u + 3 + k] = std::nextafter((float)(b[3 + k] + pad), 3.0e38f);
    }
  }
  // each placed volume's box in its mother's frame (corners moved with the full
  // matrix, InverseTransform), for the navigator's float screen
  g->pl_box.assign(6 * g->placed.size(), 0.f);
  for (size_t pv = 0; pv < g->placed.size(); ++pv) {
    float *o = &g->pl_box[6 * pv];
    double b[6];
    if (!shape_bbox(g, g->placed[pv].unplaced, b)) {
      for (int k = 0; k < 3; ++k) {
        o[k] = -3.0e38f;
        o[3 + k] = 3.0e38f;
      }
      continue;
    }
    const RawXform &x = g->raw_xforms[g->placed[pv].raw_xform];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < 8; ++c) {
      const double l[3] = {b[(c & 1) ? 3 : 0], b[(c & 2) ? 4 : 1], b[(c & 4) ? 5 : 2]};
      for (int k = 0; k < 3; ++k) {
        const double m = x.t[k] + l[0] * x.r[3 * k] + l[1] * x.r[3 * k + 1] + l[2] * x.r[3 * k + 2];
        lo[k] = std::min(lo[k], m);
        hi[k] = std::max(hi[k], m);
      }
    }
    double ext = 0.;
    for (int k = 0; k < 3; ++k) ext = std::max(ext, std::max(std::fabs(lo[k]), std::fabs(hi[k])));
    const double pad = 1e-3 + 1e-5 * ext;
    for (int k = 0; k < 3; ++k) {
      o[k] = std::nextafter((float)(lo[k] - pad), -3.0e38f);
      o[3 + k] = std::nextafter((float)(hi[k] + pad), 3.0e38f);
    }
  }
  // ABBoxManager::ComputeABBox (source/ABBoxManager.cpp:128-161): the 8 corners
  // of the shape's Extent, moved to the mother's frame with InverseTransform
  // (base/Transformation3D.h:598-632), their min / max (std::min, std::max, in
  // the reference's corner order) widened by 1e-3; InitABBoxes
  // (:185-262) keeps a float copy for the navigator's hit test
  g->abbox_ok = true;
  g->ab_box_d.assign(6 * g->placed.size(), 0.);
  g->ab_box.assign(6 * g->placed.size(), 0.f);
  for (size_t pv = 0; pv < g->placed.size(); ++pv) {
    const UnplacedRec &u = g->unplaced[g->placed[pv].unplaced];
    double lo[3], hi[3];
    if (!reference_extent(u.type, g->params.data() + u.param_off, lo, hi)) {
      // the reference's VPlacedVolume::Extent asserts for this shape
      // (volumes/PlacedVolume.h:260-263); its volumes get no box and the ABBox
      // navigator refuses the geometry
      g->abbox_ok = false;
      for (int k = 0; k < 6; ++k) g->ab_box_d[6 * pv + k] = std::numeric_limits<double>::quiet_NaN();
      continue;
    }
    const RawXform &x = g->raw_xforms[g->placed[pv].raw_xform];
    const double delta[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    double mn[3], mx[3];
    for (int k = 0; k < 3; ++k) {
      mn[k] = std::numeric_limits<double>::infinity();
      mx[k] = -std::numeric_limits<double>::infinity();
    }
    for (int cx = 0; cx <= 1; ++cx)
      for (int cy = 0; cy <= 1; ++cy)
        for (int cz = 0; cz <= 1; ++cz) {
          const double c[3] = {lo[0] + cx * delta[0], lo[1] + cy * delta[1], lo[2] + cz * delta[2]};
          for (int k = 0; k < 3; ++k) {
            double m = x.t[k];
            m = m + c[0] * x.r[3 * k];
            m = m + c[1] * x.r[3 * k + 1];
            m = m + c[2] * x.r[3 * k + 2];
            mn[k] = vmin(mn[k], m);
            mx[k] = vmax(mx[k], m);
          }
        }
    for (int k = 0; k < 3; ++k) {
      g->ab_box_d[6 * pv + k] = mn[k] - 1E-3;
      g->ab_box_d[6 * pv + 3 + k] = mx[k] + 1E-3;
    }
    for (int k = 0; k < 6; ++k) g->ab_box[6 * pv + k] = (float)g->ab_box_d[6 * pv + k];
  }
  // the navigator reads the boxes of a volume's daughters in daughter order
  g->ab_slot.assign(2 * g->daughters.size(), float4{0.f, 0.f, 0.f, 0.f});
  for (size_t k = 0; k < g->daughters.size(); ++k) {
    const float *b = &g->ab_box[6 * (size_t)g->daughters[k]];
    g->ab_slot[2 * k] = float4{b[0], b[1], b[2], 0.f};
    g->ab_slot[2 * k + 1] = float4{b[3], b[4], b[5], 0.f};
  }
  return VGB_OK;
}

extern "C" {

vgb_status vgb_geometry_close(vgb_geometry *g) {
  VGB_CHECK_OPEN(g);
  vgb_status s0 = prepare_tables(g);
  if (s0 != VGB_OK) return s0;
  // shape records that hold device pointers are fixed up after the pool lands
  cudaError_t e = cudaGetDevice(&g->device);
  if (e != cudaSuccess) return cuda_error(e, "vgb_geometry_close: cudaGetDevice");
  vgb_status s;
  {
    // allocate the pool, let shape records that reference other parts of the
    // pool store device addresses, then copy it
    const size_t n = g->params.empty() ? 2 : g->params.size();
    e = cudaMalloc((void **)&g->dev.params, n * sizeof(double));
    if (e != cudaSuccess) return cuda_error(e, "vgb_geometry_close: cudaMalloc");
    g->dev.bytes += (int64_t)(n * sizeof(double));
    if ((s = finalize_shapes(g)) != VGB_OK) return s;
    if (!g->params.empty()) {
      e = cudaMemcpy(g->dev.params, g->params.data(), g->params.size() * sizeof(double),
                     cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return cuda_error(e, "vgb_geometry_close: cudaMemcpy");
    }
  }
  if ((s = upload(g->unplaced, &g->dev.unplaced, &g->dev.bytes)) != VGB_OK) return s;
  if ((s = upload(g->xforms, &g->dev.xforms, &g->dev.bytes)) != VGB_OK) return s;
  if ((s = upload(g->nav_raw, &g->dev.raw, &g->dev.bytes)) != VGB_OK) return s;
  if ((s = upload(g->placed, &g->dev.placed, &g->dev.bytes)) != VGB_OK) return s;
  if ((s = upload(g->logicals, &g->dev.logicals, &g->dev.bytes)) != VGB_OK) return s;
  if ((s = upload(g->daughters, &g->dev.daughters, &g->dev.bytes)) != VGB_OK) return s;
  {
    const std::vector<uint32_t> zero(1, 0u);
    if ((s = upload(zero, &g->dev.nav_flags, &g->dev.bytes)) != VGB_OK) return s;
  }
  if ((s = upload(g->pl_box, &g->dev.pl_box, &g->dev.bytes)) != VGB_OK) return s;
  if ((s = upload(g->ab_box, &g->dev.ab_box, &g->dev.bytes)) != VGB_OK) return s;
  if ((s = upload(g->ab_slot, &g->dev.ab_slot, &g->dev.bytes)) != VGB_OK) return s;
  g->closed = true;
  return VGB_OK;
}

vgb_status vgb_abbox_compute(const vgb_geometry *g, int32_t placed, double *lower_upper) {
  if (!g || !lower_upper) return set_error(VGB_EINVAL, "vgb_abbox_compute: NULL argument");
  if (placed < 0 || placed >= (int32_t)g->placed.size())
    return set_error(VGB_EINVAL, "vgb_abbox_compute: unknown placed volume %d", placed);
  vgb_geometry *gm = const_cast<vgb_geometry *>(g);
  if (!g->closed) {
    vgb_status s = prepare_tables(gm);
    if (s != VGB_OK) return s;
  }
  const UnplacedRec &u = g->unplaced[g->placed[placed].unplaced];
  double lo[3], hi[3];
  if (!reference_extent(u.type, g->params.data() + u.param_off, lo, hi))
    return set_error(VGB_ENOTSUP, "vgb_abbox_compute: shape type %d has no Extent in the reference",
                     u.type);
  for (int k = 0; k < 6; ++k) lower_upper[k] = g->ab_box_d[6 * (size_t)placed + k];
  return VGB_OK;
}

vgb_status vgb_geometry_max_depth(const vgb_geometry *g, int32_t *depth) {
  VGB_CHECK_G(g);
  if (!depth) return set_error(VGB_EINVAL, "vgb_geometry_max_depth: out pointer is NULL");
  *depth = g->max_depth;
  return VGB_OK;
}

vgb_status vgb_geometry_device_bytes(const vgb_geometry *g, int64_t *bytes) {
  VGB_CHECK_G(g);
  if (!bytes) return set_error(VGB_EINVAL, "vgb_geometry_device_bytes: out pointer is NULL");
  *bytes = g->dev.bytes;
  return VGB_OK;
}

}  // extern "C"

namespace vgb {
vgb_status finalize_shapes(vgb_geometry *g) {
  (void)g;
  return VGB_OK;
}
}  // namespace vgb

