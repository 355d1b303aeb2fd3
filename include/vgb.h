/* vgb.h -- C ABI of the B200-native VecGeom hot path (libvgb.so).
 *
 * The library replaces, for one NVIDIA B200 (sm_100a), the data-parallel hot
 * path of VecGeom: the VPlacedVolume SOA3D batch virtuals (Inside/Contains,
 * DistanceToIn/DistanceToOut, SafetyToIn/SafetyToOut and their Minimize
 * forms), the CudaManager geometry upload, and the SimpleNavigator step
 * (FindNextBoundaryAndStep, GetSafety) over a device NavStatePool.
 *
 * Conventions kept from the reference (base/Global.h:196-207, :267-302):
 *   - Precision is double; Inside_t is int with kInside=0, kSurface=1, kOutside=2.
 *   - kTolerance = 1e-9 (mm); kInfinity = +inf.
 *   - Contains/Inside/DistanceToIn/SafetyToIn take mother-frame points and apply
 *     the volume's placement; DistanceToOut/SafetyToOut take local points
 *     (volumes/PlacedVolume.h:145-250).
 *   - DistanceToIn returns -1 for a point inside a box and kInfinity on a miss.
 * Every pointer argument may be device memory (the kernels read it in place) or
 * host memory (the call stages it through device buffers in chunks, after the
 * work already queued on the given stream; pinned host memory lets the copies
 * in and out of neighbouring chunks run at the same time).
 * Buffers belong to the caller.  Nothing aborts: every entry point returns a
 * vgb_status and vgb_last_error() describes the last failure on this thread.
 */
#ifndef VGB_H
#define VGB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; the reference instead asserts and aborts
 * (source/backend/cuda/Interface.cpp:20-39). */
typedef enum {
  VGB_OK = 0,
  VGB_EINVAL = 1,    /* bad argument, unknown id, geometry not closed, ... */
  VGB_ENOMEM = 2,    /* device or host allocation failed */
  VGB_ECUDA = 3,     /* a CUDA runtime call failed */
  VGB_ELOOPCAP = 4,  /* a device loop hit its iteration cap (e.g. navigation steps) */
  VGB_ETIMEDOUT = 5, /* a bounded host wait ran out */
  VGB_ENOTSUP = 6,   /* operation not supported for this shape / mode */
  VGB_ENOSPC = 7     /* a fixed-size buffer is too small for the request */
} vgb_status;

/* base/Global.h:196-207 EnumInside */
enum { VGB_kInside = 0, VGB_kSurface = 1, VGB_kOutside = 2 };

/* Arithmetic of the batch kernels.  FP64 reproduces the reference Scalar
 * backend operation by operation; FP32_REFINE does the bulk in float and
 * re-resolves in double where stability needs it. */
typedef enum { VGB_PREC_FP64 = 0, VGB_PREC_FP32_REFINE = 1 } vgb_precision;

/* Operations of the VPlacedVolume SOA3D interface (volumes/PlacedVolume.h). */
typedef enum {
  VGB_OP_CONTAINS = 0,                /* :147  Contains(SOA3D, bool*)                  */
  VGB_OP_INSIDE = 1,                  /* :165  Inside(SOA3D, Inside_t*)                */
  VGB_OP_DISTANCE_TO_IN = 2,          /* :176  DistanceToIn(SOA3D, SOA3D, step*, out*) */
  VGB_OP_DISTANCE_TO_OUT = 3,         /* :212  DistanceToOut(SOA3D, SOA3D, step*, out*)*/
  VGB_OP_SAFETY_TO_IN = 4,            /* :231  SafetyToIn(SOA3D, out*)                 */
  VGB_OP_SAFETY_TO_OUT = 5,           /* :243  SafetyToOut(SOA3D, out*)                */
  VGB_OP_DISTANCE_TO_IN_MINIMIZE = 6, /* :181  DistanceToInMinimize(...)               */
  VGB_OP_SAFETY_TO_IN_MINIMIZE = 7,   /* :237  SafetyToInMinimize(SOA3D, inout*)       */
  VGB_OP_SAFETY_TO_OUT_MINIMIZE = 8,  /* :249  SafetyToOutMinimize(SOA3D, inout*)      */
  VGB_OP_DISTANCE_TO_OUT_NODE = 9,    /* :217  DistanceToOut(..., int* nextnodeindex)  */
  VGB_OP_PLACED_DISTANCE_TO_OUT = 10, /* :207  PlacedDistanceToOut (applies placement) */
  VGB_OP_COUNT = 11
} vgb_op;

/* Shape types (volumes/Unplaced*.h). */
typedef enum {
  VGB_SHAPE_BOX = 1,
  VGB_SHAPE_TUBE = 2,
  VGB_SHAPE_CONE = 3,
  VGB_SHAPE_SPHERE = 4,
  VGB_SHAPE_TORUS = 5,
  VGB_SHAPE_POLYCONE = 6,
  VGB_SHAPE_POLYHEDRON = 7,
  VGB_SHAPE_BOOLEAN = 8,
  VGB_SHAPE_TRD = 9,
  VGB_SHAPE_ORB = 10,
  VGB_SHAPE_PARALLELEPIPED = 11,
  VGB_SHAPE_PARABOLOID = 12,
  VGB_SHAPE_TRAPEZOID = 13
} vgb_shape_type;

/* volumes/UnplacedBooleanVolume.h:10-14 */
enum { VGB_BOOL_UNION = 0, VGB_BOOL_INTERSECTION = 1, VGB_BOOL_SUBTRACTION = 2 };

typedef struct vgb_geometry vgb_geometry;

/* ---------------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------------- */
const char *vgb_last_error(void);
const char *vgb_version(void);
/* Number of kernels this thread launched since the last reset (the count a
 * benchmark reports as its launches). */
int64_t vgb_launch_count(void);
void vgb_launch_count_reset(void);

/* Measurement support, no counterpart in the reference: the FP64 (fp32 = 0) or
 * FP32 (fp32 = 1) FMA throughput of the current GPU.  One launch of independent
 * FMA chains filling every SM, `iters` FMAs per chain, timed with CUDA events
 * on `stream` (synchronises it).  Returns the flops executed (an FMA counts 2)
 * and the launch time; flops / ms is the peak the compute-bound kernels are
 * reported against. */
vgb_status vgb_measure_fma_peak(int32_t fp32, int32_t iters, void *stream, double *flops,
                                float *ms);
/* Measurement support, no counterpart in the reference: how many points the
 * FP32+refine kernels settled with their float selection (certified) and how
 * many they sent to the FP64 path, summed since the last reset (reset != 0
 * zeroes the counts after reading; synchronises the device). */
vgb_status vgb_refine_counts(int64_t *certified, int64_t *fallback, int32_t reset);

/* ---------------------------------------------------------------------------
 * Geometry construction and upload.
 * Replaces the host object graph (Unplaced*, LogicalVolume, Transformation3D,
 * GeoManager) and its CudaManager upload (source/CudaManager.cpp:39-322): the
 * geometry is recorded on the host, then vgb_geometry_close() flattens it into
 * device tables with one copy per table (no per-object constructor kernels).
 * Ids are dense, non-negative ints returned in *id.
 * ------------------------------------------------------------------------- */
vgb_status vgb_geometry_create(vgb_geometry **g);
vgb_status vgb_geometry_destroy(vgb_geometry *g);

/* Unplaced shapes; arguments as the reference constructors take them.       */
/* volumes/UnplacedBox.h:30 */
vgb_status vgb_unplaced_box(vgb_geometry *g, double dx, double dy, double dz, int32_t *id);
/* volumes/UnplacedTube.h:65 (angles in radians) */
vgb_status vgb_unplaced_tube(vgb_geometry *g, double rmin, double rmax, double dz, double sphi,
                             double dphi, int32_t *id);
/* volumes/UnplacedCone.h:108 (angles in radians) */
vgb_status vgb_unplaced_cone(vgb_geometry *g, double rmin1, double rmax1, double rmin2,
                             double rmax2, double dz, double sphi, double dphi, int32_t *id);
/* volumes/UnplacedSphere.h:219 (angles in radians) */
vgb_status vgb_unplaced_sphere(vgb_geometry *g, double rmin, double rmax, double sphi,
                               double dphi, double stheta, double dtheta, int32_t *id);
/* volumes/UnplacedTorus.h:61 (angles in radians) */
vgb_status vgb_unplaced_torus(vgb_geometry *g, double rmin, double rmax, double rtor, double sphi,
                              double dphi, int32_t *id);
/* volumes/UnplacedPolycone.h:82 (angles in radians) */
vgb_status vgb_unplaced_polycone(vgb_geometry *g, double sphi, double dphi, int32_t nz,
                                 const double *rmin, const double *rmax, const double *z,
                                 int32_t *id);
/* volumes/UnplacedPolyhedron.h:169 (phi in degrees, as the reference) */
vgb_status vgb_unplaced_polyhedron(vgb_geometry *g, double phi_start_deg, double phi_delta_deg,
                                   int32_t sides, int32_t nz, const double *z,
                                   const double *rmin, const double *rmax, int32_t *id);
/* volumes/UnplacedTrd.h:73 */
vgb_status vgb_unplaced_trd(vgb_geometry *g, double dx1, double dx2, double dy1, double dy2,
                            double dz, int32_t *id);
/* volumes/UnplacedOrb.h:45 */
vgb_status vgb_unplaced_orb(vgb_geometry *g, double r, int32_t *id);
/* volumes/UnplacedParallelepiped.h:34 (half-lengths; alpha, theta, phi in degrees) */
vgb_status vgb_unplaced_parallelepiped(vgb_geometry *g, double x, double y, double z,
                                       double alpha_deg, double theta_deg, double phi_deg,
                                       int32_t *id);
/* UnplacedParaboloid(rlo, rhi, dz), source/UnplacedParaboloid.cpp:45-67 */
vgb_status vgb_unplaced_paraboloid(vgb_geometry *g, double rlo, double rhi, double dz,
                                   int32_t *id);
/* volumes/UnplacedTrapezoid.h:93-95, UnplacedTrapezoid(pDz, pTheta, pPhi, pDy1,
   pDx1, pDx2, pTanAlpha1, pDy2, pDx3, pDx4, pTanAlpha2); theta, phi in radians */
vgb_status vgb_unplaced_trapezoid(vgb_geometry *g, double dz, double theta, double phi,
                                  double dy1, double dx1, double dx2, double tan_alpha1,
                                  double dy2, double dx3, double dx4, double tan_alpha2,
                                  int32_t *id);
/* volumes/UnplacedTrapezoid.h:103, UnplacedTrapezoid(TrapCorners_t): corners[24] =
   8 corners (x, y, z), 0-3 at z = -dz, 4-7 at z = +dz, in the reference's order */
vgb_status vgb_unplaced_trapezoid_corners(vgb_geometry *g, const double *corners,
                                          int32_t *id);
/* volumes/UnplacedBooleanVolume.h:46 (left/right are placed-volume ids) */
vgb_status vgb_unplaced_boolean(vgb_geometry *g, int32_t op, int32_t left_placed,
                                int32_t right_placed, int32_t *id);

/* Transformation3D(tx,ty,tz, phi,theta,psi) with Euler angles in degrees
 * (source/Transformation3D.cpp:36-44, :93-114). */
vgb_status vgb_transformation(vgb_geometry *g, double tx, double ty, double tz, double phi,
                              double theta, double psi, int32_t *id);
/* Transformation3D(tx,ty,tz, r0..r8) (source/Transformation3D.cpp:46-55). */
vgb_status vgb_transformation_matrix(vgb_geometry *g, double tx, double ty, double tz,
                                     const double *r9, int32_t *id);

/* LogicalVolume(label, unplaced) (volumes/LogicalVolume.h:66). */
vgb_status vgb_logical_volume(vgb_geometry *g, const char *label, int32_t unplaced,
                              int32_t *id);
/* LogicalVolume::Place(transformation) (source/LogicalVolume.cpp:60-64). */
vgb_status vgb_place(vgb_geometry *g, int32_t logical, int32_t transformation, int32_t *placed);
/* LogicalVolume::PlaceDaughter(volume, transformation) (source/LogicalVolume.cpp:80-97);
 * daughter order is insertion order. */
vgb_status vgb_place_daughter(vgb_geometry *g, int32_t mother_logical, int32_t daughter_logical,
                              int32_t transformation, int32_t *placed);
/* GeoManager::SetWorld (management/GeoManager.h:164). */
vgb_status vgb_set_world(vgb_geometry *g, int32_t placed);
/* GeoManager::CloseGeometry + CudaManager::LoadGeometry/Synchronize: computes
 * the maximum depth and uploads all tables to the current device. */
vgb_status vgb_geometry_close(vgb_geometry *g);
/* GeoManager::getMaxDepth (management/GeoManager.h:191). */
vgb_status vgb_geometry_max_depth(const vgb_geometry *g, int32_t *depth);
/* Bytes the geometry occupies on the device. */
vgb_status vgb_geometry_device_bytes(const vgb_geometry *g, int64_t *bytes);

/* ---------------------------------------------------------------------------
 * Ingestion and export formats.
 *
 * Flat image: the recorded object graph (shape records with their constructor
 * arguments, transformations, logical volumes and labels, placements, world)
 * in one checksummed little-endian blob.  The reference has no such image (it
 * rebuilds its object graph from ROOT, Geant4 or generated C++ source,
 * source/RootGeoManager.cpp:48-169, source/CppExporter.cpp); it is the
 * ingestion path of this library.  Serialising writes *len bytes into buf when
 * cap suffices (buf NULL: only *len); VGB_ENOSPC when cap is too small.
 * Deserialising creates a new, open geometry with the same ids; close it as
 * usual.  A malformed or corrupted image is VGB_EINVAL. */
vgb_status vgb_geometry_serialize(const vgb_geometry *g, void *buf, size_t cap, size_t *len);
vgb_status vgb_geometry_deserialize(const void *buf, size_t len, vgb_geometry **g);
vgb_status vgb_geometry_save(const vgb_geometry *g, const char *path);
vgb_status vgb_geometry_load(const char *path, vgb_geometry **g);
/* GeomCppExporter::DumpGeometry (management/CppExporter.h, source/CppExporter.cpp):
 * C++ source of `VPlacedVolume const * generateDetector()` that rebuilds the
 * geometry with VecGeom's API; numbers with 17 significant digits; a comment
 * lists this geometry's placed ids in the order the function creates the
 * placements.  Buffer convention as vgb_geometry_serialize (no terminating NUL). */
vgb_status vgb_geometry_export_cpp(const vgb_geometry *g, char *buf, size_t cap, size_t *len);

/* ---------------------------------------------------------------------------
 * Batched shape operations (the VPlacedVolume SOA3D virtuals).
 *
 * One call runs one operation over n points for one placed volume.
 *   x,y,z        positions (SOA3D x(), y(), z())
 *   dx,dy,dz     directions (unit vectors), DistanceTo* only
 *   step_max     per-point step limit, DistanceTo* only
 *   out          uint8 (Contains), int32 (Inside) or double; for the Minimize
 *                forms it is the in/out distance or safety array
 *   aux          int32: DistanceToInMinimize's next-daughter id list (in/out)
 *                and DistanceToOut's node index (-1 leaves, -2 stays)
 *   daughter     the daughter index written by DistanceToInMinimize
 *   stream       cudaStream_t (NULL = legacy default stream)
 * The call is asynchronous for device pointers; with host pointers it returns
 * once the results are back in host memory.
 * ------------------------------------------------------------------------- */
vgb_status vgb_batch(const vgb_geometry *g, int32_t placed, int32_t op, int64_t n,
                     const double *x, const double *y, const double *z, const double *dx,
                     const double *dy, const double *dz, const double *step_max, void *out,
                     int32_t *aux, int32_t daughter, int32_t precision, void *stream);

/* Per-operation forms with the reference's argument order. */
vgb_status vgb_Contains(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                        const double *y, const double *z, uint8_t *out, void *stream);
vgb_status vgb_Inside(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                      const double *y, const double *z, int32_t *out, void *stream);
vgb_status vgb_DistanceToIn(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                            const double *y, const double *z, const double *dx,
                            const double *dy, const double *dz, const double *step_max,
                            double *out, void *stream);
vgb_status vgb_DistanceToOut(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                             const double *y, const double *z, const double *dx,
                             const double *dy, const double *dz, const double *step_max,
                             double *out, void *stream);
vgb_status vgb_SafetyToIn(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                          const double *y, const double *z, double *out, void *stream);
vgb_status vgb_SafetyToOut(const vgb_geometry *g, int32_t placed, int64_t n, const double *x,
                           const double *y, const double *z, double *out, void *stream);

/* Several operations over the same points in one pass (one read of x,y,z and
 * the directions).  ops is a bit mask of (1 << vgb_op) over CONTAINS, INSIDE,
 * DISTANCE_TO_IN, DISTANCE_TO_OUT, SAFETY_TO_IN, SAFETY_TO_OUT; outs[op] is the
 * output of each requested op.  With VGB_FUSED_DTO_INSIDE_ONLY set in flags,
 * DistanceToOut is evaluated only for points Contains() accepts; the others
 * get kInfinity.  VGB_FUSED_LOCAL_INSIDE_ONLY does the same for DistanceToOut
 * and SafetyToOut (the local-frame ops, meaningful for points inside), so one
 * call covers what a caller would otherwise run as two (all points, then the
 * inside subset).  Buffers are all device or all host memory; host buffers
 * cross to the device once per chunk for all the requested ops (staged as in
 * vgb_batch), and the call returns with the outputs written. */
enum { VGB_FUSED_DTO_INSIDE_ONLY = 1, VGB_FUSED_LOCAL_INSIDE_ONLY = 2 };
vgb_status vgb_batch_fused(const vgb_geometry *g, int32_t placed, uint32_t ops, int64_t n,
                           const double *x, const double *y, const double *z, const double *dx,
                           const double *dy, const double *dz, const double *step_max,
                           void *const *outs, uint32_t flags, int32_t precision, void *stream);

/* ---------------------------------------------------------------------------
 * Baskets: many placed volumes (of any shapes) and their point batches in one
 * persistent launch.  The reference runs one SOA3D virtual call per volume and
 * batch (volumes/PlacedVolume.h:145-250, the basket loops of
 * SimpleNavigator.h:599-743); a plan packs all baskets into tiles of points that
 * the CTAs of one launch take in turn, each tile belonging to one basket (one
 * shape), so the shape dispatch is uniform per tile.
 *
 * The points of all baskets are concatenated: basket b owns [offset, offset +
 * count) of x..dz, step_max and of every output array.  Each basket evaluates
 * the ops of the plan's mask with vgb_batch_fused's semantics (outs[op]).
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t placed; /* placed volume of this basket */
  int32_t pad;
  int64_t offset; /* first point of the basket in the concatenated arrays */
  int64_t count;  /* number of points */
} vgb_basket;

typedef struct vgb_basket_plan vgb_basket_plan;

/* Builds the tile table of nb baskets (host array) for the op mask `ops` (bits
 * 1 << vgb_op over CONTAINS, INSIDE, DISTANCE_TO_IN, DISTANCE_TO_OUT,
 * SAFETY_TO_IN, SAFETY_TO_OUT).  block = threads per CTA (256 or 512) and
 * tile = points per tile (a multiple of block); 0 picks the defaults (256,
 * 1024) until vgb_basket_tune chooses.  A launch runs one kernel per shape kind
 * present (booleans per component pair), as concurrent branches of the
 * caller's stream. */
vgb_status vgb_basket_plan_create(const vgb_geometry *g, const vgb_basket *baskets, int32_t nb,
                                  uint32_t ops, int32_t block, int32_t tile,
                                  vgb_basket_plan **plan);
vgb_status vgb_basket_plan_destroy(vgb_basket_plan *plan);
/* total points and tiles of the plan, and its current launch shape */
vgb_status vgb_basket_plan_info(const vgb_basket_plan *plan, int64_t *points, int64_t *tiles,
                                int32_t *block, int32_t *tile);

/* One persistent launch over every basket of the plan (device pointers). */
vgb_status vgb_basket_run(vgb_basket_plan *plan, const double *x, const double *y,
                          const double *z, const double *dx, const double *dy, const double *dz,
                          const double *step_max, void *const *outs, uint32_t flags,
                          void *stream);

/* Autotuner: times every (block, tile) candidate on these inputs (reps
 * launches each, CUDA events on `stream`), keeps the fastest in the plan and
 * returns it with its time per launch.  The outputs are overwritten. */
vgb_status vgb_basket_tune(vgb_basket_plan *plan, const double *x, const double *y,
                           const double *z, const double *dx, const double *dy, const double *dz,
                           const double *step_max, void *const *outs, uint32_t flags, int32_t reps,
                           void *stream, int32_t *best_block, int32_t *best_tile,
                           float *best_ms);

/* Captures vgb_basket_run with these pointers into a CUDA graph held by the
 * plan; vgb_basket_graph_launch replays it on `stream`. */
vgb_status vgb_basket_graph_capture(vgb_basket_plan *plan, const double *x, const double *y,
                                    const double *z, const double *dx, const double *dy,
                                    const double *dz, const double *step_max, void *const *outs,
                                    uint32_t flags);
vgb_status vgb_basket_graph_launch(vgb_basket_plan *plan, void *stream);

/* The basket launch of vgb_basket_run for callers that cannot allocate device
 * memory: a framework that has handed the GPU's memory to its own pool at
 * start-up, or an online event loop where a cudaMalloc could stall or fail in
 * the middle of a run.  This entry point calls no cudaMalloc/cudaFree and no
 * allocating routine, on the device or the host.  The basket tables live in a
 * fixed array compiled into the library (one per GPU, about 450 KB, held until the
 * process exits), so it takes at most VGB_NOALLOC_MAX_BASKETS baskets and
 * returns VGB_ENOSPC beyond that.  It has no counterpart in the reference.
 *
 *  - baskets is a host array, pageable or pinned; the call copies it into a
 *    host array of its own before the device copy starts, so the caller may
 *    refill it as soon as the call returns.  Launch shape: 256 threads per CTA,
 *    1024 points per tile.
 *  - The first call on each device looks up the array's device address; make
 *    that first call from a thread whose current device is the geometry's,
 *    and before any stream capture begins.
 *  - Every call reuses the same array and leaves its tables in it; nothing in
 *    it needs to start at zero, since each call writes every entry it reads.
 *    Calls whose work overlaps on the GPU (two streams, or two threads) race
 *    on the array: issue them on one stream, or wait for one before the next. */
enum { VGB_NOALLOC_MAX_BASKETS = 8192 };
vgb_status vgb_basket_run_noalloc(const vgb_geometry *g, const vgb_basket *baskets, int32_t nb,
                                  uint32_t ops, const double *x, const double *y,
                                  const double *z, const double *dx, const double *dy,
                                  const double *dz, const double *step_max, void *const *outs,
                                  uint32_t flags, void *stream);

/* ---------------------------------------------------------------------------
 * Navigation (navigation/SimpleNavigator.h, NavigationState.h, NavStatePool.h).
 *
 * A pool holds n NavigationStates in device memory in the reference's field
 * layout (navigation/NavigationState.h:45-66): int32 level at byte 0, onBoundary
 * at byte 4, the {selfAlloc:1, N:31} word at byte 8 and N = max_depth + 1 path
 * slots of 8 bytes from byte 16; the stride is 16 + 8 N bytes (56 at depth 4).
 * A slot holds the placed-volume id (int64, -1 when empty) where the reference
 * holds a VPlacedVolume pointer, which is the translation the reference makes
 * when it copies a pool to the GPU (NavStatePool::CopyToGpu,
 * navigation/NavStatePool.h:110-152).
 *
 * The navigation calls take device pointers and are asynchronous on `stream`.
 * A track whose path would exceed 16 levels is not stepped; such tracks raise
 * VGB_NAV_ERR_DEPTH in the geometry's navigation flags, which
 * vgb_nav_error_flags() returns (after synchronising the device) and clears.
 * ------------------------------------------------------------------------- */
typedef struct vgb_navpool vgb_navpool;
enum { VGB_NAV_ERR_DEPTH = 1 };

/* NavStatePool(size, depth) (navigation/NavStatePool.h:46-60) for a closed geometry */
vgb_status vgb_navpool_create(const vgb_geometry *g, int64_t n, vgb_navpool **pool);
vgb_status vgb_navpool_destroy(vgb_navpool *pool);
/* device address, state stride in bytes and capacity */
vgb_status vgb_navpool_info(const vgb_navpool *pool, void **device, int64_t *stride, int64_t *n);
/* NavStatePool::CopyToGpu / CopyFromGpu (:110-152): n states from / to a host
 * buffer in the same layout (slots hold placed-volume ids) */
vgb_status vgb_navpool_upload(vgb_navpool *pool, const void *host, int64_t n, void *stream);
vgb_status vgb_navpool_download(const vgb_navpool *pool, void *host, int64_t n, void *stream);

/* SimpleNavigator::LocatePoint(world, point, state, true)
 * (navigation/SimpleNavigator.h:204-240) for n global points into states[0..n) */
vgb_status vgb_nav_locate(const vgb_geometry *g, int64_t n, const double *x, const double *y,
                          const double *z, vgb_navpool *states, void *stream);

/* SimpleNavigator::FindNextBoundaryAndStep (:340-470) for n tracks: global
 * points and directions, current states `cur`, proposed steps pstep[i]; writes
 * the new states into `next` and the steps into step[i].  If safety is not
 * NULL, safety[i] receives SimpleNavigator::GetSafety (:572-596) at the point
 * in the current state.  cur and next must be different pools.
 * precision VGB_PREC_FP32_REFINE puts a float screen in front of the daughter
 * loops (a daughter whose widened box the ray misses or enters beyond the
 * running best step is not evaluated, nor a box daughter whose float safety is
 * certainly above the running minimum; the culling of ABBoxNavigator,
 * navigation/ABBoxNavigator.h:148-452); results equal the FP64 form's. */
vgb_status vgb_nav_find_next_boundary_and_step(const vgb_geometry *g, int64_t n, const double *x,
                                               const double *y, const double *z,
                                               const double *dx, const double *dy,
                                               const double *dz, const vgb_navpool *cur,
                                               vgb_navpool *next, const double *pstep,
                                               double *step, double *safety, int32_t precision,
                                               void *stream);

/* The basket form of SimpleNavigator::FindNextBoundaryAndStep
 * (navigation/SimpleNavigator.h:637-743) with GetSafeties (:599-632): per track
 * the current volume's DistanceToOut with its node index, every daughter's
 * DistanceToInMinimize (volumes/ShapeImplementationHelper.h:637-658) and the
 * relocation pushed 1e-9 past the boundary.  distance[i] is the step (pstep[i]
 * when the geometry is further), nextnode[i] the reference's next-node
 * workspace entry (daughter position, -1 leaving, -2 staying; may be NULL) and
 * safety[i] GetSafeties' value (may be NULL).  The reference takes the
 * volume of a basket's first track for all of its tracks; here every track
 * uses its own state, which is the same for a basket of one volume. */
vgb_status vgb_nav_find_next_boundary_and_step_basket(
    const vgb_geometry *g, int64_t n, const double *x, const double *y, const double *z,
    const double *dx, const double *dy, const double *dz, const vgb_navpool *cur,
    vgb_navpool *next, const double *pstep, double *distance, double *safety, int32_t *nextnode,
    void *stream);

/* Transport of n straight tracks from their start points to the world exit:
 * LocatePoint from the world, then per step GetSafety, FindNextBoundaryAndStep
 * and point += direction * step, until the state is outside or max_steps steps
 * were taken.  Per track i and step k < nsteps[i] (records at i * max_steps + k):
 * next_ids = placed id of the new state's Top() (-1 once outside), steps, and
 * safeties (at the step's start point).  next_ids, steps and safeties may be
 * NULL; nsteps may not.  A client loop over the reference's calls (which
 * source/benchmarking/NavigationBenchmarker.cpp:48-110 times one step at a time);
 * it has no counterpart of its own in the reference. */
vgb_status vgb_nav_trace(const vgb_geometry *g, int64_t n, const double *x, const double *y,
                         const double *z, const double *dx, const double *dy, const double *dz,
                         double pstep, int32_t max_steps, int32_t *next_ids, double *steps,
                         double *safeties, int32_t *nsteps, int32_t precision, void *stream);

/* ABBoxNavigator::FindNextBoundaryAndStep (navigation/ABBoxNavigator.h:200-420)
 * for n tracks; arguments and results as vgb_nav_find_next_boundary_and_step.
 * The daughters are culled by ABBoxManager's aligned boxes (float ray-box
 * test, source/ABBoxManager.cpp:88-126) and visited in the order of their box
 * distance, and the new state follows ABBoxNavigator's own decisions (an
 * infinite step beyond pstep returns pstep; leaving pops while the relocated
 * path ends in the volume left).  safety[i] receives ABBoxNavigator::GetSafety
 * (:424-452).  Equal box distances are visited in daughter order (libstdc++'s
 * std::sort keeps that order for up to 16 hits). */
vgb_status vgb_abbox_nav_find_next_boundary_and_step(const vgb_geometry *g, int64_t n,
                                                     const double *x, const double *y,
                                                     const double *z, const double *dx,
                                                     const double *dy, const double *dz,
                                                     const vgb_navpool *cur, vgb_navpool *next,
                                                     const double *pstep, double *step,
                                                     double *safety, void *stream);

/* vgb_nav_trace with ABBoxNavigator's step (and its GetSafety). */
vgb_status vgb_abbox_nav_trace(const vgb_geometry *g, int64_t n, const double *x, const double *y,
                               const double *z, const double *dx, const double *dy,
                               const double *dz, double pstep, int32_t max_steps,
                               int32_t *next_ids, double *steps, double *safeties,
                               int32_t *nsteps, void *stream);

/* ABBoxManager::ComputeABBox (source/ABBoxManager.cpp:128-161) of a placed
 * volume: lower xyz, upper xyz of its aligned box in the mother's frame, as
 * doubles (the navigator uses them rounded to float).  Works on an open
 * geometry too (host tables only). */
vgb_status vgb_abbox_compute(const vgb_geometry *g, int32_t placed, double *lower_upper);

/* Navigation error flags (VGB_NAV_ERR_*) raised since the last call; clears them. */
vgb_status vgb_nav_error_flags(const vgb_geometry *g, uint32_t *flags);

/* ---------------------------------------------------------------------------
 * Navigation server: continuous batching of track baskets (no counterpart in
 * the reference, whose navigators step one caller-given basket at a time,
 * navigation/SimpleNavigator.h:599-743).
 *
 * Requests (baskets of straight tracks, host arrays) are queued by
 * vgb_server_submit.  Each vgb_server_step is one iteration: it admits queued
 * requests in arrival order while the device track slots (allocated once, at
 * create, from free HBM) can hold them, advances every live track of every
 * admitted request by up to steps_per_launch navigation steps in one launch,
 * and retires the requests whose tracks all finished: their results move to
 * host memory and their slots are free for the next admission.  A track
 * finishes when its state leaves the world or after max_steps steps.  Per track
 * the server keeps what vgb_nav_trace would produce: the step count, the final
 * point and a 64-bit FNV-1a hash of its sequence of (next placed id, step,
 * safety) records (int32, double, double, little-endian), so a request's
 * results do not depend on what else was in flight.
 * ------------------------------------------------------------------------- */
typedef struct vgb_server vgb_server;

/* max_tracks = 0 sizes the slots to a quarter of the free device memory
 * (at most 2^22 tracks).  Fails with VGB_ENOMEM when the slots do not fit. */
vgb_status vgb_server_create(const vgb_geometry *g, int64_t max_tracks, int32_t steps_per_launch,
                             int32_t max_steps, double pstep, int32_t precision,
                             vgb_server **server);
vgb_status vgb_server_destroy(vgb_server *server);
/* slot capacity (tracks) and device bytes held */
vgb_status vgb_server_info(const vgb_server *server, int64_t *max_tracks, int64_t *device_bytes);
/* Queues a request of n tracks (host arrays, copied); VGB_ENOSPC if n exceeds
 * the slot capacity.  Request ids increase from 0. */
vgb_status vgb_server_submit(vgb_server *server, int64_t n, const double *x, const double *y,
                             const double *z, const double *dx, const double *dy,
                             const double *dz, int64_t *request_id);
/* One iteration (admit, launch, retire); synchronous.  Writes up to
 * max_completed finished request ids; *live = tracks still in flight,
 * *queued = requests waiting for admission. */
vgb_status vgb_server_step(vgb_server *server, int64_t *completed, int32_t max_completed,
                           int32_t *ncompleted, int64_t *live, int64_t *queued);
/* Results of a finished request (arrays of its n tracks; any may be NULL);
 * the request is then forgotten. */
vgb_status vgb_server_result(vgb_server *server, int64_t request_id, int32_t *nsteps, double *x,
                             double *y, double *z, uint64_t *hash);

#ifdef __cplusplus
}
#endif
#endif /* VGB_H */
