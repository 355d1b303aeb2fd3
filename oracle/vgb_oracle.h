/* vgb_oracle.h -- test infrastructure, NOT product code.
 *
 * A plain-C, scalar restatement of the reference VecGeom algorithms on the
 * geometry hot path (shape Inside/Contains/DistanceToIn/DistanceToOut/
 * SafetyToIn/SafetyToOut, placement transforms, SimpleNavigator steps).  Each
 * function cites the reference file:line it restates.  It exists to check the
 * CUDA library: only tests/, the package smoke check and bench.py's CPU
 * baseline leg load it.  It is compiled with -ffp-contract=off so every
 * a*b+c rounds twice, like the reference Scalar build.
 *
 * Parity is pinned against the reference itself: tests/golden/ holds vectors
 * produced by the reference Scalar backend (oracle/_ref, built from the
 * reference sources) and tests/test_oracle_golden.py checks this restatement
 * against them.
 */
#ifndef VGB_ORACLE_H
#define VGB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* base/Global.h:196-207, :267-302 */
#define OR_kInside 0
#define OR_kSurface 1
#define OR_kOutside 2

enum or_op {
  OR_CONTAINS = 0,
  OR_INSIDE = 1,
  OR_DISTANCE_TO_IN = 2,
  OR_DISTANCE_TO_OUT = 3,
  OR_SAFETY_TO_IN = 4,
  OR_SAFETY_TO_OUT = 5
};

enum or_shape {
  OR_BOX = 1,
  OR_TUBE = 2,
  OR_CONE = 3,
  OR_SPHERE = 4,
  OR_TORUS = 5,
  OR_POLYCONE = 6,
  OR_POLYHEDRON = 7,
  OR_BOOLEAN_SUB = 8,
  OR_TRD = 9
};

/* Placement transform as the reference holds it (base/Transformation3D.h:40-46)
 * plus the two specialisation codes VolumeFactory picks from
 * (source/Transformation3D.cpp:138-162, management/TransformationSpecializations.icc). */
typedef struct {
  double t[3];
  double r[9];
  int trans_code; /* 0 = kIdentity, -1 = kGeneric */
  int rot_code;   /* one of the specialised codes, 0x200 identity, -1 generic */
} or_xform;

/* Build a transform from translation + Euler angles in degrees
 * (source/Transformation3D.cpp:36-44, :93-114). */
void or_xform_euler(or_xform *x, double tx, double ty, double tz, double phi, double theta,
                    double psi);
void or_xform_matrix(or_xform *x, double tx, double ty, double tz, const double *r9);
/* Specialised shapes use the codes; force_generic mimics shapes that always take
 * the generic transform (source/UnplacedPolyhedron.cpp:321-333). */
void or_xform_set_generic(or_xform *x);
void or_transform_point(const or_xform *x, const double m[3], double l[3]);
void or_transform_dir(const or_xform *x, const double m[3], double l[3]);

/* Opaque shape handle; parameters are given as the reference constructors take
 * them (volumes/Unplaced*.h). */
typedef struct or_shape_s or_shape_t;
or_shape_t *or_box(double dx, double dy, double dz);
or_shape_t *or_tube(double rmin, double rmax, double dz, double sphi, double dphi);
void or_shape_free(or_shape_t *s);

/* Batch call over SOA arrays, the VPlacedVolume SOA3D virtuals
 * (volumes/PlacedVolume.h:145-250): Contains/Inside/DistanceToIn/SafetyToIn take
 * mother-frame points and apply the placement; DistanceToOut/SafetyToOut take
 * local points.  out is uint8 (Contains), int32 (Inside) or double. */
int or_batch(const or_shape_t *s, const or_xform *xf, int op, int64_t n, const double *x,
             const double *y, const double *z, const double *dx, const double *dy,
             const double *dz, const double *step_max, void *out);

#ifdef __cplusplus
}
#endif
#endif
