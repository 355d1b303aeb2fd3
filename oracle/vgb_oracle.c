/* vgb_oracle.c -- test infrastructure, NOT product code.
 *
 * Scalar C restatement of the reference VecGeom algorithms (see vgb_oracle.h).
 * Functions follow the reference's operation order so that, compiled with
 * -ffp-contract=off, they round exactly as the reference Scalar build does.
 */
#include "vgb_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* base/Global.h:267-302 */
static const double kPi = 3.14159265358979323846;
static const double kTolerance = 1e-9;
static const double kHalfTolerance = 0.5 * 1e-9;
#define kInfinity (INFINITY)
#define kMinimum (DBL_MIN)

/* ------------------------------------------------------------------------- */
/* Transformation3D                                                          */
/* ------------------------------------------------------------------------- */

/* source/Transformation3D.cpp:138-150 */
static int gen_rot_code(const double *r) {
  int code = 0;
  for (int i = 0; i < 9; ++i) code |= (1 << i) * (fabs(r[i]) > kTolerance);
  if (code == 0x111 && (r[0] == 1. && r[4] == 1. && r[8] == 1.)) code = 0x200;
  return code;
}

/* management/TransformationSpecializations.icc: the rotation codes that get a
 * specialised placed volume; anything else is rotation::kGeneric. */
static int specialised_rot(int code) {
  static const int codes[] = {0x1b1, 0x18e, 0x076, 0x16a, 0x155, 0x0ad, 0x0dc, 0x0e3,
                              0x11b, 0x0a1, 0x10a, 0x046, 0x062, 0x054, 0x111, 0x200};
  for (unsigned i = 0; i < sizeof(codes) / sizeof(codes[0]); ++i)
    if (codes[i] == code) return code;
  return -1;
}

/* source/Transformation3D.cpp:80-89 (SetProperties) and
 * source/UnplacedVolume.cpp:23-24 (codes used to specialise). */
static void set_codes(or_xform *x) {
  int has_t = fabs(x->t[0]) > kTolerance || fabs(x->t[1]) > kTolerance ||
              fabs(x->t[2]) > kTolerance;
  x->trans_code = has_t ? -1 : 0;
  x->rot_code = specialised_rot(gen_rot_code(x->r));
}

void or_xform_euler(or_xform *x, double tx, double ty, double tz, double phi, double theta,
                    double psi) {
  /* source/Transformation3D.cpp:93-114 */
  const double kDegToRad = kPi / 180.;
  const double sinphi = sin(kDegToRad * phi), cosphi = cos(kDegToRad * phi);
  const double sinthe = sin(kDegToRad * theta), costhe = cos(kDegToRad * theta);
  const double sinpsi = sin(kDegToRad * psi), cospsi = cos(kDegToRad * psi);
  x->t[0] = tx;
  x->t[1] = ty;
  x->t[2] = tz;
  x->r[0] = cospsi * cosphi - costhe * sinphi * sinpsi;
  x->r[1] = -sinpsi * cosphi - costhe * sinphi * cospsi;
  x->r[2] = sinthe * sinphi;
  x->r[3] = cospsi * sinphi + costhe * cosphi * sinpsi;
  x->r[4] = -sinpsi * sinphi + costhe * cosphi * cospsi;
  x->r[5] = -sinthe * cosphi;
  x->r[6] = sinpsi * sinthe;
  x->r[7] = cospsi * sinthe;
  x->r[8] = costhe;
  set_codes(x);
}

void or_xform_matrix(or_xform *x, double tx, double ty, double tz, const double *r9) {
  x->t[0] = tx;
  x->t[1] = ty;
  x->t[2] = tz;
  memcpy(x->r, r9, 9 * sizeof(double));
  set_codes(x);
}

void or_xform_set_generic(or_xform *x) {
  x->trans_code = -1;
  x->rot_code = -1;
}

/* base/Transformation3D.h:367-480 (DoRotation<code>): each specialised code
 * keeps only the listed entries, summed in row order; code 0x16A reproduces the
 * reference's third row, master[2]*R[5] + master[2]*R[8]. */
static void do_rotation(const or_xform *x, const double m[3], double l[3]) {
  const double *R = x->r;
  switch (x->rot_code) {
  case 0x1B1: l[0] = m[0]*R[0]; l[1] = m[1]*R[4] + m[2]*R[7]; l[2] = m[1]*R[5] + m[2]*R[8]; return;
  case 0x18E: l[0] = m[1]*R[3]; l[1] = m[0]*R[1] + m[2]*R[7]; l[2] = m[0]*R[2] + m[2]*R[8]; return;
  case 0x076: l[0] = m[2]*R[6]; l[1] = m[0]*R[1] + m[1]*R[4]; l[2] = m[0]*R[2] + m[1]*R[5]; return;
  case 0x16A: l[0] = m[1]*R[3] + m[2]*R[6]; l[1] = m[0]*R[1]; l[2] = m[2]*R[5] + m[2]*R[8]; return;
  case 0x155: l[0] = m[0]*R[0] + m[2]*R[6]; l[1] = m[1]*R[4]; l[2] = m[0]*R[2] + m[2]*R[8]; return;
  case 0x0AD: l[0] = m[0]*R[0] + m[1]*R[3]; l[1] = m[2]*R[7]; l[2] = m[0]*R[2] + m[1]*R[5]; return;
  case 0x0DC: l[0] = m[1]*R[3] + m[2]*R[6]; l[1] = m[1]*R[4] + m[2]*R[7]; l[2] = m[0]*R[2]; return;
  case 0x0E3: l[0] = m[0]*R[0] + m[2]*R[6]; l[1] = m[0]*R[1] + m[2]*R[7]; l[2] = m[1]*R[5]; return;
  case 0x11B: l[0] = m[0]*R[0] + m[1]*R[3]; l[1] = m[0]*R[1] + m[1]*R[4]; l[2] = m[2]*R[8]; return;
  case 0x0A1: l[0] = m[0]*R[0]; l[1] = m[2]*R[7]; l[2] = m[1]*R[5]; return;
  case 0x10A: l[0] = m[1]*R[3]; l[1] = m[0]*R[1]; l[2] = m[2]*R[8]; return;
  case 0x046: l[0] = m[1]*R[3]; l[1] = m[2]*R[7]; l[2] = m[0]*R[2]; return;
  case 0x062: l[0] = m[2]*R[6]; l[1] = m[0]*R[1]; l[2] = m[1]*R[5]; return;
  case 0x054: l[0] = m[2]*R[6]; l[1] = m[1]*R[4]; l[2] = m[0]*R[2]; return;
  case 0x111: l[0] = m[0]*R[0]; l[1] = m[1]*R[4]; l[2] = m[2]*R[8]; return;
  case 0x200: l[0] = m[0]; l[1] = m[1]; l[2] = m[2]; return;
  default: break;
  }
  l[0] = m[0] * R[0];
  l[1] = m[0] * R[1];
  l[2] = m[0] * R[2];
  l[0] += m[1] * R[3];
  l[1] += m[1] * R[4];
  l[2] += m[1] * R[5];
  l[0] += m[2] * R[6];
  l[1] += m[2] * R[7];
  l[2] += m[2] * R[8];
}

/* base/Transformation3D.h:533-562 (Transform<trans_code, rot_code>) */
void or_transform_point(const or_xform *x, const double m[3], double l[3]) {
  const int tid = x->trans_code == 0, rid = x->rot_code == 0x200;
  if (tid && rid) {
    l[0] = m[0]; l[1] = m[1]; l[2] = m[2];
    return;
  }
  if (!tid && rid) {
    l[0] = m[0] - x->t[0]; l[1] = m[1] - x->t[1]; l[2] = m[2] - x->t[2];
    return;
  }
  if (tid && !rid) {
    do_rotation(x, m, l);
    return;
  }
  double tmp[3] = {m[0] - x->t[0], m[1] - x->t[1], m[2] - x->t[2]};
  do_rotation(x, tmp, l);
}

/* base/Transformation3D.h:751-767 (TransformDirection<rot_code>) */
void or_transform_dir(const or_xform *x, const double m[3], double l[3]) {
  if (x->rot_code == 0x200) {
    l[0] = m[0]; l[1] = m[1]; l[2] = m[2];
    return;
  }
  do_rotation(x, m, l);
}

/* ------------------------------------------------------------------------- */
/* Shapes                                                                    */
/* ------------------------------------------------------------------------- */

/* Wedge (volumes/Wedge.h:42-330, source/Wedge.cpp:14-45) */
typedef struct {
  double a1x, a1y, a2x, a2y, n1x, n1y, n2x, n2y, dphi;
} or_wedge;

/* UnplacedTube with its cached values (volumes/UnplacedTube.h:26-60) */
typedef struct {
  double rmin, rmax, z, sphi, dphi, rmin2, rmax2, a1x, a1y, a2x, a2y;
  double tolIrmin2, tolIrmax2, tolIz;
  or_wedge w;
} or_tube_p;

struct or_shape_s {
  int type;
  double p[8];
  or_tube_p tube;
};

or_shape_t *or_box(double dx, double dy, double dz) {
  or_shape_t *s = (or_shape_t *)calloc(1, sizeof(or_shape_t));
  s->type = OR_BOX;
  s->p[0] = dx;
  s->p[1] = dy;
  s->p[2] = dz;
  return s;
}

void or_shape_free(or_shape_t *s) { free(s); }

static void wedge_init(or_wedge *w, double angle, double zero) {
  w->a1x = cos(zero);
  w->a1y = sin(zero);
  w->a2x = cos(zero + angle);
  w->a2y = sin(zero + angle);
  w->n1x = -sin(zero);
  w->n1y = cos(zero);
  w->n2x = sin(zero + angle);
  w->n2y = -cos(zero + angle);
  w->dphi = angle;
}

or_shape_t *or_tube(double rmin, double rmax, double z, double sphi, double dphi) {
  or_shape_t *s = (or_shape_t *)calloc(1, sizeof(or_shape_t));
  or_tube_p *t = &s->tube;
  s->type = OR_TUBE;
  t->rmin = rmin; t->rmax = rmax; t->z = z; t->sphi = sphi; t->dphi = dphi;
  /* volumes/UnplacedTube.h:38-60 calculateCached */
  t->tolIz = z - kTolerance;
  t->rmin2 = rmin * rmin;
  t->rmax2 = rmax * rmax;
  t->tolIrmin2 = (rmin + kTolerance) * (rmin + kTolerance);
  t->tolIrmax2 = (rmax - kTolerance) * (rmax - kTolerance);
  t->a1x = cos(sphi);
  t->a1y = sin(sphi);
  t->a2x = cos(sphi + dphi);
  t->a2y = sin(sphi + dphi);
  wedge_init(&t->w, dphi, sphi);
  return s;
}

/* ---- Box: volumes/kernel/BoxImplementation.h ---------------------------- */

/* :607-666 GenericKernelForContainsAndInside<ForInside=false> */
static int box_contains(const double *d, const double *p) {
  int outside = fabs(p[0]) > d[0];
  outside |= fabs(p[1]) > d[1];
  outside |= fabs(p[2]) > d[2];
  return !outside;
}

/* :607-666 with ForInside=true, :653-666 InsideKernel */
static int box_inside(const double *d, const double *p) {
  int outside = fabs(p[0]) > d[0] + kHalfTolerance;
  int inside = fabs(p[0]) < d[0] - kHalfTolerance;
  outside |= fabs(p[1]) > d[1] + kHalfTolerance;
  inside &= fabs(p[1]) < d[1] - kHalfTolerance;
  outside |= fabs(p[2]) > d[2] + kHalfTolerance;
  inside &= fabs(p[2]) < d[2] - kHalfTolerance;
  int r = OR_kSurface;
  if (outside) r = OR_kOutside;
  if (inside) r = OR_kInside;
  return r;
}

/* :668-746 DistanceToInKernel; `distance` is left untouched on a miss, and the
 * caller starts it at kInfinity (volumes/ShapeImplementationHelper.h:199-220). */
static double box_distance_to_in(const double *d, const double *p, const double *v,
                                 double step_max) {
  double distance = kInfinity;
  double s0 = fabs(p[0]) - d[0], s1 = fabs(p[1]) - d[1], s2 = fabs(p[2]) - d[2];
  if (s0 >= step_max || s1 >= step_max || s2 >= step_max) return distance;
  if (s0 < 0 && s1 < 0 && s2 < 0) return -1.;
  double next, c1, c2;
  next = s0 / fabs(v[0] + kMinimum);
  c1 = p[1] + next * v[1];
  c2 = p[2] + next * v[2];
  if (s0 >= 0. - kHalfTolerance && p[0] * v[0] < 0 && fabs(c1) <= d[1] && fabs(c2) <= d[2])
    return next;
  next = s1 / fabs(v[1] + kMinimum);
  c1 = p[0] + next * v[0];
  c2 = p[2] + next * v[2];
  if (s1 >= 0. - kHalfTolerance && p[1] * v[1] < 0 && fabs(c1) <= d[0] && fabs(c2) <= d[2])
    return next;
  next = s2 / fabs(v[2] + kMinimum);
  c1 = p[0] + next * v[0];
  c2 = p[1] + next * v[1];
  if (s2 >= 0. - kHalfTolerance && p[2] * v[2] < 0 && fabs(c1) <= d[0] && fabs(c2) <= d[1])
    return next;
  return distance;
}

/* :748-799 DistanceToOutKernel */
static double box_distance_to_out(const double *d, const double *p, const double *v) {
  double i0 = 1. / (v[0] + kMinimum), i1 = 1. / (v[1] + kMinimum), i2 = 1. / (v[2] + kMinimum);
  double d0 = (d[0] - p[0]) * i0, d1 = (d[1] - p[1]) * i1, d2 = (d[2] - p[2]) * i2;
  if (v[0] < 0) d0 = (-d[0] - p[0]) * i0;
  if (v[1] < 0) d1 = (-d[1] - p[1]) * i1;
  if (v[2] < 0) d2 = (-d[2] - p[2]) * i2;
  double dist = d0;
  if (d1 < dist) dist = d1;
  if (d2 < dist) dist = d2;
  return dist;
}

/* :801-818 SafetyToInKernel */
static double box_safety_to_in(const double *d, const double *p) {
  double s = -d[0] + fabs(p[0]);
  double sy = -d[1] + fabs(p[1]);
  double sz = -d[2] + fabs(p[2]);
  if (sy > s) s = sy;
  if (sz > s) s = sz;
  return s;
}

/* :820-837 SafetyToOutKernel */
static double box_safety_to_out(const double *d, const double *p) {
  double s = d[0] - fabs(p[0]);
  double sy = d[1] - fabs(p[1]);
  double sz = d[2] - fabs(p[2]);
  if (sy < s) s = sy;
  if (sz < s) s = sz;
  return s;
}

/* ---- Wedge: volumes/Wedge.h ------------------------------------------------ */

static double dmin(double a, double b) { return b < a ? b : a; } /* std::min */
static double dmax(double a, double b) { return a < b ? b : a; } /* std::max */

/* :225-237 IsOnSurfaceGeneric */
static int wedge_on_surface(double ax, double ay, double nx, double ny, double x, double y) {
  if (!(ax * x + ay * y >= 0.)) return 0;
  return fabs(nx * x + ny * y) < kTolerance;
}

/* :190-222 GenericKernelForContainsAndInside */
static void wedge_kernel(const or_wedge *w, int for_inside, double x, double y, int *cin,
                         int *cout) {
  double startCheck = (-x * w->a1y + y * w->a1x);
  double endCheck = (-w->a2x * y + w->a2y * x);
  int out = startCheck < 0.;
  if (w->dphi < kPi)
    out |= endCheck < 0.;
  else
    out &= endCheck < 0.;
  if (for_inside) {
    int on = wedge_on_surface(w->a1x, w->a1y, w->n1x, w->n1y, x, y) ||
             wedge_on_surface(w->a2x, w->a2y, w->n2x, w->n2y, x, y);
    out &= !on;
    *cin = !on && !out;
  }
  *cout = out;
}

/* ---- Tube: volumes/kernel/TubeImplementation.h (UniversalTube, Scalar) ---- */

static int tube_has_rmin(const or_tube_p *t) { return t->rmin > 0; }
static int tube_has_phi(const or_tube_p *t) { return t->dphi < 2 * kPi; }

/* :55-92 PointInCyclicalSector<onSurface=false> */
static int tube_in_sector(const or_tube_p *t, double x, double y) {
  double sc = (-x * t->a1y + y * t->a1x);
  double ec = (-t->a2x * y + t->a2y * x);
  if (t->dphi <= kPi) return (sc >= -kTolerance) && (ec >= -kTolerance);
  return (sc >= -kTolerance) || (ec >= -kTolerance);
}

/* :287-350 GenericKernelForContainsAndInside */
static void tube_kernel(const or_tube_p *t, int for_inside, const double *p, int *cin, int *cout) {
  double absz = fabs(p[2]);
  int out = absz > (for_inside ? t->z + kHalfTolerance : t->z);
  int in = absz < t->z - kHalfTolerance;
  double r2 = p[0] * p[0] + p[1] * p[1];
  out |= r2 > (for_inside ? t->rmax2 + kTolerance * t->rmax : t->rmax2);
  in &= r2 < t->rmax2 - kTolerance * t->rmax;
  if (tube_has_rmin(t)) {
    out |= r2 <= (for_inside ? t->rmin2 - kTolerance * t->rmin : t->rmin2);
    in &= r2 > t->rmin2 + kTolerance * t->rmin;
  }
  if (tube_has_phi(t)) {
    int wi = 0, wo = 0;
    wedge_kernel(&t->w, for_inside, p[0], p[1], &wi, &wo);
    out |= wo;
    in &= wi;
  }
  *cout = out;
  *cin = in;
}

static int tube_contains(const or_tube_p *t, const double *p) {
  int ci, co;
  tube_kernel(t, 0, p, &ci, &co);
  return !co;
}

static int tube_inside(const or_tube_p *t, const double *p) {
  int ci, co;
  tube_kernel(t, 1, p, &ci, &co);
  return ci ? OR_kInside : (co ? OR_kOutside : OR_kSurface);
}

/* :94-137 CircleTrajectoryIntersection<LargestSolution, insectorCheck> */
static void tube_circle(const or_tube_p *t, int largest, int sector_check, double b, double c,
                        const double *p, const double *v, double *dist, int *ok) {
  double delta = b * b - c;
  int dmask = largest ? (delta >= 0.) : (delta > 0.);
  if (!dmask) delta = 0.;
  delta = sqrt(delta);
  if (!largest) delta = -delta;
  *dist = -b + delta;
  if (sector_check) {
    double hz = p[2] + *dist * v[2], hy = p[1] + *dist * v[1], hx = p[0] + *dist * v[0];
    int insector = 1;
    if (tube_has_phi(t)) {
      int wi, wo;
      wedge_kernel(&t->w, 1, hx, hy, &wi, &wo);
      insector = !wo;
    }
    *ok = dmask && (*dist >= 0) && (fabs(hz) <= t->z) && insector;
  } else {
    *ok = dmask;
  }
}

/* :231-267 PhiPlaneTrajectoryIntersection<PositiveDirection=true, insectorCheck> */
static void tube_phi_plane(const or_tube_p *t, int sector_check, double ax, double ay,
                           const double *p, const double *v, double *dist, int *ok) {
  *dist = (ay * p[0] - ax * p[1]) / (v[1] * ax - v[0] * ay);
  double hx = p[0] + *dist * v[0], hy = p[1] + *dist * v[1];
  if (sector_check) {
    double hz = p[2] + *dist * v[2];
    double r2 = hx * hx + hy * hy;
    *ok = fabs(hz) <= t->tolIz && (r2 >= t->tolIrmin2) && (r2 <= t->tolIrmax2) && *dist > 0;
    *ok = *ok && (hx * ax + hy * ay) > 0.;
  } else {
    *ok = (hx * ax + hy * ay) >= 0.;
  }
}

/* :401-554 DistanceToIn (Scalar: early returns taken) */
static double tube_distance_to_in(const or_tube_p *t, const double *p, const double *v) {
  double distance = kInfinity;
  double rsq = p[0] * p[0] + p[1] * p[1];
  double pdx = p[0] * v[0], pdy = p[1] * v[1];
  double abspz = fabs(p[2]);
  double distz = (abspz - t->z) / fabs(v[2]);
  int okz = (p[2] * v[2]) < 0;
  if (abspz > t->z && !okz) return distance;
  if (fabs(p[0]) > t->rmax && pdx >= 0) return distance;
  if (fabs(p[1]) > t->rmax && pdy >= 0) return distance;
  double hx = p[0] + distz * v[0], hy = p[1] + distz * v[1];
  double r2 = hx * hx + hy * hy;
  okz = okz && (distz > 0) && (r2 <= t->tolIrmax2);
  if (tube_has_rmin(t)) okz = okz && (t->tolIrmin2 <= r2);
  if (tube_has_phi(t)) okz = okz && tube_in_sector(t, hx, hy);
  if (okz) return distz;
  double invnsq = 1 / (1 - v[2] * v[2]);
  double rdotn = pdx + pdy;
  double b = invnsq * rdotn;
  double crmax = invnsq * (rsq - t->rmax2);
  double d;
  int ok;
  tube_circle(t, 0, 1, b, crmax, p, v, &d, &ok);
  if (ok) return d;
  if (tube_has_rmin(t)) {
    double crmin = invnsq * (rsq - t->rmin2);
    tube_circle(t, 1, 1, b, crmin, p, v, &d, &ok);
    if (ok) distance = d;
  }
  if (tube_has_phi(t)) {
    tube_phi_plane(t, 1, t->a1x, t->a1y, p, v, &d, &ok);
    if (ok && d < distance) distance = d;
    tube_phi_plane(t, 1, t->a2x, t->a2y, p, v, &d, &ok);
    if (ok && d < distance) distance = d;
  }
  return distance;
}

/* :556-655 DistanceToOut */
static double tube_distance_to_out(const or_tube_p *t, const double *p, const double *v) {
  double distance = kInfinity;
  double sgn = v[2] < 0 ? -1. : 1.;
  double distz = (t->z * sgn - p[2]) / v[2];
  if (distz >= 0) distance = distz;
  double invnsq = 1 / (v[0] * v[0] + v[1] * v[1]);
  double rdotn = v[0] * p[0] + v[1] * p[1];
  double rsq = p[0] * p[0] + p[1] * p[1];
  double b = invnsq * rdotn;
  double d;
  int ok;
  if (tube_has_rmin(t)) {
    tube_circle(t, 0, 0, b, invnsq * (rsq - t->rmin2), p, v, &d, &ok);
    if (ok && d >= 0 && d < distance) distance = d;
  }
  tube_circle(t, 1, 0, b, invnsq * (rsq - t->rmax2), p, v, &d, &ok);
  if (ok && d >= 0 && d < distance) distance = d;
  if (tube_has_phi(t)) {
    tube_phi_plane(t, 0, t->a1x, t->a1y, p, v, &d, &ok);
    if (ok && d > 0 && d < distance) distance = d;
    tube_phi_plane(t, 0, t->a2x, t->a2y, p, v, &d, &ok);
    if (ok && d > 0 && d < distance) distance = d;
  }
  return distance;
}

/* :183-214 PhiPlaneSafety<inside> */
static double tube_phi_safety(const or_tube_p *t, int inside, const double *p) {
  double phi1 = p[0] * t->a1y - p[1] * t->a1x;
  if (inside) phi1 *= -1;
  if (phi1 < 0 || p[0] * t->a1x + p[1] * t->a1y < 0) phi1 = kInfinity;
  double phi2 = p[0] * t->a2y - p[1] * t->a2x;
  if (inside) phi2 *= -1;
  phi2 *= -1;
  if (phi2 < 0 || p[0] * t->a2x + p[1] * t->a2y < 0) phi2 = kInfinity;
  double s = dmin(phi1, phi2);
  if (s == kInfinity) s = -1;
  return s;
}

/* :657-697 SafetyToIn */
static double tube_safety_to_in(const or_tube_p *t, const double *p) {
  double r = sqrt(p[0] * p[0] + p[1] * p[1]);
  double s = dmax(fabs(p[2]) - t->z, r - t->rmax);
  if (tube_has_rmin(t)) s = dmax(s, t->rmin - r);
  if (tube_has_phi(t)) {
    if (tube_in_sector(t, p[0], p[1])) return s;
    s = dmax(s, tube_phi_safety(t, 0, p));
  }
  return s;
}

/* :699-730 SafetyToOut */
static double tube_safety_to_out(const or_tube_p *t, const double *p) {
  double r = sqrt(p[0] * p[0] + p[1] * p[1]);
  double s = dmin(t->z - fabs(p[2]), t->rmax - r);
  if (tube_has_rmin(t)) s = dmin(s, r - t->rmin);
  if (tube_has_phi(t)) {
    double sp = tube_phi_safety(t, 1, p);
    if (sp < 0) sp = kInfinity;
    s = dmin(s, sp);
  }
  return s;
}

/* ------------------------------------------------------------------------- */
/* Dispatch                                                                  */
/* ------------------------------------------------------------------------- */

static int shape_contains(const or_shape_t *s, const double *lp) {
  switch (s->type) {
  case OR_BOX: return box_contains(s->p, lp);
  case OR_TUBE: return tube_contains(&s->tube, lp);
  }
  return 0;
}
static int shape_inside(const or_shape_t *s, const double *lp) {
  switch (s->type) {
  case OR_BOX: return box_inside(s->p, lp);
  case OR_TUBE: return tube_inside(&s->tube, lp);
  }
  return OR_kOutside;
}
static double shape_dti(const or_shape_t *s, const double *lp, const double *lv, double smax) {
  switch (s->type) {
  case OR_BOX: return box_distance_to_in(s->p, lp, lv, smax);
  case OR_TUBE: return tube_distance_to_in(&s->tube, lp, lv);
  }
  return kInfinity;
}
static double shape_dto(const or_shape_t *s, const double *lp, const double *lv, double smax) {
  (void)smax;
  switch (s->type) {
  case OR_BOX: return box_distance_to_out(s->p, lp, lv);
  case OR_TUBE: return tube_distance_to_out(&s->tube, lp, lv);
  }
  return kInfinity;
}
static double shape_sti(const or_shape_t *s, const double *lp) {
  switch (s->type) {
  case OR_BOX: return box_safety_to_in(s->p, lp);
  case OR_TUBE: return tube_safety_to_in(&s->tube, lp);
  }
  return kInfinity;
}
static double shape_sto(const or_shape_t *s, const double *lp) {
  switch (s->type) {
  case OR_BOX: return box_safety_to_out(s->p, lp);
  case OR_TUBE: return tube_safety_to_out(&s->tube, lp);
  }
  return kInfinity;
}

int or_batch(const or_shape_t *s, const or_xform *xf, int op, int64_t n, const double *x,
             const double *y, const double *z, const double *dx, const double *dy,
             const double *dz, const double *step_max, void *out) {
  for (int64_t i = 0; i < n; ++i) {
    double m[3] = {x[i], y[i], z[i]}, lp[3], lv[3];
    switch (op) {
    case OR_CONTAINS:
      or_transform_point(xf, m, lp);
      ((uint8_t *)out)[i] = (uint8_t)shape_contains(s, lp);
      break;
    case OR_INSIDE:
      or_transform_point(xf, m, lp);
      ((int32_t *)out)[i] = shape_inside(s, lp);
      break;
    case OR_DISTANCE_TO_IN: {
      double md[3] = {dx[i], dy[i], dz[i]};
      or_transform_point(xf, m, lp);
      or_transform_dir(xf, md, lv);
      ((double *)out)[i] = shape_dti(s, lp, lv, step_max[i]);
      break;
    }
    case OR_DISTANCE_TO_OUT: {
      double md[3] = {dx[i], dy[i], dz[i]};
      ((double *)out)[i] = shape_dto(s, m, md, step_max[i]);
      break;
    }
    case OR_SAFETY_TO_IN:
      or_transform_point(xf, m, lp);
      ((double *)out)[i] = shape_sti(s, lp);
      break;
    case OR_SAFETY_TO_OUT:
      ((double *)out)[i] = shape_sto(s, m);
      break;
    default:
      return -1;
    }
  }
  return 0;
}
