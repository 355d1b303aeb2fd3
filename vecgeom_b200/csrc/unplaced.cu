// unplaced.cu -- the unplaced-shape constructors of the C ABI.
//
// Each computes the shape's cached values with the reference constructor's
// formulas (host code, -ffp-contract=off, glibc cos/sin as in the reference),
// so the device kernels see bit-identical constants.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "geometry.h"
#include "shapes.cuh"

using namespace vgb;

namespace vgb {

// Wedge::Wedge(angle, zeroangle) (source/Wedge.cpp:14-45)
WedgeP make_wedge(double dphi, double sphi) {
  WedgeP w;
  std::memset(&w, 0, sizeof(w));
  w.a1x = std::cos(sphi);
  w.a1y = std::sin(sphi);
  w.a2x = std::cos(sphi + dphi);
  w.a2y = std::sin(sphi + dphi);
  w.n1x = -std::sin(sphi);
  w.n1y = std::cos(sphi);
  w.n2x = std::sin(sphi + dphi);
  w.n2y = -std::cos(sphi + dphi);
  w.dphi = dphi;
  w.lt_pi = dphi < kPi;
  return w;
}

// UnplacedTube::calculateCached (volumes/UnplacedTube.h:38-60)
TubeP make_tube(double rmin, double rmax, double z, double sphi, double dphi) {
  TubeP t;
  std::memset(&t, 0, sizeof(t));
  t.rmin = rmin;
  t.rmax = rmax;
  t.z = z;
  t.sphi = sphi;
  t.dphi = dphi;
  t.tolIz = z - kTolerance;
  t.tolOz = z + kTolerance;
  t.rmin2 = rmin * rmin;
  t.rmax2 = rmax * rmax;
  const double tolOrmin = rmin - kTolerance, tolIrmin = rmin + kTolerance;
  t.tolOrmin2 = tolOrmin * tolOrmin;
  t.tolIrmin2 = tolIrmin * tolIrmin;
  const double tolOrmax = rmax + kTolerance, tolIrmax = rmax - kTolerance;
  t.tolOrmax2 = tolOrmax * tolOrmax;
  t.tolIrmax2 = tolIrmax * tolIrmax;
  t.a1x = std::cos(sphi);
  t.a1y = std::sin(sphi);
  t.a2x = std::cos(sphi + dphi);
  t.a2y = std::sin(sphi + dphi);
  t.wedge = make_wedge(dphi, sphi);
  // volumes/kernel/shapetypes/TubeTypes.h:104-158 (UniversalTube: run-time checks)
  t.has_rmin = rmin > 0;
  t.has_phi = dphi < 2 * M_PI;
  t.le_pi = dphi <= M_PI;
  return t;
}

// UnplacedCone constructor (volumes/UnplacedCone.h:108-170)
ConeP make_cone(double rmin1, double rmax1, double rmin2, double rmax2, double dz, double sphi,
                double dphi) {
  ConeP c;
  std::memset(&c, 0, sizeof(c));
  c.rmin1 = rmin1;
  c.rmax1 = rmax1;
  c.rmin2 = rmin2;
  c.rmax2 = rmax2;
  c.dz = dz;
  c.sphi = sphi;
  c.dphi = dphi;
  const double hDPhi = 0.5 * dphi;
  const double cPhi = sphi + hDPhi;
  const double ePhi = sphi + dphi;
  c.sinCPhi = std::sin(cPhi);
  c.cosCPhi = std::cos(cPhi);
  c.cosHDPhi = std::cos(hDPhi);
  c.cosHDPhiIT = std::cos(hDPhi - 0.5 * kAngTolerance);
  c.cosHDPhiOT = std::cos(hDPhi + 0.5 * kAngTolerance);
  c.sinSPhi = std::sin(sphi);
  c.cosSPhi = std::cos(sphi);
  c.sinEPhi = std::sin(ePhi);
  c.cosEPhi = std::cos(ePhi);
  c.tanRMin = (rmin2 - rmin1) * 0.5 / dz;
  c.secRMin = std::sqrt(1.0 + c.tanRMin * c.tanRMin);
  c.invSecRMin = 1. / c.secRMin;
  c.tanRMax = (rmax2 - rmax1) * 0.5 / dz;
  c.secRMax = std::sqrt(1.0 + c.tanRMax * c.tanRMax);
  c.invSecRMax = 1. / c.secRMax;
  c.innerSlope = -(rmin1 - rmin2) / (2. * dz);
  c.outerSlope = -(rmax1 - rmax2) / (2. * dz);
  c.innerOffset = rmin2 - c.innerSlope * dz;
  c.outerOffset = rmax2 - c.outerSlope * dz;
  c.wedge = make_wedge(dphi, sphi);
  c.full_phi = dphi == kTwoPi;
  // volumes/kernel/shapetypes/ConeTypes.h:107-162 (UniversalCone: run-time checks)
  c.has_rmin = rmin1 > 0 || rmin2 > 0;
  c.has_phi = dphi < 2. * M_PI;
  return c;
}

// UnplacedSphere constructor (source/UnplacedSphere.cpp:24-95 with
// CheckPhiAngles/CheckThetaAngles, volumes/UnplacedSphere.h:56-210); USphere
// (USolids/src/USphere.cc:30-55) computes the same values.
SphereP make_sphere(double rmin, double rmax, double sphi, double dphi, double stheta,
                    double dtheta) {
  SphereP s;
  std::memset(&s, 0, sizeof(s));
  const double kAngTol = 1e-9, kRadTol = 1e-9, fEpsilon = 2.e-11;
  s.rmin = rmin;
  s.rmax = rmax;
  s.rminTolerance = (rmin != 0) ? std::max(kRadTol, fEpsilon * rmin) : 0;
  s.mkTolerance = std::max(kRadTol, fEpsilon * rmax);
  bool fullPhi = true, fullTheta = true, full = true;
  // CheckPhiAngles -> CheckDPhiAngle, CheckSPhiAngle
  double fSPhi = 0, fDPhi = 0;
  if (dphi >= 2 * kPi - kAngTol * 0.5) {
    fDPhi = 2 * kPi;
    fSPhi = 0;
  } else {
    fullPhi = false;
    if (dphi > 0) fDPhi = dphi;
  }
  if (!fullPhi) {
    if (sphi < 0)
      fSPhi = 2 * kPi - std::fmod(std::fabs(sphi), 2 * kPi);
    else
      fSPhi = std::fmod(sphi, 2 * kPi);
    if (fSPhi + fDPhi > 2 * kPi) fSPhi -= 2 * kPi;
  }
  full = fullPhi && fullTheta;
  s.sphi = fSPhi;
  s.dphi = fDPhi;
  s.hDPhi = 0.5 * fDPhi;
  s.cPhi = fSPhi + s.hDPhi;
  s.ePhi = fSPhi + fDPhi;
  s.sinCPhi = std::sin(s.cPhi);
  s.cosCPhi = std::cos(s.cPhi);
  s.cosHDPhiIT = std::cos(s.hDPhi - 0.5 * kAngTol);
  s.cosHDPhiOT = std::cos(s.hDPhi + 0.5 * kAngTol);
  s.sinSPhi = std::sin(fSPhi);
  s.cosSPhi = std::cos(fSPhi);
  s.sinEPhi = std::sin(s.ePhi);
  s.cosEPhi = std::cos(s.ePhi);
  // CheckThetaAngles
  double fSTheta = 0, fDTheta = 0;
  if (!((stheta < 0) || (stheta > kPi))) fSTheta = stheta;
  if (dtheta + stheta >= kPi)
    fDTheta = kPi - stheta;
  else if (dtheta > 0)
    fDTheta = dtheta;
  fullTheta = !(fDTheta - fSTheta < kPi);
  full = fullPhi && fullTheta;
  s.stheta = fSTheta;
  s.dtheta = fDTheta;
  s.eTheta = fSTheta + fDTheta;
  s.sinSTheta = std::sin(fSTheta);
  s.cosSTheta = std::cos(fSTheta);
  s.sinETheta = std::sin(s.eTheta);
  s.cosETheta = std::cos(s.eTheta);
  const double tanS = std::tan(fSTheta), tanE = std::tan(s.eTheta);
  s.tanSTheta2 = tanS * tanS;
  s.tanETheta2 = tanE * tanE;
  // evaluated per point by the reference kernels; constant per shape
  s.cosHDPhi = std::cos(s.hDPhi);
  const double phim = 0.5 * (fSPhi + s.ePhi);
  s.sinPhim = std::sin(phim);
  s.cosPhim = std::cos(phim);
  s.fullPhi = fullPhi;
  s.fullTheta = fullTheta;
  s.full = full;
  // the polar-angle cuts the kernels compare with, as the kernels compute them
  // (Inside: stheta -/+ ht, stheta + dtheta -/+ ht; DistanceToIn: tolSTheta =
  // stheta - ht, tolETheta = eTheta + ht, and those moved inwards by kAngTol)
  const double ht = 0.5 * kAngTol;
  const double eT = fSTheta + fDTheta;
  const double tolS = fSTheta - ht, tolE = s.eTheta + ht;
  const double cuts[kCuts] = {fSTheta - ht, fSTheta + ht, eT - ht, eT + ht,
                              tolS,         tolE,         tolS + kAngTol, tolE - kAngTol};
  for (int k = 0; k < kCuts; ++k) {
    ThetaCut &c = s.cut[k];
    c.c = cuts[k];
    c.sn = std::sin(cuts[k]);
    c.cs = std::cos(cuts[k]);
    c.mode = cuts[k] < 0 ? 1 : (cuts[k] > kPi ? 2 : 0);
  }
  return s;
}

// UnplacedOrb(r) (source/UnplacedOrb.cpp:33-44) reads frTolerance in its
// initialiser list before that member is initialised (members are initialised
// in declaration order, volumes/UnplacedOrb.h:27-35), so the tolerance it
// computes is undefined (garbage memory made it huge in some runs here).  This
// takes the values the reference's own SetRadius (:52-60) computes, with
// frTolerance = 1e-9: fRTolerance = Max(1e-9, fepsilon * fR).
OrbP make_orb(double r) {
  OrbP o;
  std::memset(&o, 0, sizeof(o));
  const double fepsilon = 2e-11, frTolerance = 1e-9;
  o.r = r;
  o.rTolerance = vmax(frTolerance, fepsilon * r);
  o.rTolI = r - o.rTolerance;
  o.rTolO = r + o.rTolerance;
  return o;
}

// UnplacedParallelepiped(x, y, z, alpha, theta, phi), angles in degrees
// (source/UnplacedParallelepiped.cpp:24-65); ctx / cty as the safeties compute
// them (ParallelepipedImplementation.h:270-276)
ParaP make_parallelepiped(double x, double y, double z, double alpha, double theta, double phi) {
  ParaP a;
  std::memset(&a, 0, sizeof(a));
  a.dims.d[0] = x;
  a.dims.d[1] = y;
  a.dims.d[2] = z;
  a.tanAlpha = std::tan(kDegToRad * alpha);
  a.tanThetaCosPhi = std::tan(kDegToRad * theta) * std::cos(kDegToRad * phi);
  a.tanThetaSinPhi = std::tan(kDegToRad * theta) * std::sin(kDegToRad * phi);
  a.ctx = 1.0 / std::sqrt(1. + a.tanAlpha * a.tanAlpha + a.tanThetaCosPhi * a.tanThetaCosPhi);
  a.cty = 1.0 / std::sqrt(1. + a.tanThetaSinPhi * a.tanThetaSinPhi);
  return a;
}

// UnplacedParaboloid(rlo, rhi, dz) -> SetRloAndRhiAndDz
// (source/UnplacedParaboloid.cpp:90-128) and ComputeBoundingBox (:242-245)
ParaboloidP make_paraboloid(double rlo, double rhi, double dz) {
  ParaboloidP q;
  std::memset(&q, 0, sizeof(q));
  q.rlo = rlo;
  q.rhi = rhi;
  q.rlo2 = rlo * rlo;
  q.rhi2 = rhi * rhi;
  q.dz = dz;
  const double dd = 1. / (q.rhi2 - q.rlo2);
  q.a = 2. * dz * dd;
  q.b = -dz * (q.rlo2 + q.rhi2) * dd;
  q.ainv = 1 / q.a;
  q.a2 = q.a * q.a;
  q.tolOz = dz + kHalfTolerance;
  q.dx = vmax(rhi, rlo);
  return q;
}

// UnplacedTrapezoid::fromParametersToCorners (source/UnplacedTrapezoid.cpp:673-685)
void trapezoid_corners(const TrapezoidP &t, double pt[8][3]) {
  const double mz = -t.dz, pz = t.dz;
  const double xs[8] = {mz * t.tthetaCphi - t.dy1 * t.tanAlpha1 - t.dx1,
                        mz * t.tthetaCphi - t.dy1 * t.tanAlpha1 + t.dx1,
                        mz * t.tthetaCphi + t.dy1 * t.tanAlpha1 - t.dx2,
                        mz * t.tthetaCphi + t.dy1 * t.tanAlpha1 + t.dx2,
                        pz * t.tthetaCphi - t.dy2 * t.tanAlpha2 - t.dx3,
                        pz * t.tthetaCphi - t.dy2 * t.tanAlpha2 + t.dx3,
                        pz * t.tthetaCphi + t.dy2 * t.tanAlpha2 - t.dx4,
                        pz * t.tthetaCphi + t.dy2 * t.tanAlpha2 + t.dx4};
  const double ys[4] = {mz * t.tthetaSphi - t.dy1, mz * t.tthetaSphi + t.dy1,
                        pz * t.tthetaSphi - t.dy2, pz * t.tthetaSphi + t.dy2};
  for (int k = 0; k < 8; ++k) {
    pt[k][0] = xs[k];
    pt[k][1] = ys[k / 2];
    pt[k][2] = k < 4 ? mz : pz;
  }
}

// UnplacedTrapezoid::MakePlane (source/UnplacedTrapezoid.cpp:272-330): the
// plane through the quadrilateral p1..p4, its normal (p3 - p1) x (p4 - p2)
// scaled to unit length; the reference's coplanarity check only prints.
static void trapezoid_plane(TrapezoidP &t, int i, const double *p1, const double *p2,
                            const double *p3, const double *p4) {
  const double a = (p3[1] - p1[1]) * (p4[2] - p2[2]) - (p4[1] - p2[1]) * (p3[2] - p1[2]);
  const double b = -(p3[0] - p1[0]) * (p4[2] - p2[2]) + (p4[0] - p2[0]) * (p3[2] - p1[2]);
  const double c = (p3[0] - p1[0]) * (p4[1] - p2[1]) - (p4[0] - p2[0]) * (p3[1] - p1[1]);
  const double norm = 1.0 / std::sqrt(a * a + b * b + c * c);
  t.a[i] = a * norm;
  t.b[i] = b * norm;
  t.c[i] = c * norm;
  t.d[i] = -(t.a[i] * p1[0] + t.b[i] * p1[1] + t.c[i] * p1[2]);
}

// UnplacedTrapezoid::MakePlanes(corners) (source/UnplacedTrapezoid.cpp:215-262):
// -Y, +Y, -X, +X faces
void trapezoid_planes(TrapezoidP &t, const double pt[8][3]) {
  trapezoid_plane(t, 0, pt[0], pt[1], pt[5], pt[4]);
  trapezoid_plane(t, 1, pt[2], pt[6], pt[7], pt[3]);
  trapezoid_plane(t, 2, pt[0], pt[4], pt[6], pt[2]);
  trapezoid_plane(t, 3, pt[1], pt[3], pt[7], pt[5]);
}

// UnplacedTrapezoid(pDz, pTheta, pPhi, pDy1, pDx1, pDx2, pTanAlpha1, pDy2,
// pDx3, pDx4, pTanAlpha2), angles in radians (source/UnplacedTrapezoid.cpp:29-52)
TrapezoidP make_trapezoid(double dz, double theta, double phi, double dy1, double dx1,
                          double dx2, double tanAlpha1, double dy2, double dx3, double dx4,
                          double tanAlpha2) {
  TrapezoidP t;
  std::memset(&t, 0, sizeof(t));
  t.dz = dz;
  t.theta = theta;
  t.phi = phi;
  t.dy1 = dy1;
  t.dx1 = dx1;
  t.dx2 = dx2;
  t.tanAlpha1 = tanAlpha1;
  t.dy2 = dy2;
  t.dx3 = dx3;
  t.dx4 = dx4;
  t.tanAlpha2 = tanAlpha2;
  t.tthetaSphi = std::tan(theta) * std::sin(phi);
  t.tthetaCphi = std::tan(theta) * std::cos(phi);
  double pt[8][3];
  trapezoid_corners(t, pt);
  trapezoid_planes(t, pt);
  return t;
}

// UnplacedTrapezoid(TrapCorners_t) (source/UnplacedTrapezoid.cpp:96-105): the
// planes from the corners as given, then fromCornersToParameters (:651-671)
TrapezoidP make_trapezoid_corners(const double pt[8][3]) {
  TrapezoidP t;
  std::memset(&t, 0, sizeof(t));
  trapezoid_planes(t, pt);
  t.dz = pt[7][2];
  const double dzRecip = 1.0 / t.dz;
  t.dy1 = 0.50 * (pt[2][1] - pt[0][1]);
  t.dx1 = 0.50 * (pt[1][0] - pt[0][0]);
  t.dx2 = 0.50 * (pt[3][0] - pt[2][0]);
  t.tanAlpha1 = 0.25 * (pt[2][0] + pt[3][0] - pt[1][0] - pt[0][0]) / t.dy1;
  t.dy2 = 0.50 * (pt[6][1] - pt[4][1]);
  t.dx3 = 0.50 * (pt[5][0] - pt[4][0]);
  t.dx4 = 0.50 * (pt[7][0] - pt[6][0]);
  t.tanAlpha2 = 0.25 * (pt[6][0] + pt[7][0] - pt[5][0] - pt[4][0]) / t.dy2;
  t.tthetaCphi = (pt[4][0] + t.dy2 * t.tanAlpha2 + t.dx3) * dzRecip;
  t.tthetaSphi = (pt[4][1] + t.dy2) * dzRecip;
  t.theta = std::atan(std::sqrt(t.tthetaSphi * t.tthetaSphi + t.tthetaCphi * t.tthetaCphi));
  t.phi = std::atan2(t.tthetaSphi, t.tthetaCphi);
  return t;
}

// UnplacedTrd::calculateCached (volumes/UnplacedTrd.h:38-51)
TrdP make_trd(double dx1, double dx2, double dy1, double dy2, double dz) {
  TrdP t;
  std::memset(&t, 0, sizeof(t));
  t.dx1 = dx1;
  t.dx2 = dx2;
  t.dy1 = dy1;
  t.dy2 = dy2;
  t.dz = dz;
  t.x2minusx1 = dx2 - dx1;
  t.y2minusy1 = dy2 - dy1;
  t.halfx1plusx2 = 0.5 * (dx1 + dx2);
  t.halfy1plusy2 = 0.5 * (dy1 + dy2);
  t.dztimes2 = dz * 2;
  t.fx = 0.5 * (dx1 - dx2) / dz;
  t.fy = 0.5 * (dy1 - dy2) / dz;
  t.calfx = 1. / std::sqrt(1.0 + t.fx * t.fx);
  t.calfy = 1. / std::sqrt(1.0 + t.fy * t.fy);
  t.varying_y = dy1 != dy2;
  return t;
}

// UnplacedTorus constructor (volumes/UnplacedTorus.h:40-70): cached squares,
// phi wedge and the bounding tube (rtor-rmax-kTolerance, rtor+rmax+kTolerance,
// rmax, sphi, dphi), which DistanceToIn runs as TubeTypes::HollowTube
// (TorusImplementation.h:908-923): rmin always checked, phi never.
TorusP make_torus(double rmin, double rmax, double rtor, double sphi, double dphi) {
  TorusP t;
  std::memset(&t, 0, sizeof(t));
  t.rmin = rmin;
  t.rmax = rmax;
  t.rtor = rtor;
  t.sphi = sphi;
  t.dphi = dphi;
  t.rmin2 = rmin * rmin;
  t.rmax2 = rmax * rmax;
  t.rtor2 = rtor * rtor;
  t.wedge = make_wedge(dphi, sphi);
  t.btube = make_tube(rtor - rmax - kTolerance, rtor + rmax + kTolerance, rmax, sphi, dphi);
  t.btube.has_rmin = 1;
  t.btube.has_phi = 0;
  t.has_phi = dphi < kTwoPi;
  return t;
}

// UnplacedPolycone::Init (source/UnplacedPolycone.cpp:22-165): one cone section
// per pair of consecutive, increasing z planes; equal z planes add no section.
// Returns the record (header, sections, fZs) as a double blob.
std::vector<double> make_polycone(double sphi, double dphi, int nz, const double *rmin,
                                  const double *rmax, const double *z) {
  std::vector<PolySec> secs;
  std::vector<double> zsv;
  double prevZ = z[0], prevRmax = 0, prevRmin = 0;
  int dirZ = 1;
  if (nz > 1 && z[1] < z[0]) dirZ = -1;
  for (int i = 0; i < nz; ++i) {
    const double rMin = rmin[i], rMax = rmax[i], zi = z[i];
    if (i > 0) {
      if (((zi > prevZ) && (dirZ > 0)) || ((zi < prevZ) && (dirZ < 0))) {
        const double dz = (zi - prevZ) / 2;
        PolySec s;
        std::memset(&s, 0, sizeof(s));
        s.cone = make_cone(prevRmin, prevRmax, rMin, rMax, dz, sphi, dphi);
        zsv.push_back(zi);
        const size_t k = zsv.size() - 1;
        s.shift = zsv[k - 1] + 0.5 * (zsv[k] - zsv[k - 1]);
        secs.push_back(s);
      }
    } else {
      zsv.push_back(zi);
    }
    prevZ = zi;
    prevRmin = rMin;
    prevRmax = rMax;
  }
  PolyconeP h;
  std::memset(&h, 0, sizeof(h));
  const int hdr = (int)((sizeof(PolyconeP) + 15) / 16 * 2);
  const int secd = (int)(sizeof(PolySec) / sizeof(double));
  h.nsec = (int32_t)secs.size();
  h.sec_off = hdr;
  h.zs_off = hdr + h.nsec * secd;
  std::vector<double> blob(h.zs_off + zsv.size() + 1, 0.);
  std::memcpy(blob.data(), &h, sizeof(h));
  if (!secs.empty()) std::memcpy(blob.data() + h.sec_off, secs.data(), secs.size() * sizeof(PolySec));
  std::memcpy(blob.data() + h.zs_off, zsv.data(), zsv.size() * sizeof(double));
  return blob;
}

// ---- polyhedron construction (source/UnplacedPolyhedron.cpp:20-175) --------

namespace {
struct HV {
  double x, y, z;
};
HV hv(double x, double y, double z) { return HV{x, y, z}; }
bool operator==(const HV &a, const HV &b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
HV sub(const HV &a, const HV &b) { return hv(a.x - b.x, a.y - b.y, a.z - b.z); }
double dot(const HV &a, const HV &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
double length(const HV &a) { return std::sqrt(dot(a, a)); }
HV scale(const HV &a, double s) { return hv(a.x * s, a.y * s, a.z * s); }
// Vector3D::Normalized (base/Vector3D.h:236-238): multiply by 1/Length
HV normalized(const HV &a) { return scale(a, 1. / length(a)); }
// Vector3D::FixZeroes (base/Vector3D.h:344-349)
HV fix_zeroes(HV a) {
  if (std::fabs(a.x) < kTolerance) a.x = 0.;
  if (std::fabs(a.y) < kTolerance) a.y = 0.;
  if (std::fabs(a.z) < kTolerance) a.z = 0.;
  return a;
}
// Vector3D::Cross (base/Vector3D.h:266-272)
HV cross(const HV &l, const HV &r) {
  return hv(l.y * r.z - l.z * r.y, l.z * r.x - l.x * r.z, l.x * r.y - l.y * r.x);
}
HV from_cylindrical(double r, double phi, double z) {
  return hv(r * std::cos(phi), r * std::sin(phi), z);
}
// NormalizeAngle (volumes/kernel/GenericKernels.h:106-110)
double normalize_angle(double a) { return a + kTwoPi * ((a < 0) - int(a / kTwoPi)); }

void set_quad_corner(PhQuad &q, int k, const HV &c) {
  q.c[k][0] = c.x;
  q.c[k][1] = c.y;
  q.c[k][2] = c.z;
}
HV quad_corner(const PhQuad &q, int k) { return hv(q.c[k][0], q.c[k][1], q.c[k][2]); }

// Quadrilaterals::Set (source/Quadrilaterals.cpp:38-104)
void quad_set(PhQuad &q, const HV &c0, const HV &c1, const HV &c2, const HV &c3) {
  std::memset(&q, 0, sizeof(q));
  set_quad_corner(q, 0, c0);
  set_quad_corner(q, 1, c1);
  set_quad_corner(q, 2, c2);
  set_quad_corner(q, 3, c3);
  HV chosen[4];
  chosen[0] = quad_corner(q, 0);
  int assigned = 1, tested = 1;
  while (tested <= 4) {
    do {
      chosen[assigned] = tested < 4 ? quad_corner(q, tested) : chosen[assigned - 1];
      tested++;
    } while ((chosen[assigned] == chosen[assigned - 1]) && tested < 4);
    assigned++;
    if (assigned == 3) break;
  }
  const HV &a0 = chosen[0], &a1 = chosen[1], &a2 = chosen[2];
  const double a = a0.y * (a1.z - a2.z) + a1.y * (a2.z - a0.z) + a2.y * (a0.z - a1.z);
  const double b = a0.z * (a1.x - a2.x) + a1.z * (a2.x - a0.x) + a2.z * (a0.x - a1.x);
  const double c = a0.x * (a1.y - a2.y) + a1.x * (a2.y - a0.y) + a2.x * (a0.y - a1.y);
  double d = -a0.x * (a1.y * a2.z - a2.y * a1.z) - a1.x * (a2.y * a0.z - a0.y * a2.z) -
             a2.x * (a0.y * a1.z - a1.y * a0.z);
  HV normal = hv(a, b, c);
  const double inv = 1. / length(normal);
  normal = scale(normal, inv);
  d *= inv;
  normal = fix_zeroes(normal);
  q.n[0] = normal.x;
  q.n[1] = normal.y;
  q.n[2] = normal.z;
  q.d = d;
  // ComputeSideVector + Planes::Set(index, normal, origin) (source/Planes.cpp:30-39)
  const HV cs[4] = {c0, c1, c2, c3};
  for (int j = 0; j < 4; ++j) {
    const HV &s0 = cs[j], &s1 = cs[(j + 1) % 4];
    if (!(s1 == s0)) {
      const HV sv = normalized(cross(normal, sub(s1, s0)));
      const HV fixed = fix_zeroes(sv);
      const double il = 1. / length(fixed);
      const HV nn = scale(fixed, il);
      q.sn[j][0] = nn.x;
      q.sn[j][1] = nn.y;
      q.sn[j][2] = nn.z;
      q.sd[j] = il * -dot(fixed, s0);
    } else {
      q.sn[j][0] = q.sn[j][1] = q.sn[j][2] = 0.;
      q.sd[j] = 0.;
    }
  }
}

// Quadrilaterals::FlipSign -> Planes::FlipSign (source/Planes.cpp:48-51)
void quad_flip(PhQuad &q) {
  q.n[0] = -q.n[0];
  q.n[1] = -q.n[1];
  q.n[2] = -q.n[2];
  q.d = -q.d;
}
HV quad_normal(const PhQuad &q) { return hv(q.n[0], q.n[1], q.n[2]); }
}  // namespace

std::vector<double> make_polyhedron(double phiStart, double phiDelta, int sides, int nz,
                                    const double *zPlanes, const double *rMin, const double *rMax) {
  const bool hasPhiCutout = phiDelta < 360;
  const bool largePhiCutout = phiDelta < 180;
  bool hasInnerRadii = false;
  const int nseg = nz - 1;
  std::vector<PhSeg> segs(nseg);
  std::vector<PhQuad> quads;
  std::vector<int> outer_n(nseg), inner_n(nseg), phi_n(nseg), has_inner(nseg);
  for (int i = 0; i < nseg; ++i) {
    has_inner[i] = rMin[i] > 0 || rMin[i + 1] > 0;
    outer_n[i] = sides * ((zPlanes[i] == zPlanes[i + 1] && rMax[i] == rMax[i + 1]) ? 0 : 1);
    phi_n[i] = hasPhiCutout ? 2 * ((zPlanes[i] == zPlanes[i + 1]) ? 0 : 1) : 0;
    const int mult = (zPlanes[i] == zPlanes[i + 1] && rMin[i] == rMin[i + 1]) ? 0 : 1;
    inner_n[i] = 0;
    if (has_inner[i]) {
      inner_n[i] = sides * mult;
      hasInnerRadii = true;
    }
  }
  phiStart = normalize_angle(kDegToRad * phiStart);
  phiDelta *= kDegToRad;
  if (phiDelta > kTwoPi) phiDelta = kTwoPi;
  const double sidePhi = phiDelta / sides;
  std::vector<double> vphi(sides + 1);
  std::vector<HV> phisec(sides + 1);
  for (int i = 0; i < sides + 1; ++i) {
    vphi[i] = normalize_angle(phiStart + i * sidePhi);
    const HV cv = fix_zeroes(normalized(from_cylindrical(1., vphi[i], 0)));
    phisec[i] = cross(normalized(cv), hv(0, 0, -1));
  }
  if (!hasPhiCutout) vphi[sides] = vphi[0];
  const double cosHalfDeltaPhi = std::cos(0.5 * sidePhi);
  double innerRadius = HUGE_VAL, outerRadius = -HUGE_VAL;
  for (int i = 0; i < nz; ++i) {
    if (rMin[i] < innerRadius) innerRadius = rMin[i];
    if (rMax[i] > outerRadius) outerRadius = rMax[i];
  }
  outerRadius /= cosHalfDeltaPhi;
  const double boundingTubeZ = zPlanes[nz - 1] - zPlanes[0] + 2. * kTolerance;
  const double boundsPhiStart = !hasPhiCutout ? 0 : phiStart;
  const double boundsPhiDelta = !hasPhiCutout ? kTwoPi : phiDelta;

  const int nv = nz * (sides + 1);
  std::vector<HV> ov(nv), iv(nv);
  auto vi = [&](int plane, int corner) { return plane * (sides + 1) + corner; };
  for (int i = 0; i < nz; ++i) {
    for (int j = 0, jMax = sides + (hasPhiCutout ? 1 : 0); j < jMax; ++j) {
      ov[vi(i, j)] = fix_zeroes(from_cylindrical(rMax[i] / cosHalfDeltaPhi, vphi[j], zPlanes[i]));
      iv[vi(i, j)] = fix_zeroes(from_cylindrical(rMin[i] / cosHalfDeltaPhi, vphi[j], zPlanes[i]));
    }
    if (!hasPhiCutout) {
      ov[vi(i, sides)] = ov[vi(i, 0)];
      iv[vi(i, sides)] = iv[vi(i, 0)];
    }
  }
  auto wrong_normal = [](const HV &n, const HV &c) { return n.x * c.x + n.y * c.y < 0; };
  for (int p = 0; p < nseg; ++p) {
    PhSeg &s = segs[p];
    std::memset(&s, 0, sizeof(s));
    // Segment p's quadrilaterals start at an index = p (mod 16).  A quadrilateral
    // is 33 doubles, so index mod 16 is its first shared-memory bank pair: the
    // lanes of a warp on the same phi side of different segments then read
    // different banks.  The inserted quadrilaterals are never read.
    while ((int)(quads.size() % 16) != p % 16) {
      PhQuad pad;
      std::memset(&pad, 0, sizeof(pad));
      quads.push_back(pad);
    }
    s.has_inner = has_inner[p];
    s.outer_off = (int32_t)quads.size();
    s.outer_n = outer_n[p];
    for (int k = 0; k < outer_n[p]; ++k) {
      PhQuad q;
      quad_set(q, ov[vi(p, k)], ov[vi(p, k + 1)], ov[vi(p + 1, k + 1)], ov[vi(p + 1, k)]);
      if (wrong_normal(quad_normal(q), ov[vi(p, k)])) quad_flip(q);
      quads.push_back(q);
    }
    s.inner_off = (int32_t)quads.size();
    s.inner_n = inner_n[p];
    for (int k = 0; k < inner_n[p]; ++k) {
      PhQuad q;
      quad_set(q, iv[vi(p, k)], iv[vi(p, k + 1)], iv[vi(p + 1, k + 1)], iv[vi(p + 1, k)]);
      if (wrong_normal(quad_normal(q), iv[vi(p, k)])) quad_flip(q);
      quads.push_back(q);
    }
    s.phi_off = (int32_t)quads.size();
    s.phi_n = phi_n[p];
    if (hasPhiCutout && phi_n[p] == 2) {
      PhQuad q0, q1;
      quad_set(q0, iv[vi(p, 0)], iv[vi(p + 1, 0)], ov[vi(p + 1, 0)], ov[vi(p, 0)]);
      if (dot(quad_normal(q0), phisec[0]) > 0) quad_flip(q0);
      quad_set(q1, ov[vi(p, sides)], ov[vi(p + 1, sides)], iv[vi(p + 1, sides)], iv[vi(p, sides)]);
      if (dot(quad_normal(q1), phisec[sides]) < 0) quad_flip(q1);
      quads.push_back(q0);
      quads.push_back(q1);
    }
  }

  PolyhedronP h;
  std::memset(&h, 0, sizeof(h));
  h.sides = sides;
  h.nseg = nseg;
  h.has_inner_radii = hasInnerRadii;
  h.has_phi_cutout = hasPhiCutout;
  h.large_phi_cutout = largePhiCutout;
  h.btube = make_tube(innerRadius - kTolerance, outerRadius + kTolerance, 0.5 * boundingTubeZ,
                      boundsPhiStart, boundsPhiDelta);
  // HasInnerRadiiTraits (PolyhedronImplementation.h:150-160): HollowTube or
  // NonHollowTube kernels, neither with phi treatment
  h.btube.has_rmin = hasInnerRadii;
  h.btube.has_phi = 0;
  h.btube_offset = zPlanes[0] + 0.5 * boundingTubeZ;
  const int hdr = (int)((sizeof(PolyhedronP) + 15) / 16 * 2);
  h.seg_off = hdr;
  h.quad_off = h.seg_off + (int)((nseg * sizeof(PhSeg) + 15) / 16 * 2);
  h.zp_off = h.quad_off + (int)(quads.size() * sizeof(PhQuad) / sizeof(double));
  h.phisec_off = h.zp_off + nz + (nz % 2);
  std::vector<double> blob(h.phisec_off + 3 * (sides + 1) + 1, 0.);
  std::memcpy(blob.data(), &h, sizeof(h));
  std::memcpy(blob.data() + h.seg_off, segs.data(), nseg * sizeof(PhSeg));
  if (!quads.empty())
    std::memcpy(blob.data() + h.quad_off, quads.data(), quads.size() * sizeof(PhQuad));
  for (int i = 0; i < nz; ++i) blob[h.zp_off + i] = zPlanes[i];
  for (int i = 0; i < sides + 1; ++i) {
    blob[h.phisec_off + 3 * i] = phisec[i].x;
    blob[h.phisec_off + 3 * i + 1] = phisec[i].y;
    blob[h.phisec_off + 3 * i + 2] = phisec[i].z;
  }
  return blob;
}

// Enclosing axis-aligned box of a shape in its own frame (used by the float
// screen of the FP32+refine form; only its enclosure matters).
bool shape_bbox(const vgb_geometry *g, int32_t u, double b[6]) {
  const UnplacedRec &r = g->unplaced[u];
  const double *rec = g->params.data() + r.param_off;
  auto sym = [&](double x, double y, double z) {
    b[0] = -x; b[1] = -y; b[2] = -z; b[3] = x; b[4] = y; b[5] = z;
    return true;
  };
  switch (r.type) {
    case VGB_SHAPE_BOX: {
      const BoxP &p = *reinterpret_cast<const BoxP *>(rec);
      return sym(p.d[0], p.d[1], p.d[2]);
    }
    case VGB_SHAPE_TUBE: {
      const TubeP &p = *reinterpret_cast<const TubeP *>(rec);
      return sym(p.rmax, p.rmax, p.z);
    }
    case VGB_SHAPE_CONE: {
      const ConeP &p = *reinterpret_cast<const ConeP *>(rec);
      const double rm = std::max(p.rmax1, p.rmax2);
      return sym(rm, rm, p.dz);
    }
    case VGB_SHAPE_SPHERE: {
      const SphereP &p = *reinterpret_cast<const SphereP *>(rec);
      return sym(p.rmax, p.rmax, p.rmax);
    }
    case VGB_SHAPE_TORUS: {
      const TorusP &p = *reinterpret_cast<const TorusP *>(rec);
      return sym(p.rtor + p.rmax, p.rtor + p.rmax, p.rmax);
    }
    case VGB_SHAPE_TRD: {
      const TrdP &p = *reinterpret_cast<const TrdP *>(rec);
      return sym(std::max(p.dx1, p.dx2), std::max(p.dy1, p.dy2), p.dz);
    }
    case VGB_SHAPE_ORB: {
      const OrbP &p = *reinterpret_cast<const OrbP *>(rec);
      return sym(p.rTolO, p.rTolO, p.rTolO);
    }
    case VGB_SHAPE_PARABOLOID: {
      const ParaboloidP &p = *reinterpret_cast<const ParaboloidP *>(rec);
      return sym(p.dx, p.dx, p.dz);
    }
    case VGB_SHAPE_TRAPEZOID: {  // the Extent encloses the solid exactly
      double lo[3], hi[3];
      reference_extent(VGB_SHAPE_TRAPEZOID, rec, lo, hi);
      b[0] = lo[0]; b[1] = lo[1]; b[2] = lo[2]; b[3] = hi[0]; b[4] = hi[1]; b[5] = hi[2];
      return true;
    }
    case VGB_SHAPE_PARALLELEPIPED: {
      // the box's corners mapped back through the shear
      const ParaP &p = *reinterpret_cast<const ParaP *>(rec);
      const double z = p.dims.d[2], y = std::fabs(p.dims.d[1]) + std::fabs(p.tanThetaSinPhi) * z;
      const double x = std::fabs(p.dims.d[0]) + std::fabs(p.tanThetaCosPhi) * z +
                       std::fabs(p.tanAlpha) * y;
      return sym(x, y, z);
    }
    case VGB_SHAPE_POLYCONE: {
      const PolyconeP &p = *reinterpret_cast<const PolyconeP *>(rec);
      const PolySec *sec = reinterpret_cast<const PolySec *>(rec + p.sec_off);
      double rm = 0., zlo = 1e300, zhi = -1e300;
      for (int i = 0; i < p.nsec; ++i) {
        rm = std::max(rm, std::max(sec[i].cone.rmax1, sec[i].cone.rmax2));
        zlo = std::min(zlo, sec[i].shift - sec[i].cone.dz);
        zhi = std::max(zhi, sec[i].shift + sec[i].cone.dz);
      }
      b[0] = b[1] = -rm;
      b[3] = b[4] = rm;
      b[2] = zlo;
      b[5] = zhi;
      return p.nsec > 0;
    }
    case VGB_SHAPE_POLYHEDRON: {
      const PolyhedronP &p = *reinterpret_cast<const PolyhedronP *>(rec);
      b[0] = b[1] = -p.btube.rmax;
      b[3] = b[4] = p.btube.rmax;
      b[2] = p.btube_offset - p.btube.z;
      b[5] = p.btube_offset + p.btube.z;
      return true;
    }
    case VGB_SHAPE_BOOLEAN: {
      // the components' boxes moved into the boolean's frame: the left one
      // encloses a subtraction or an intersection, both enclose a union
      const BooleanP &p = *reinterpret_cast<const BooleanP *>(rec);
      b[0] = b[1] = b[2] = 1e300;
      b[3] = b[4] = b[5] = -1e300;
      auto add = [&](const BoolComp &c) {
        if (c.xf.flags & kXfQuirk16A) return false;  // not a rigid motion
        const int32_t off = r.param_off + c.rec_off;
        int32_t u = -1;
        for (size_t k = 0; k < g->unplaced.size(); ++k)
          if (g->unplaced[k].param_off == off) u = (int32_t)k;
        double cb[6];
        if (u < 0 || !shape_bbox(g, u, cb)) return false;
        for (int q = 0; q < 8; ++q) {
          const V3<double> l = {cb[(q & 1) ? 3 : 0], cb[(q & 2) ? 4 : 1], cb[(q & 4) ? 5 : 2]};
          const V3<double> m = xf_inverse_point(c.xf, l);
          const double v[3] = {m.x, m.y, m.z};
          for (int k = 0; k < 3; ++k) {
            b[k] = std::min(b[k], v[k]);
            b[3 + k] = std::max(b[3 + k], v[k]);
          }
        }
        return true;
      };
      if (!add(p.left)) return false;
      if (p.op == VGB_BOOL_UNION && !add(p.right)) return false;
      return true;
    }
    default:
      return false;
  }
}

// UnplacedTube::Extent (source/UnplacedTube.cpp:244-295): the full box, cut
// back on the sides whose axis direction (phi = 0, 90, 180, 270 deg) lies
// outside the phi section.
static void tube_extent(const TubeP &t, double lo[3], double hi[3]) {
  lo[0] = -t.rmax; lo[1] = -t.rmax; lo[2] = -t.z;
  hi[0] = t.rmax; hi[1] = t.rmax; hi[2] = t.z;
  if (t.dphi == 2. * kPi) return;
  const double rin = 0.5 * (t.rmax + t.rmin);
  auto out = [&](double x, double y) {
    bool ci, co;
    WedgeOps<double>::contains_inside<false>(t.wedge, x, y, ci, co);
    return co;
  };
  const bool o0 = out(rin, 0.), o90 = out(0., rin), o180 = out(-rin, 0.), o270 = out(0., -rin);
  if (!(o0 || o90 || o180 || o270)) return;
  const double cx = t.rmax * std::cos(t.sphi), dx = t.rmax * std::cos(t.sphi + t.dphi);
  const double cy = t.rmax * std::sin(t.sphi), dy = t.rmax * std::sin(t.sphi + t.dphi);
  if (o0) hi[0] = vmax(cx, dx);
  if (o90) hi[1] = vmax(cy, dy);
  if (o180) lo[0] = vmin(cx, dx);
  if (o270) lo[1] = vmin(cy, dy);
  if (t.dphi >= kPi) return;
  const double ax = t.rmin * std::cos(t.sphi), bx = t.rmin * std::cos(t.sphi + t.dphi);
  const double ay = t.rmin * std::sin(t.sphi), by = t.rmin * std::sin(t.sphi + t.dphi);
  double v = vmax(ax, bx);
  hi[0] = v > hi[0] ? v : hi[0];
  v = vmax(ay, by);
  hi[1] = v > hi[1] ? v : hi[1];
  v = vmin(ax, bx);
  lo[0] = v < lo[0] ? v : lo[0];
  v = vmin(ay, by);
  lo[1] = v < lo[1] ? v : lo[1];
}

bool reference_extent(int type, const double *rec, double lo[3], double hi[3]) {
  auto set = [&](double x0, double y0, double z0, double x1, double y1, double z1) {
    lo[0] = x0; lo[1] = y0; lo[2] = z0;
    hi[0] = x1; hi[1] = y1; hi[2] = z1;
    return true;
  };
  switch (type) {
    case VGB_SHAPE_BOX: {  // source/UnplacedBox.cpp:29-34
      const BoxP &p = *reinterpret_cast<const BoxP *>(rec);
      return set(-p.d[0], -p.d[1], -p.d[2], p.d[0], p.d[1], p.d[2]);
    }
    case VGB_SHAPE_TUBE:
      tube_extent(*reinterpret_cast<const TubeP *>(rec), lo, hi);
      return true;
    case VGB_SHAPE_CONE: {  // volumes/UnplacedCone.h:324-328
      const ConeP &p = *reinterpret_cast<const ConeP *>(rec);
      const double m = p.rmax1 > p.rmax2 ? p.rmax1 : p.rmax2;
      return set(-m, -m, -p.dz, m, m, p.dz);
    }
    case VGB_SHAPE_SPHERE: {  // source/UnplacedSphere.cpp:174-179
      const SphereP &p = *reinterpret_cast<const SphereP *>(rec);
      return set(-p.rmax, -p.rmax, -p.rmax, p.rmax, p.rmax, p.rmax);
    }
    case VGB_SHAPE_TRAPEZOID: {  // source/UnplacedTrapezoid.cpp:428-466
      const TrapezoidP &p = *reinterpret_cast<const TrapezoidP *>(rec);
      double pt[8][3];
      trapezoid_corners(p, pt);
      // per axis: std::max / std::min of corner pairs, then the pairs' pairs
      for (int ax = 0; ax < 2; ++ax) {
        double e01 = vmax(pt[0][ax], pt[1][ax]), e23 = vmax(pt[2][ax], pt[3][ax]);
        double e45 = vmax(pt[4][ax], pt[5][ax]), e67 = vmax(pt[6][ax], pt[7][ax]);
        double ea = e01 > e23 ? e01 : e23, eb = e45 > e67 ? e45 : e67;
        hi[ax] = ea > eb ? ea : eb;
        e01 = vmin(pt[0][ax], pt[1][ax]);
        e23 = vmin(pt[2][ax], pt[3][ax]);
        e45 = vmin(pt[4][ax], pt[5][ax]);
        e67 = vmin(pt[6][ax], pt[7][ax]);
        ea = e01 < e23 ? e01 : e23;
        eb = e45 < e67 ? e45 : e67;
        lo[ax] = ea < eb ? ea : eb;
      }
      lo[2] = -p.dz;
      hi[2] = p.dz;
      return true;
    }
    case VGB_SHAPE_PARABOLOID: {  // source/UnplacedParaboloid.cpp:169-176
      const ParaboloidP &p = *reinterpret_cast<const ParaboloidP *>(rec);
      return set(-p.dx, -p.dx, -p.dz, p.dx, p.dx, p.dz);
    }
    case VGB_SHAPE_ORB: {  // source/UnplacedOrb.cpp:69-74
      const OrbP &p = *reinterpret_cast<const OrbP *>(rec);
      return set(-p.r, -p.r, -p.r, p.r, p.r, p.r);
    }
    case VGB_SHAPE_TORUS:  // volumes/UnplacedTorus.h:178-180: the bounding tube's
      tube_extent(reinterpret_cast<const TorusP *>(rec)->btube, lo, hi);
      return true;
    case VGB_SHAPE_TRD: {
      // volumes/UnplacedTrd.h:147-150; the upper x bound reads fDY1 where fDX1
      // is meant, kept as the reference computes it
      const TrdP &p = *reinterpret_cast<const TrdP *>(rec);
      return set(-vmax(p.dx1, p.dx2), -vmax(p.dy1, p.dy2), -p.dz, vmax(p.dy1, p.dx2),
                 vmax(p.dy1, p.dy2), p.dz);
    }
    case VGB_SHAPE_POLYCONE: {  // source/UnplacedPolycone.cpp:755-774
      const PolyconeP &p = *reinterpret_cast<const PolyconeP *>(rec);
      const PolySec *sec = reinterpret_cast<const PolySec *>(rec + p.sec_off);
      const double *zs = rec + p.zs_off;
      double m = 0.;
      for (int i = 0; i < p.nsec; ++i) {
        if (m < sec[i].cone.rmax1) m = sec[i].cone.rmax1;
        if (m < sec[i].cone.rmax2) m = sec[i].cone.rmax2;
      }
      return set(-m, -m, zs[0], m, m, zs[p.nsec]);
    }
    case VGB_SHAPE_POLYHEDRON: {  // source/UnplacedPolyhedron.cpp:342-347
      const PolyhedronP &p = *reinterpret_cast<const PolyhedronP *>(rec);
      tube_extent(p.btube, lo, hi);
      lo[2] += p.btube_offset;
      hi[2] += p.btube_offset;
      return true;
    }
    case VGB_SHAPE_BOOLEAN: {
      // source/UnplacedBooleanVolume.cpp:94-121: from the components' extents
      // in their own frames (their placements are not applied): a
      // subtraction's is its left component's, a union's the enclosing box of
      // both, an intersection's their overlap (Min / Max of the bounds)
      const BooleanP &p = *reinterpret_cast<const BooleanP *>(rec);
      double rlo[3], rhi[3];
      if (!reference_extent(p.left.type, rec + p.left.rec_off, lo, hi)) return false;
      if (!reference_extent(p.right.type, rec + p.right.rec_off, rlo, rhi)) return false;
      if (p.op == VGB_BOOL_UNION) {
        for (int k = 0; k < 3; ++k) {
          lo[k] = vmin(lo[k], rlo[k]);
          hi[k] = vmax(hi[k], rhi[k]);
        }
      } else if (p.op == VGB_BOOL_INTERSECTION) {
        for (int k = 0; k < 3; ++k) {
          lo[k] = vmax(lo[k], rlo[k]);
          hi[k] = vmin(hi[k], rhi[k]);
        }
      }
      return true;
    }
    default:
      return false;
  }
}

}  // namespace vgb

// add_unplaced plus the constructor's own arguments, which the flat image and
// the C++ export carry
static vgb_status add_shape(vgb_geometry *g, int type, const void *rec, size_t bytes,
                            int32_t extra, int32_t *id, std::vector<double> args,
                            int32_t form = kCtorDefault) {
  int32_t uid = -1;
  vgb_status s = add_unplaced(g, type, rec, bytes, extra, &uid);
  if (s != VGB_OK) return s;
  g->ctor_form[uid] = form;
  g->ctor_args[uid] = std::move(args);
  if (id) *id = uid;
  return VGB_OK;
}

extern "C" {

vgb_status vgb_unplaced_polyhedron(vgb_geometry *g, double phi_start_deg, double phi_delta_deg,
                                   int32_t sides, int32_t nz, const double *z,
                                   const double *rmin, const double *rmax, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (nz < 2 || sides < 1 || !z || !rmin || !rmax || !(phi_delta_deg > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_polyhedron: need nz >= 2, sides >= 1, phi delta > 0");
  for (int i = 0; i < nz; ++i)
    if (rmin[i] < 0 || !(rmax[i] > 0) || rmin[i] > rmax[i])
      return set_error(VGB_EINVAL, "vgb_unplaced_polyhedron: invalid radii at plane %d", i);
  for (int i = 1; i < nz; ++i)
    if (z[i] < z[i - 1])
      return set_error(VGB_EINVAL, "vgb_unplaced_polyhedron: z planes must not decrease");
  std::vector<double> blob =
      make_polyhedron(phi_start_deg, phi_delta_deg, sides, nz, z, rmin, rmax);
  std::vector<double> args = {phi_start_deg, phi_delta_deg, (double)sides, (double)nz};
  args.insert(args.end(), z, z + nz);
  args.insert(args.end(), rmin, rmin + nz);
  args.insert(args.end(), rmax, rmax + nz);
  return add_shape(g, VGB_SHAPE_POLYHEDRON, blob.data(), blob.size() * sizeof(double), 0, id,
                   std::move(args));
}

vgb_status vgb_unplaced_polycone(vgb_geometry *g, double sphi, double dphi, int32_t nz,
                                 const double *rmin, const double *rmax, const double *z,
                                 int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (nz < 2 || !rmin || !rmax || !z)
    return set_error(VGB_EINVAL, "vgb_unplaced_polycone: need nz >= 2 and the three arrays");
  for (int i = 0; i < nz; ++i)
    if (rmin[i] < 0 || rmax[i] < rmin[i])
      return set_error(VGB_EINVAL, "vgb_unplaced_polycone: rmin[%d] > rmax[%d]", i, i);
  for (int i = 1; i < nz; ++i)
    if (z[i] < z[i - 1])
      return set_error(VGB_EINVAL, "vgb_unplaced_polycone: z planes must not decrease");
  std::vector<double> blob = make_polycone(sphi, dphi, nz, rmin, rmax, z);
  if (reinterpret_cast<const PolyconeP *>(blob.data())->nsec < 1)
    return set_error(VGB_EINVAL, "vgb_unplaced_polycone: no section (all z planes equal)");
  std::vector<double> args = {sphi, dphi, (double)nz};
  args.insert(args.end(), rmin, rmin + nz);
  args.insert(args.end(), rmax, rmax + nz);
  args.insert(args.end(), z, z + nz);
  return add_shape(g, VGB_SHAPE_POLYCONE, blob.data(), blob.size() * sizeof(double), 0, id,
                   std::move(args));
}

vgb_status vgb_unplaced_torus(vgb_geometry *g, double rmin, double rmax, double rtor, double sphi,
                              double dphi, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(rmin >= 0 && rmax > rmin && rtor > rmax && dphi > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_torus: need 0 <= rmin < rmax < rtor, dphi > 0");
  TorusP t = make_torus(rmin, rmax, rtor, sphi, dphi);
  return add_shape(g, VGB_SHAPE_TORUS, &t, sizeof(t), 0, id, {rmin, rmax, rtor, sphi, dphi});
}

vgb_status vgb_unplaced_trd(vgb_geometry *g, double dx1, double dx2, double dy1, double dy2,
                            double dz, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(dx1 >= 0 && dx2 >= 0 && dy1 >= 0 && dy2 >= 0 && dz > 0 && (dx1 > 0 || dx2 > 0) &&
        (dy1 > 0 || dy2 > 0)))
    return set_error(VGB_EINVAL, "vgb_unplaced_trd: invalid half-lengths");
  TrdP t = make_trd(dx1, dx2, dy1, dy2, dz);
  return add_shape(g, VGB_SHAPE_TRD, &t, sizeof(t), 0, id, {dx1, dx2, dy1, dy2, dz});
}

vgb_status vgb_unplaced_orb(vgb_geometry *g, double r, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(r > 0)) return set_error(VGB_EINVAL, "vgb_unplaced_orb: radius must be > 0");
  OrbP o = make_orb(r);
  return add_shape(g, VGB_SHAPE_ORB, &o, sizeof(o), 0, id, {r});
}

vgb_status vgb_unplaced_parallelepiped(vgb_geometry *g, double x, double y, double z,
                                       double alpha_deg, double theta_deg, double phi_deg,
                                       int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(x > 0 && y > 0 && z > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_parallelepiped: half-lengths must be > 0");
  ParaP a = make_parallelepiped(x, y, z, alpha_deg, theta_deg, phi_deg);
  return add_shape(g, VGB_SHAPE_PARALLELEPIPED, &a, sizeof(a), 0, id,
                   {x, y, z, alpha_deg, theta_deg, phi_deg});
}

vgb_status vgb_unplaced_paraboloid(vgb_geometry *g, double rlo, double rhi, double dz,
                                   int32_t *id) {
  VGB_CHECK_OPEN(g);
  // the reference prints an error and keeps zeros for these
  // (source/UnplacedParaboloid.cpp:93-96); here they are refused
  if (!(rlo >= 0 && rhi >= 0 && dz > 0 && rhi != rlo))
    return set_error(VGB_EINVAL, "vgb_unplaced_paraboloid: need rlo, rhi >= 0, rlo != rhi, dz > 0");
  ParaboloidP q = make_paraboloid(rlo, rhi, dz);
  return add_shape(g, VGB_SHAPE_PARABOLOID, &q, sizeof(q), 0, id, {rlo, rhi, dz});
}

vgb_status vgb_unplaced_trapezoid(vgb_geometry *g, double dz, double theta, double phi,
                                  double dy1, double dx1, double dx2, double tan_alpha1,
                                  double dy2, double dx3, double dx4, double tan_alpha2,
                                  int32_t *id) {
  VGB_CHECK_OPEN(g);
  // the reference prints "Invalid input length parameters" and goes on
  // (source/UnplacedTrapezoid.cpp:37-46); here they are refused
  if (!(dz > 0 && dy1 > 0 && dx1 > 0 && dx2 > 0 && dy2 > 0 && dx3 > 0 && dx4 > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_trapezoid: half-lengths must be > 0");
  TrapezoidP t = make_trapezoid(dz, theta, phi, dy1, dx1, dx2, tan_alpha1, dy2, dx3, dx4,
                                tan_alpha2);
  return add_shape(g, VGB_SHAPE_TRAPEZOID, &t, sizeof(t), 0, id,
                   {dz, theta, phi, dy1, dx1, dx2, tan_alpha1, dy2, dx3, dx4, tan_alpha2});
}

vgb_status vgb_unplaced_trapezoid_corners(vgb_geometry *g, const double *corners,
                                          int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!corners) return set_error(VGB_EINVAL, "vgb_unplaced_trapezoid_corners: null corners");
  double pt[8][3];
  std::memcpy(pt, corners, sizeof(pt));
  // the corner layout the reference expects: z = -dz for 0..3, +dz for 4..7
  const double dz = pt[7][2];
  for (int k = 0; k < 8; ++k)
    if (!(pt[k][2] == (k < 4 ? -dz : dz)))
      return set_error(VGB_EINVAL,
                       "vgb_unplaced_trapezoid_corners: corners 0-3 need z = -dz, 4-7 z = +dz");
  if (!(dz > 0 && pt[2][1] > pt[0][1] && pt[1][0] > pt[0][0] && pt[3][0] > pt[2][0] &&
        pt[6][1] > pt[4][1] && pt[5][0] > pt[4][0] && pt[7][0] > pt[6][0]))
    return set_error(VGB_EINVAL, "vgb_unplaced_trapezoid_corners: degenerate corners");
  TrapezoidP t = make_trapezoid_corners(pt);
  return add_shape(g, VGB_SHAPE_TRAPEZOID, &t, sizeof(t), 0, id,
                   std::vector<double>(corners, corners + 24), kCtorCorners);
}

vgb_status vgb_unplaced_sphere(vgb_geometry *g, double rmin, double rmax, double sphi,
                               double dphi, double stheta, double dtheta, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(rmin >= 0 && rmax > rmin && rmax >= 1.1 * kRadTolerance && dphi > 0 && dtheta > 0 &&
        stheta >= 0 && stheta <= kPi))
    return set_error(VGB_EINVAL, "vgb_unplaced_sphere: invalid radii or angles");
  SphereP s = make_sphere(rmin, rmax, sphi, dphi, stheta, dtheta);
  return add_shape(g, VGB_SHAPE_SPHERE, &s, sizeof(s), 0, id,
                   {rmin, rmax, sphi, dphi, stheta, dtheta});
}

vgb_status vgb_unplaced_cone(vgb_geometry *g, double rmin1, double rmax1, double rmin2,
                             double rmax2, double dz, double sphi, double dphi, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(dz > 0 && rmin1 >= 0 && rmin2 >= 0 && rmax1 >= rmin1 && rmax2 >= rmin2 && dphi > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_cone: invalid radii, dz or dphi");
  ConeP c = make_cone(rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi);
  return add_shape(g, VGB_SHAPE_CONE, &c, sizeof(c), 0, id,
                   {rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi});
}

vgb_status vgb_unplaced_box(vgb_geometry *g, double dx, double dy, double dz, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(dx > 0 && dy > 0 && dz > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_box: half-lengths must be > 0");
  BoxP b;
  b.d[0] = dx;
  b.d[1] = dy;
  b.d[2] = dz;
  return add_shape(g, VGB_SHAPE_BOX, &b, sizeof(b), 0, id, {dx, dy, dz});
}

vgb_status vgb_unplaced_tube(vgb_geometry *g, double rmin, double rmax, double dz, double sphi,
                             double dphi, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (!(rmin >= 0 && rmax > rmin && dz > 0 && dphi > 0))
    return set_error(VGB_EINVAL, "vgb_unplaced_tube: need 0 <= rmin < rmax, dz > 0, dphi > 0");
  TubeP t = make_tube(rmin, rmax, dz, sphi, dphi);
  return add_shape(g, VGB_SHAPE_TUBE, &t, sizeof(t), 0, id, {rmin, rmax, dz, sphi, dphi});
}

// ---------------------------------------------------------------------------
// shapes not yet uploaded by this build report VGB_ENOTSUP
// ---------------------------------------------------------------------------
// UnplacedBooleanVolume(op, left, right) (volumes/UnplacedBooleanVolume.h:46-51):
// the components are placed volumes whose transforms and shape records the
// boolean record carries (offsets relative to the record, since the pool
// moves to the device as one block).
vgb_status vgb_unplaced_boolean(vgb_geometry *g, int32_t op, int32_t left_placed,
                                int32_t right_placed, int32_t *id) {
  VGB_CHECK_OPEN(g);
  if (op != VGB_BOOL_SUBTRACTION && op != VGB_BOOL_UNION && op != VGB_BOOL_INTERSECTION)
    return set_error(VGB_EINVAL, "vgb_unplaced_boolean: unknown operation %d", op);
  const int32_t np = (int32_t)g->placed.size();
  if (left_placed < 0 || left_placed >= np || right_placed < 0 || right_placed >= np)
    return set_error(VGB_EINVAL, "vgb_unplaced_boolean: unknown placed volume");
  const PlacedRec &pl = g->placed[left_placed], &pr = g->placed[right_placed];
  const int lt = g->unplaced[pl.unplaced].type, rt = g->unplaced[pr.unplaced].type;
  if (lt == VGB_SHAPE_BOOLEAN || rt == VGB_SHAPE_BOOLEAN)
    return set_error(VGB_ENOTSUP, "vgb_unplaced_boolean: components must be primitive shapes");
  BooleanP b;
  std::memset(&b, 0, sizeof(b));
  b.op = op;
  b.left.xf = g->xforms[pl.xform];
  b.left.type = lt;
  b.right.xf = g->xforms[pr.xform];
  b.right.type = rt;
  b.right_generic = effective_xform(g->raw_xforms[pr.raw_xform], true);
  int32_t uid = -1;
  vgb_status s = add_shape(g, VGB_SHAPE_BOOLEAN, &b, sizeof(b), left_placed, &uid,
                           {(double)op, (double)left_placed, (double)right_placed});
  if (s != VGB_OK) return s;
  const int32_t off = g->unplaced[uid].param_off;
  BooleanP *rec = reinterpret_cast<BooleanP *>(g->params.data() + off);
  rec->left.rec_off = g->unplaced[pl.unplaced].param_off - off;
  rec->right.rec_off = g->unplaced[pr.unplaced].param_off - off;
  if (id) *id = uid;
  return VGB_OK;
}

}  // extern "C"
